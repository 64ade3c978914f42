/* Stand-in for Intel MKL's mkl_types.h, just enough for the reference sources
 * (d3qd2_src/d3qd2_mkl_solver.c, bem3_aw_qd2_solve_bieq.c) to compile without
 * MKL.  ILP64 integers, as the reference Makefile selects -DMKL_ILP64. */
#ifndef ORACLE_SHIM_MKL_TYPES_H
#define ORACLE_SHIM_MKL_TYPES_H
typedef long long MKL_INT;
typedef struct { double real, imag; } MKL_Complex16;
typedef struct { float real, imag; } MKL_Complex8;
#endif
