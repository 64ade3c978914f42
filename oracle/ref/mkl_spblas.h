/* Stand-in for mkl_spblas.h: the reference includes it but calls nothing from it. */
#ifndef ORACLE_SHIM_MKL_SPBLAS_H
#define ORACLE_SHIM_MKL_SPBLAS_H
#include "mkl_types.h"
#endif
