/* Stand-in for mkl_lapacke.h: LAPACKE_zgesv routed to the ILP64 OpenBLAS that
 * ships inside numpy (symbol scipy_LAPACKE_zgesv64_). */
#ifndef ORACLE_SHIM_MKL_LAPACKE_H
#define ORACLE_SHIM_MKL_LAPACKE_H
#include "mkl_types.h"
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102
MKL_INT scipy_LAPACKE_zgesv64_(int layout, MKL_INT n, MKL_INT nrhs, MKL_Complex16 *a,
                               MKL_INT lda, MKL_INT *ipiv, MKL_Complex16 *b, MKL_INT ldb);
#define LAPACKE_zgesv scipy_LAPACKE_zgesv64_
#endif
