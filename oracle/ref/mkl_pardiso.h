/* Stand-in for mkl_pardiso.h.  PARDISO is provided by pardiso_dense.c in this
 * directory: a dense LU solve of the CSR system (see that file). */
#ifndef ORACLE_SHIM_MKL_PARDISO_H
#define ORACLE_SHIM_MKL_PARDISO_H
#include "mkl_types.h"
void PARDISO(void *pt, const MKL_INT *maxfct, const MKL_INT *mnum, const MKL_INT *mtype,
             const MKL_INT *phase, const MKL_INT *n, const void *a, const MKL_INT *ia,
             const MKL_INT *ja, MKL_INT *perm, const MKL_INT *nrhs, MKL_INT *iparm,
             const MKL_INT *msglvl, void *b, void *x, MKL_INT *error);
#endif
