/* PARDISO stand-in for building the reference without MKL.
 *
 * The reference calls PARDISO (d3qd2_src/d3qd2_mkl_solver.c:18-148) on a
 * complex unsymmetric (mtype 13) one-based CSR matrix in three phases:
 * 11 (analysis), 22 (factorisation), 33 (solve), -1 (release).  This stand-in
 * keeps the CSR arrays at phase 22, expands them to a dense row-major matrix at
 * phase 33 and solves with LAPACKE zgesv (partial pivoting).  MKL's scaling,
 * matching, 1e-13 pivot perturbation and two refinement steps are not
 * reproduced; on the well-conditioned BEM systems here the solutions agree to
 * ~1e-12 relative. */
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#include "mkl_pardiso.h"
#include "mkl_lapacke.h"

void PARDISO(void *pt, const MKL_INT *maxfct, const MKL_INT *mnum, const MKL_INT *mtype,
             const MKL_INT *phase, const MKL_INT *n, const void *a, const MKL_INT *ia,
             const MKL_INT *ja, MKL_INT *perm, const MKL_INT *nrhs, MKL_INT *iparm,
             const MKL_INT *msglvl, void *b, void *x, MKL_INT *error)
{
  (void)pt; (void)maxfct; (void)mnum; (void)perm; (void)iparm; (void)msglvl;
  *error = 0;
  if (*mtype != 13 && *mtype != 6) { *error = -3; return; }
  if (*phase != 33 && *phase != 331) return;  /* analysis / factorisation / release: nothing to do */
  MKL_INT N = *n, nr = *nrhs;
  MKL_Complex16 *A = (MKL_Complex16 *)calloc((size_t)N * N, sizeof(MKL_Complex16));
  MKL_INT *ipiv = (MKL_INT *)malloc((size_t)N * sizeof(MKL_INT));
  if (!A || !ipiv) { *error = -2; free(A); free(ipiv); return; }
  const MKL_Complex16 *av = (const MKL_Complex16 *)a;
  for (MKL_INT r = 0; r < N; r++)
    for (MKL_INT k = ia[r] - 1; k < ia[r + 1] - 1; k++) A[(size_t)r * N + (ja[k] - 1)] = av[k];
  MKL_Complex16 *X = (MKL_Complex16 *)x;
  const MKL_Complex16 *B = (const MKL_Complex16 *)b;
  /* PARDISO stores several right-hand sides one after another (column-major
     n x nrhs); the dense matrix is row-major, so solve one column at a time
     with the row-major LAPACKE layout. */
  MKL_INT info = 0;
  for (MKL_INT c = 0; c < nr && info == 0; c++) {
    if (c > 0) {  /* zgesv overwrote A with its LU factors: rebuild it */
      memset(A, 0, (size_t)N * N * sizeof(MKL_Complex16));
      for (MKL_INT r = 0; r < N; r++)
        for (MKL_INT k = ia[r] - 1; k < ia[r + 1] - 1; k++) A[(size_t)r * N + (ja[k] - 1)] = av[k];
    }
    memcpy(X + (size_t)c * N, B + (size_t)c * N, (size_t)N * sizeof(MKL_Complex16));
    info = scipy_LAPACKE_zgesv64_(LAPACK_ROW_MAJOR, N, 1, A, N, ipiv, X + (size_t)c * N, 1);
  }
  if (info != 0) *error = -4;
  free(A); free(ipiv);
}
