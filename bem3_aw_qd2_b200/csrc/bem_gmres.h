// GMRES-based iterative refinement with low-precision LU factors as the
// preconditioner; see bem_gmres.cu.
#pragma once
#include <cuda_runtime.h>
#include <float.h>

#define GMRES_MAXM 32  // largest Krylov dimension per outer step

// z = M^-1 r with the low-precision factors (r, z: n complex FP64, device)
typedef int (*bem_gmres_precond)(void *ctx, const double2 *r, double2 *z, cudaStream_t st);

struct bem_gmres {
  double2 *V = nullptr, *w = nullptr, *r = nullptr;  // Krylov basis (rows), work vectors
  double *h = nullptr, *y = nullptr;                  // projections, least-squares solution
  int cap_n = 0;
  char err[200] = {0};
};

extern "C" {
// Solve A x = b (A row-major n x n complex FP64, b and x n complex FP64 on the
// device; x holds the start and gets the result) to ||b - A x|| <= tol ||b||,
// at most max_outer refinement steps of GMRES(m) on M^-1 A.  Reports the
// outer steps, the Krylov steps in all and the final relative residual.
int bem_gmres_ir(bem_gmres *g, const double *A, int n, const double *b, double *x, int m, double tol, int max_outer,
                 bem_gmres_precond precond, void *pctx, int *outer_steps, int *inner_steps, double *rel_res,
                 cudaStream_t st);
void bem_gmres_free(bem_gmres *g);
}
