// Mixed-precision dense solve (complex FP32 LU + FP64 iterative refinement);
// see bem_mixed.cu.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include "bem_lu.h"
#include "bem_gmres.h"

// requested arithmetic of the LU trailing updates (bemgpu_set_precision); the
// mode in effect is in bem_mixed.mode
#define BEM_MIXED_FP32 1    // FP32 CUDA cores
#define BEM_MIXED_TF32 2    // one TF32 product on the tensor cores (tcgen05), FP32 accumulation
#define BEM_MIXED_TF32X3 3  // FP32-accurate: three split TF32 products on the tensor cores
#define BEM_MIXED_FAST 4    // a single low-precision product: runs as mode 2

struct bem_mixed {
  int req_mode = 0;          // arithmetic asked for (bemgpu_set_precision)
  int mode = 0;              // arithmetic of the trailing updates in effect
  bem_lu lu;                 // pivoting, panel scratch and captured graph of the FP32 factorisation
  bool lu_ready = false;
  float2 *M = nullptr;       // n x n FP32 factors, row-major
  size_t M_cap = 0;
  float2 *R32 = nullptr;     // residual / correction in FP32
  size_t R32_cap = 0;
  double2 *X = nullptr, *R = nullptr;
  size_t X_cap = 0, R_cap = 0;
  unsigned long long *norms = nullptr;  // max |d|, max |x| of the last refinement step
  bem_gmres gm;                         // GMRES-IR workspace
  bem_tc tc;                            // tensor-core trailing updates (modes 2-4)
  int gm_n = 0;                         // size of the factored system (for the preconditioner)
  char err[256] = {0};
};

extern "C" {
int bem_mixed_init(bem_mixed *m, int mode, cudaStream_t st);
void bem_mixed_free(bem_mixed *m);
// round the row-major FP64 matrix A (n x n) to FP32 and factor it
int bem_mixed_factor(bem_mixed *m, const double *A, int n, cudaStream_t st);
// solve A X = B by refinement; B column-major n x nrhs complex FP64 (nrhs <= 4),
// overwritten by X.  iters / rel_corr: steps taken and max|last correction| / max|x|
int bem_mixed_solve(bem_mixed *m, const double *A, int n, int nrhs, double *B, int max_iter, double tol, int *iters,
                    double *rel_corr, cudaStream_t st);
// the same by GMRES-IR (bem_gmres.cu), one column of B after the other,
// starting from the values in B's place (zero: b itself is not a start);
// iters: Krylov steps in all, rel_res: the largest final ||b - A x|| / ||b||
int bem_mixed_solve_gmres(bem_mixed *m, const double *A, int n, int nrhs, double *B, double tol, int *iters,
                          double *rel_res, cudaStream_t st);
// status bits of the FP32 factorisation since the last call (BEM_LU_ST_ZERO:
// a zero pivot); waits for st
unsigned bem_mixed_status(bem_mixed *m, cudaStream_t st);
}
