// Mixed-precision dense solve (complex FP32 LU on the tensor cores + FP64
// iterative refinement); see bem_mixed.cu.
#pragma once
#include <cublas_v2.h>
#include <cuComplex.h>
#include <cuda_runtime.h>
#include <stddef.h>

// GEMM arithmetic of the LU trailing updates
#define BEM_MIXED_FP32 1    // FP32 CUDA cores
#define BEM_MIXED_TF32 2    // TF32 tensor cores, FP32 accumulation
#define BEM_MIXED_BF16X9 3  // FP32 emulated by three BF16 products on the tensor cores
#define BEM_MIXED_BF16 4    // BF16 tensor cores, FP32 accumulation
#define BEM_MIXED_BLAS_WS (32u << 20)  // cuBLAS workspace bytes per dense system

struct bem_mixed {
  cublasHandle_t blas = nullptr;
  int mode = 0;
  cuComplex *M = nullptr;  // n x n factors, column-major
  size_t M_cap = 0;
  int *piv = nullptr;
  size_t piv_cap = 0;
  cuComplex *R32 = nullptr;
  size_t R32_cap = 0;
  double2 *X = nullptr, *R = nullptr, *D = nullptr;
  size_t X_cap = 0, R_cap = 0, D_cap = 0;
  int *ts_i = nullptr;                 // panel scratch: candidate rows, displaced positions
  size_t ts_i_cap = 0;
  cuComplex *ts_c = nullptr;           // panel scratch: factored top block, displaced rows
  size_t ts_c_cap = 0;
  // the factorisation as a CUDA graph, captured on the first call for a size
  // and its buffers and replayed while they stay the same
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  int g_n = 0, g_mode = 0;
  const void *g_A = nullptr;
  const void *g_M = nullptr, *g_ts = nullptr;
  void *blas_ws = nullptr;             // cuBLAS workspace (no allocation inside a capture)
  unsigned *status = nullptr;          // 0x20: zero pivot
  unsigned long long *norms = nullptr; // max |d|, max |x| of the last refinement step
  char err[256] = {0};                 // the failing call of the last error
};

extern "C" {
int bem_mixed_init(bem_mixed *m, int mode, cudaStream_t st);
void bem_mixed_free(bem_mixed *m);
// round the row-major FP64 matrix A (n x n) to FP32 and factor it
int bem_mixed_factor(bem_mixed *m, const double *A, int n, cudaStream_t st);
// solve A X = B by refinement; B column-major n x nrhs complex FP64, overwritten by X.
// iters / rel_corr: steps taken and max|last correction| / max|x|
int bem_mixed_solve(bem_mixed *m, const double *A, int n, int nrhs, double *B, int max_iter, double tol, int *iters,
                    double *rel_corr, cudaStream_t st);
unsigned bem_mixed_status(bem_mixed *m, cudaStream_t st);
}
