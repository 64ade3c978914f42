// Mixed-precision dense solve: complex FP32 LU with its trailing updates on the
// tensor cores, FP64 accuracy won back by iterative refinement against the
// FP64-assembled matrix.  Replaces the FP64 LU of the global system
// (b_mkl_solver_pardiso_d, d3qd2_mkl_solver.c:18-148) and of the per-domain
// dpv systems (LAPACKE_zgesv in solve_dpv_bv, bem3_aw_qd2_solve_bieq.c:533-653)
// when a context runs in mixed precision.
//
// The FP64 matrices are row-major (the layout of the reference's temporary
// files); read as column-major they are the transpose M = A^T.  M is rounded to
// complex FP32 and factored M = P L U by a recursive right-looking LU:
//   rec(j0, w): w <= 32 -> one-CTA panel kernel (partial pivoting, |re|+|im|
//   pivot as LAPACK's icamax); else factor the left half, apply its row swaps
//   to the right half, U12 = L11^-1 A12 (TRSM), A22 -= L21 U12 (GEMM on the
//   tensor cores), factor the right half, apply its swaps to the left half.
// A x = b is then M^T x = b: U^T w = b, L^T v = w, x = P v.  Each refinement
// step forms r = b - A x in FP64 (ZGEMM on the FP64 matrix), solves for the
// correction in FP32 and adds it in FP64.
#include <cublas_v2.h>
#include <cuComplex.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include "bem_mixed.h"

#define LEAF_W 32
#define LEAF_THREADS 1024

// ---------------------------------------------------------------- kernels
__global__ void k_round_c32(const double2 *__restrict__ a, cuComplex *__restrict__ m, size_t count) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x) {
    const double2 v = a[i];
    m[i] = make_cuComplex((float)v.x, (float)v.y);
  }
}

__global__ void k_widen_c64(const cuComplex *__restrict__ m, double2 *__restrict__ a, size_t count) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x) {
    const cuComplex v = m[i];
    a[i] = make_double2(v.x, v.y);
  }
}

// x += d (FP64); norms[0] = max |d|, norms[1] = max |x| (|re| + |im|).
// Non-negative doubles order as their bit patterns, so atomicMax on the bits works.
__global__ void k_axpy_norms(double2 *__restrict__ x, const double2 *__restrict__ d, size_t count,
                             unsigned long long *norms) {
  double md = 0.0, mx = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x) {
    const double2 a = d[i];
    double2 v = x[i];
    v.x += a.x;
    v.y += a.y;
    x[i] = v;
    md = fmax(md, fabs(a.x) + fabs(a.y));
    mx = fmax(mx, fabs(v.x) + fabs(v.y));
  }
  for (int o = 16; o > 0; o >>= 1) {
    md = fmax(md, __shfl_down_sync(0xffffffffu, md, o));
    mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(norms, (unsigned long long)__double_as_longlong(md));
    atomicMax(norms + 1, (unsigned long long)__double_as_longlong(mx));
  }
}

// Panel factorisation of columns [j0, j0 + w), rows [j0, n), one CTA.
__global__ void __launch_bounds__(LEAF_THREADS) k_lu_leaf(cuComplex *__restrict__ M, int n, int j0, int w,
                                                          int *__restrict__ piv, unsigned *status) {
  __shared__ float sv[LEAF_THREADS / 32];
  __shared__ int si[LEAF_THREADS / 32];
  __shared__ cuComplex row[LEAF_W];
  __shared__ int sp;
  const size_t ld = (size_t)n;
  for (int jj = 0; jj < w; ++jj) {
    const int j = j0 + jj;
    cuComplex *col = M + (size_t)j * ld;
    // pivot: the first row of largest |re| + |im| in column j
    float best = -1.f;
    int bi = j;
    for (int i = j + threadIdx.x; i < n; i += blockDim.x) {
      const cuComplex a = col[i];
      const float v = fabsf(a.x) + fabsf(a.y);
      if (v > best) { best = v; bi = i; }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const float ov = __shfl_down_sync(0xffffffffu, best, o);
      const int oi = __shfl_down_sync(0xffffffffu, bi, o);
      if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
    }
    if ((threadIdx.x & 31) == 0) { sv[threadIdx.x >> 5] = best; si[threadIdx.x >> 5] = bi; }
    __syncthreads();
    if (threadIdx.x == 0) {
      float b = sv[0];
      int p = si[0];
      for (int k = 1; k < (int)(blockDim.x >> 5); ++k)
        if (sv[k] > b || (sv[k] == b && si[k] < p)) { b = sv[k]; p = si[k]; }
      if (!(b > 0.f)) { atomicOr(status, 0x20u); p = j; }
      piv[j] = p;
      sp = p;
    }
    __syncthreads();
    const int p = sp;
    // swap rows j and p across the panel, keep row j of the panel in shared memory
    for (int c = threadIdx.x; c < w; c += blockDim.x) {
      cuComplex *cc = M + (size_t)(j0 + c) * ld;
      const cuComplex a = cc[j], b = cc[p];
      cc[j] = b;
      cc[p] = a;
      row[c] = b;
    }
    __syncthreads();
    const cuComplex d = row[jj];
    const float dn = d.x * d.x + d.y * d.y;
    if (dn > 0.f) {
      const cuComplex inv = make_cuComplex(d.x / dn, -d.y / dn);
      for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) {
        const cuComplex l = cuCmulf(col[i], inv);
        col[i] = l;
        for (int c = jj + 1; c < w; ++c) {
          cuComplex *cc = M + (size_t)(j0 + c) * ld;
          cc[i] = cuCsubf(cc[i], cuCmulf(l, row[c]));
        }
      }
    }
    __syncthreads();
  }
}

// Row swaps k in [k0, k1) (sequential, LAPACK order) on columns [c0, c1).
__global__ void k_lu_swaps(cuComplex *__restrict__ M, int n, int k0, int k1, int c0, int c1, const int *__restrict__ piv) {
  const int c = c0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= c1) return;
  cuComplex *cc = M + (size_t)c * n;
  for (int k = k0; k < k1; ++k) {
    const int p = piv[k];
    if (p != k) {
      const cuComplex a = cc[k];
      cc[k] = cc[p];
      cc[p] = a;
    }
  }
}

// x = P v for nrhs columns: the swaps in reverse order
__global__ void k_lu_unpivot(cuComplex *__restrict__ X, int n, int nrhs, const int *__restrict__ piv) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nrhs) return;
  cuComplex *x = X + (size_t)c * n;
  for (int k = n - 1; k >= 0; --k) {
    const int p = piv[k];
    if (p != k) {
      const cuComplex a = x[k];
      x[k] = x[p];
      x[p] = a;
    }
  }
}

// ---------------------------------------------------------------- host driver
static int grid_for(size_t count) {
  size_t g = (count + 255) / 256;
  if (g > 148 * 16) g = 148 * 16;
  return (int)(g ? g : 1);
}

static cublasComputeType_t compute_type(int mode) {
  switch (mode) {
    case BEM_MIXED_TF32: return CUBLAS_COMPUTE_32F_FAST_TF32;
    case BEM_MIXED_BF16X9: return CUBLAS_COMPUTE_32F_EMULATED_16BFX9;
    case BEM_MIXED_BF16: return CUBLAS_COMPUTE_32F_FAST_16BF;
    default: return CUBLAS_COMPUTE_32F;
  }
}

// failures record the call and its status in m->err
#define CKB(x)                                                                    \
  do {                                                                            \
    const cublasStatus_t _s = (x);                                                \
    if (_s != CUBLAS_STATUS_SUCCESS) {                                            \
      snprintf(m->err, sizeof(m->err), "%s: cuBLAS status %d", #x, (int)_s);      \
      return -1;                                                                  \
    }                                                                             \
  } while (0)
#define CKC(x)                                                                    \
  do {                                                                            \
    const cudaError_t _e = (x);                                                   \
    if (_e != cudaSuccess) {                                                      \
      snprintf(m->err, sizeof(m->err), "%s: %s", #x, cudaGetErrorString(_e));     \
      return -1;                                                                  \
    }                                                                             \
  } while (0)

static int rec_lu(bem_mixed *m, int n, int j0, int w, cudaStream_t st) {
  cuComplex *M = m->M;
  if (w <= LEAF_W) {
    k_lu_leaf<<<1, LEAF_THREADS, 0, st>>>(M, n, j0, w, m->piv, m->status);
    CKC(cudaGetLastError());
    return 0;
  }
  int w1 = (w / 2 + LEAF_W - 1) / LEAF_W * LEAF_W;
  if (w1 >= w) w1 = w - LEAF_W;
  const int w2 = w - w1;
  if (rec_lu(m, n, j0, w1, st)) return -1;
  k_lu_swaps<<<(w2 + 127) / 128, 128, 0, st>>>(M, n, j0, j0 + w1, j0 + w1, j0 + w, m->piv);
  CKC(cudaGetLastError());
  const cuComplex one = make_cuComplex(1.f, 0.f), mone = make_cuComplex(-1.f, 0.f);
  const size_t ld = (size_t)n;
  cuComplex *A11 = M + j0 + (size_t)j0 * ld, *A12 = M + j0 + (size_t)(j0 + w1) * ld;
  cuComplex *A21 = M + (j0 + w1) + (size_t)j0 * ld, *A22 = M + (j0 + w1) + (size_t)(j0 + w1) * ld;
  CKB(cublasCtrsm(m->blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N, CUBLAS_DIAG_UNIT, w1, w2, &one, A11, n,
                  A12, n));
  const int rows = n - j0 - w1;
  if (rows > 0) {
    cublasStatus_t gs = cublasGemmEx(m->blas, CUBLAS_OP_N, CUBLAS_OP_N, rows, w2, w1, &mone, A21, CUDA_C_32F, n, A12,
                                     CUDA_C_32F, n, &one, A22, CUDA_C_32F, n, compute_type(m->mode), CUBLAS_GEMM_DEFAULT);
    if (gs == CUBLAS_STATUS_NOT_SUPPORTED && m->mode == BEM_MIXED_BF16X9) {
      // a cuBLAS older than 12.9 in the process has no BF16x9 emulation: TF32 instead
      m->mode = BEM_MIXED_TF32;
      gs = cublasGemmEx(m->blas, CUBLAS_OP_N, CUBLAS_OP_N, rows, w2, w1, &mone, A21, CUDA_C_32F, n, A12, CUDA_C_32F, n,
                        &one, A22, CUDA_C_32F, n, compute_type(m->mode), CUBLAS_GEMM_DEFAULT);
    }
    CKB(gs);
  }
  if (rec_lu(m, n, j0 + w1, w2, st)) return -1;
  k_lu_swaps<<<(w1 + 127) / 128, 128, 0, st>>>(M, n, j0 + w1, j0 + w, j0, j0 + w1, m->piv);
  CKC(cudaGetLastError());
  return 0;
}

template <class T>
static int grow(bem_mixed *m, T **p, size_t *cap, size_t count) {
  if (count <= *cap) return 0;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  CKC(cudaMalloc((void **)p, count * sizeof(T)));
  *cap = count;
  return 0;
}

extern "C" int bem_mixed_init(bem_mixed *m, int mode, cudaStream_t st) {
  *m = bem_mixed();
  m->mode = mode;
  if (cublasCreate(&m->blas) != CUBLAS_STATUS_SUCCESS) return -1;
  CKB(cublasSetStream(m->blas, st));
  CKC(cudaMalloc(&m->status, sizeof(unsigned)));
  CKC(cudaMalloc(&m->norms, 2 * sizeof(unsigned long long)));
  CKC(cudaMemsetAsync(m->status, 0, sizeof(unsigned), st));
  return 0;
}

extern "C" void bem_mixed_free(bem_mixed *m) {
  if (m->blas) cublasDestroy(m->blas);
  cudaFree(m->M); cudaFree(m->piv); cudaFree(m->R32); cudaFree(m->X); cudaFree(m->R); cudaFree(m->D);
  cudaFree(m->status); cudaFree(m->norms);
  *m = bem_mixed();
}

extern "C" int bem_mixed_factor(bem_mixed *m, const double *A, int n, cudaStream_t st) {
  CKB(cublasSetStream(m->blas, st));
  if (grow(m, &m->M, &m->M_cap, (size_t)n * n) || grow(m, &m->piv, &m->piv_cap, (size_t)n)) return -1;
  const size_t count = (size_t)n * n;
  k_round_c32<<<grid_for(count), 256, 0, st>>>((const double2 *)A, m->M, count);
  CKC(cudaGetLastError());
  return rec_lu(m, n, 0, n, st);
}

// B (n x nrhs, column-major complex FP64): right-hand sides in, solutions out
extern "C" int bem_mixed_solve(bem_mixed *m, const double *A, int n, int nrhs, double *B, int max_iter, double tol,
                               int *iters, double *rel_corr, cudaStream_t st) {
  CKB(cublasSetStream(m->blas, st));
  const size_t cnt = (size_t)n * nrhs;
  if (grow(m, &m->R32, &m->R32_cap, cnt) || grow(m, &m->X, &m->X_cap, cnt) || grow(m, &m->R, &m->R_cap, cnt) ||
      grow(m, &m->D, &m->D_cap, cnt))
    return -1;
  const cuComplex one32 = make_cuComplex(1.f, 0.f);
  const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0), mone = make_cuDoubleComplex(-1.0, 0.0);
  CKC(cudaMemsetAsync(m->X, 0, cnt * sizeof(double2), st));
  CKC(cudaMemcpyAsync(m->R, B, cnt * sizeof(double2), cudaMemcpyDeviceToDevice, st));
  int it = 0;
  double rc = 1.0, prev = INFINITY;
  for (; it < max_iter; ++it) {
    // correction d = A^-1 r from the FP32 factors: U^T w = r, L^T v = w, d = P v
    k_round_c32<<<grid_for(cnt), 256, 0, st>>>(m->R, m->R32, cnt);
    CKC(cudaGetLastError());
    CKB(cublasCtrsm(m->blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_T, CUBLAS_DIAG_NON_UNIT, n, nrhs, &one32,
                    m->M, n, m->R32, n));
    CKB(cublasCtrsm(m->blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_T, CUBLAS_DIAG_UNIT, n, nrhs, &one32,
                    m->M, n, m->R32, n));
    k_lu_unpivot<<<(nrhs + 31) / 32, 32, 0, st>>>(m->R32, n, nrhs, m->piv);
    k_widen_c64<<<grid_for(cnt), 256, 0, st>>>(m->R32, m->D, cnt);
    CKC(cudaMemsetAsync(m->norms, 0, 2 * sizeof(unsigned long long), st));
    k_axpy_norms<<<grid_for(cnt), 256, 0, st>>>(m->X, m->D, cnt, m->norms);
    CKC(cudaGetLastError());
    // r = b - A x in FP64 (A row-major = (A^T) column-major, hence op T)
    CKC(cudaMemcpyAsync(m->R, B, cnt * sizeof(double2), cudaMemcpyDeviceToDevice, st));
    CKB(cublasZgemm(m->blas, CUBLAS_OP_T, CUBLAS_OP_N, n, nrhs, n, &mone, (const cuDoubleComplex *)A, n, m->X, n, &one,
                    m->R, n));
    unsigned long long nb[2];
    CKC(cudaMemcpyAsync(nb, m->norms, sizeof(nb), cudaMemcpyDeviceToHost, st));
    CKC(cudaStreamSynchronize(st));
    double dn, xn;
    memcpy(&dn, &nb[0], sizeof(double));
    memcpy(&xn, &nb[1], sizeof(double));
    rc = xn > 0.0 ? dn / xn : 0.0;
    // stop when converged, when the corrections no longer shrink fourfold
    // (the FP64 residual's own accuracy is reached), or when they grow
    // (divergence: the caller falls back to FP64)
    if (rc <= tol || !(rc <= prev * 2.0) || (rc <= 1e-12 && rc > 0.25 * prev)) { ++it; break; }
    prev = rc;
  }
  *iters = it;
  *rel_corr = rc;
  CKC(cudaMemcpyAsync(B, m->X, cnt * sizeof(double2), cudaMemcpyDeviceToDevice, st));
  return 0;
}

extern "C" unsigned bem_mixed_status(bem_mixed *m, cudaStream_t st) {
  unsigned s = 0;
  cudaMemcpyAsync(&s, m->status, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
  cudaStreamSynchronize(st);
  cudaMemsetAsync(m->status, 0, sizeof(unsigned), st);
  return s;
}
