// Mixed-precision dense solve: the complex FP32 LU of bem_lu.cu (tournament-
// pivoting panels, trailing updates, flag-ordered triangular solves, all the
// library's own kernels), FP64 accuracy won back by iterative refinement
// against the FP64-assembled matrix.  Replaces the FP64 LU of the global
// system (b_mkl_solver_pardiso_d, d3qd2_mkl_solver.c:18-148) and of the
// per-domain dpv systems (LAPACKE_zgesv in solve_dpv_bv,
// bem3_aw_qd2_solve_bieq.c:533-653) when a context runs in mixed precision.
//
// The row-major FP64 matrix A is rounded to complex FP32 and factored P M = L U
// (captured as a CUDA graph per matrix and size).  A x = b is then refined:
// each step forms r = b - A x in FP64 (one warp per row of A), solves for the
// correction with the FP32 factors and adds it in FP64, until the correction
// is below the tolerance, stops shrinking, or grows (the caller then falls
// back to FP64 factors).  FP64 stays in the assembly, the residuals and the
// updates.
#include "bem_count.h"
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include "bem_mixed.h"
#include "bem_refine.h"

#define CKC(call)                                                                                   \
  do {                                                                                             \
    cudaError_t _e = (call);                                                                       \
    if (_e != cudaSuccess) {                                                                       \
      snprintf(m->err, sizeof(m->err), "%s (%s:%d)", cudaGetErrorString(_e), __FILE__, __LINE__);  \
      return -1;                                                                                   \
    }                                                                                              \
  } while (0)

static unsigned grid_for(size_t count) {
  const size_t b = (count + 255) / 256;
  return (unsigned)(b < 4096 ? (b ? b : 1) : 4096);
}

__global__ void k_round_c32(const double2 *__restrict__ a, float2 *__restrict__ m, size_t count) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x) {
    const double2 v = a[i];
    m[i] = make_float2((float)v.x, (float)v.y);
  }
}

// x += d (d in FP32, x in FP64); norms[0] = max |d|, norms[1] = max |x|
// (|re| + |im|), +inf in norms[0] if any entry is not finite
// (bem_refine_norms).  Non-negative doubles, +inf included, order as their
// bit patterns, so atomicMax on the bits works.
__global__ void k_axpy_norms(double2 *__restrict__ x, const float2 *__restrict__ d, size_t count,
                             unsigned long long *norms) {
  double md = 0.0, mx = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x) {
    const float2 a = d[i];
    double2 v = x[i];
    v.x += (double)a.x;
    v.y += (double)a.y;
    x[i] = v;
    bem_refine_norms(a.x, a.y, v.x, v.y, &md, &mx);
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
  m->req_mode = mode;
  m->mode = BEM_MIXED_FP32;
  int dev = 0;
  CKC(cudaGetDevice(&dev));
  if (bem_lu_init(&m->lu, dev)) {
    snprintf(m->err, sizeof(m->err), "%s", m->lu.err);
    return -1;
  }
  m->lu_ready = true;
  CKC(cudaMalloc(&m->norms, 2 * sizeof(unsigned long long)));
  CKC(cudaMemsetAsync(m->norms, 0, 2 * sizeof(unsigned long long), st));
  return 0;
}

extern "C" void bem_mixed_free(bem_mixed *m) {
  if (m->lu_ready) bem_lu_free(&m->lu);
  bem_gmres_free(&m->gm);
  bem_tc_free(&m->tc);
  cudaFree(m->M); cudaFree(m->R32); cudaFree(m->X); cudaFree(m->R); cudaFree(m->norms);
  *m = bem_mixed();
}

extern "C" int bem_mixed_factor(bem_mixed *m, const double *A, int n, cudaStream_t st) {
  const size_t count = (size_t)n * n;
  if (grow(m, &m->M, &m->M_cap, count)) return -1;
  k_round_c32<<<grid_for(count), 256, 0, st>>>((const double2 *)A, m->M, count);
  bem_count_launches(1);
  CKC(cudaGetLastError());
  // trailing updates: mode 1 on the CUDA cores; 2 and 4 one TF32 product, 3
  // three split products on the tensor cores (buffers and TMA maps prepared
  // here, outside any capture); a failed set-up leaves the CUDA cores
  m->lu.tc = nullptr;
  m->mode = BEM_MIXED_FP32;
  if (m->req_mode >= BEM_MIXED_TF32) {
    const int nprod = m->req_mode == BEM_MIXED_TF32X3 ? 3 : 1;
    if (bem_tc_prepare(&m->tc, n, nprod) == 0) {
      m->lu.tc = &m->tc;
      m->mode = nprod == 3 ? BEM_MIXED_TF32X3 : BEM_MIXED_TF32;
    }
  }
  if (bem_lu_factor_c(&m->lu, (float *)m->M, n, st)) {
    snprintf(m->err, sizeof(m->err), "%s", m->lu.err);
    return -1;
  }
  return 0;
}

extern "C" int bem_mixed_solve(bem_mixed *m, const double *A, int n, int nrhs, double *B, int max_iter, double tol,
                               int *iters, double *rel_corr, cudaStream_t st) {
  const size_t cnt = (size_t)n * nrhs;
  if (grow(m, &m->R32, &m->R32_cap, cnt) || grow(m, &m->X, &m->X_cap, cnt) || grow(m, &m->R, &m->R_cap, cnt)) return -1;
  CKC(cudaMemsetAsync(m->X, 0, cnt * sizeof(double2), st));
  CKC(cudaMemcpyAsync(m->R, B, cnt * sizeof(double2), cudaMemcpyDeviceToDevice, st));
  int it = 0;
  double rc = 1.0, prev = INFINITY;
  for (; it < max_iter; ++it) {
    // correction d = A^-1 r from the FP32 factors
    k_round_c32<<<grid_for(cnt), 256, 0, st>>>(m->R, m->R32, cnt);
    bem_count_launches(1);
    CKC(cudaGetLastError());
    if (bem_lu_solve_c(&m->lu, (const float *)m->M, n, nrhs, (float *)m->R32, st)) {
      snprintf(m->err, sizeof(m->err), "%s", m->lu.err);
      return -1;
    }
    CKC(cudaMemsetAsync(m->norms, 0, 2 * sizeof(unsigned long long), st));
    k_axpy_norms<<<grid_for(cnt), 256, 0, st>>>(m->X, m->R32, cnt, m->norms);
    bem_count_launches(1);
    CKC(cudaGetLastError());
    // r = b - A x in FP64
    if (bem_lu_resid_z(A, n, nrhs, (const double *)m->X, B, (double *)m->R, st)) {
      snprintf(m->err, sizeof(m->err), "refinement residual launch failed");
      return -1;
    }
    unsigned long long nb[2];
    CKC(cudaMemcpyAsync(nb, m->norms, sizeof(nb), cudaMemcpyDeviceToHost, st));
    CKC(cudaStreamSynchronize(st));
    double dn, xn;
    memcpy(&dn, &nb[0], sizeof(double));
    memcpy(&xn, &nb[1], sizeof(double));
    rc = bem_refine_rel(dn, xn);
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

__global__ void k_widen(const float2 *__restrict__ a, double2 *__restrict__ b, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    b[i] = make_double2((double)a[i].x, (double)a[i].y);
}

// the GMRES-IR preconditioner: z = M^-1 r with the FP32 factors
static int mixed_precond(void *pctx, const double2 *r, double2 *z, cudaStream_t st) {
  bem_mixed *m = (bem_mixed *)pctx;
  const int n = m->gm_n;
  k_round_c32<<<grid_for((size_t)n), 256, 0, st>>>(r, m->R32, (size_t)n);
  bem_count_launches(1);
  if (bem_lu_solve_c(&m->lu, (const float *)m->M, n, 1, (float *)m->R32, st)) return -1;
  k_widen<<<grid_for((size_t)n), 256, 0, st>>>(m->R32, z, n);
  bem_count_launches(1);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int bem_mixed_solve_gmres(bem_mixed *m, const double *A, int n, int nrhs, double *B, double tol, int *iters,
                                     double *rel_res, cudaStream_t st) {
  if (grow(m, &m->R32, &m->R32_cap, (size_t)n) || grow(m, &m->X, &m->X_cap, (size_t)n)) return -1;
  m->gm_n = n;
  int total = 0;
  double worst = 0.0;
  for (int q = 0; q < nrhs; ++q) {
    double *b = B + 2 * (size_t)q * n;
    CKC(cudaMemsetAsync(m->X, 0, (size_t)n * sizeof(double2), st));
    int outer = 0, inner = 0;
    double rr = 0.0;
    if (bem_gmres_ir(&m->gm, A, n, b, (double *)m->X, 20, tol, 10, mixed_precond, m, &outer, &inner, &rr, st)) {
      snprintf(m->err, sizeof(m->err), "%s", m->gm.err);
      return -1;
    }
    CKC(cudaMemcpyAsync(b, m->X, (size_t)n * sizeof(double2), cudaMemcpyDeviceToDevice, st));
    total += inner;
    worst = !(rr <= worst) ? rr : worst;
  }
  *iters = total;
  *rel_res = worst;
  return 0;
}

extern "C" unsigned bem_mixed_status(bem_mixed *m, cudaStream_t st) {
  const unsigned s = bem_lu_status(&m->lu, st);
  return s == 0xffffffffu ? BEM_LU_ST_ZERO : s;
}
