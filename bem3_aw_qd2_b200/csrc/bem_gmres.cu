// GMRES-based iterative refinement (GMRES-IR) of a dense complex system with
// low-precision LU factors as the preconditioner: the FP64 accuracy of the
// mixed-precision solves when plain refinement converges slowly or not at all
// (factors of a TF32 trailing update, or an ill-conditioned system).
// No counterpart in the reference, whose solves are FP64 throughout
// (b_mkl_solver_pardiso_d, d3qd2_mkl_solver.c:18-148).
//
// Outer steps: r = b - A x in FP64; the correction d solves A d = r by GMRES
// on the left-preconditioned system M^-1 A d = M^-1 r, M = the FP32 factors,
// with the Krylov basis and its Hessenberg matrix in FP64 (classical
// Gram-Schmidt, applied twice); x += d.  Each Krylov step is one FP64 matvec
// with A, one FP32 solve with the factors, and two projection passes; the
// small least-squares problem (Givens rotations) is solved on the host.
#include "bem_count.h"
#include <cuda_runtime.h>
#include <float.h>
#include <math.h>
#include <stdio.h>
#include <string.h>
#include <complex>
#include <vector>
#include "bem_gmres.h"

#define GM_TH 256

__global__ void k_gm_matvec(const double2 *__restrict__ A, int n, const double2 *__restrict__ v,
                            double2 *__restrict__ y) {
  const int lane = threadIdx.x & 31;
  const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (row >= n) return;
  const double2 *a = A + (size_t)row * n;
  double re = 0.0, im = 0.0;
  for (int c = lane; c < n; c += 32) {
    const double2 x = a[c], z = v[c];
    re = fma(x.x, z.x, fma(-x.y, z.y, re));
    im = fma(x.x, z.y, fma(x.y, z.x, im));
  }
  for (int o = 16; o > 0; o >>= 1) {
    re += __shfl_down_sync(0xffffffffu, re, o);
    im += __shfl_down_sync(0xffffffffu, im, o);
  }
  if (lane == 0) y[row] = make_double2(re, im);
}

// h[i] += sum_r conj(V[i][r]) w[r] for i < j (h zeroed by the caller); V is
// j x n (basis vectors as rows).  Blocks stride over rows; each keeps j
// partial sums and adds them once.
__global__ void k_gm_dots(const double2 *__restrict__ V, int n, int j, const double2 *__restrict__ w,
                          double *__restrict__ h) {
  __shared__ double sre[GM_TH / 32][GMRES_MAXM + 1], sim[GM_TH / 32][GMRES_MAXM + 1];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int i = 0; i < j; ++i) {
    double re = 0.0, im = 0.0;
    const double2 *vi = V + (size_t)i * n;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
      const double2 a = vi[r], b = w[r];
      re = fma(a.x, b.x, fma(a.y, b.y, re));
      im = fma(a.x, b.y, fma(-a.y, b.x, im));
    }
    for (int o = 16; o > 0; o >>= 1) {
      re += __shfl_down_sync(0xffffffffu, re, o);
      im += __shfl_down_sync(0xffffffffu, im, o);
    }
    if (lane == 0) { sre[wid][i] = re; sim[wid][i] = im; }
  }
  __syncthreads();
  if (threadIdx.x < j) {
    double re = 0.0, im = 0.0;
    for (int q = 0; q < GM_TH / 32; ++q) { re += sre[q][threadIdx.x]; im += sim[q][threadIdx.x]; }
    atomicAdd(h + 2 * threadIdx.x, re);
    atomicAdd(h + 2 * threadIdx.x + 1, im);
  }
}

// w -= sum_{i<j} V[i] h[i]; also, with acc, hacc[i] += h[i]
__global__ void k_gm_project(const double2 *__restrict__ V, int n, int j, const double *__restrict__ h,
                             double2 *__restrict__ w) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    double2 x = w[r];
    for (int i = 0; i < j; ++i) {
      const double2 v = V[(size_t)i * n + r];
      const double hr = h[2 * i], hi = h[2 * i + 1];
      x.x -= v.x * hr - v.y * hi;
      x.y -= v.x * hi + v.y * hr;
    }
    w[r] = x;
  }
}

__global__ void k_gm_scale(double2 *__restrict__ dst, const double2 *__restrict__ src, int n, double s) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
    dst[r] = make_double2(src[r].x * s, src[r].y * s);
}

// x += sum_{i<j} V[i] y[i]
__global__ void k_gm_combine(const double2 *__restrict__ V, int n, int j, const double *__restrict__ y,
                             double2 *__restrict__ x) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    double2 a = x[r];
    for (int i = 0; i < j; ++i) {
      const double2 v = V[(size_t)i * n + r];
      a.x += v.x * y[2 * i] - v.y * y[2 * i + 1];
      a.y += v.x * y[2 * i + 1] + v.y * y[2 * i];
    }
    x[r] = a;
  }
}

__global__ void k_gm_resid(const double2 *__restrict__ A, int n, const double2 *__restrict__ x,
                           const double2 *__restrict__ b, double2 *__restrict__ r) {
  const int lane = threadIdx.x & 31;
  const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (row >= n) return;
  const double2 *a = A + (size_t)row * n;
  double re = 0.0, im = 0.0;
  for (int c = lane; c < n; c += 32) {
    const double2 p = a[c], z = x[c];
    re = fma(p.x, z.x, fma(-p.y, z.y, re));
    im = fma(p.x, z.y, fma(p.y, z.x, im));
  }
  for (int o = 16; o > 0; o >>= 1) {
    re += __shfl_down_sync(0xffffffffu, re, o);
    im += __shfl_down_sync(0xffffffffu, im, o);
  }
  if (lane == 0) r[row] = make_double2(b[row].x - re, b[row].y - im);
}

#define CKG(call)                                                                                    \
  do {                                                                                              \
    cudaError_t _e = (call);                                                                        \
    if (_e != cudaSuccess) {                                                                        \
      snprintf(g->err, sizeof(g->err), "GMRES-IR: %s (%s:%d)", cudaGetErrorString(_e), __FILE__, __LINE__); \
      return -1;                                                                                    \
    }                                                                                               \
  } while (0)

static unsigned blocks_for(int n) {
  const int b = (n + GM_TH - 1) / GM_TH;
  return (unsigned)(b < 1184 ? (b ? b : 1) : 1184);
}

extern "C" void bem_gmres_free(bem_gmres *g) {
  cudaFree(g->V); cudaFree(g->w); cudaFree(g->r); cudaFree(g->h); cudaFree(g->y);
  *g = bem_gmres();
}

static int gm_grow(bem_gmres *g, int n) {
  if (g->cap_n >= n) return 0;
  cudaFree(g->V); cudaFree(g->w); cudaFree(g->r); cudaFree(g->h); cudaFree(g->y);
  g->V = g->w = g->r = nullptr;
  g->h = g->y = nullptr;
  g->cap_n = 0;
  CKG(cudaMalloc(&g->V, (size_t)(GMRES_MAXM + 1) * n * sizeof(double2)));
  CKG(cudaMalloc(&g->w, (size_t)n * sizeof(double2)));
  CKG(cudaMalloc(&g->r, (size_t)n * sizeof(double2)));
  CKG(cudaMalloc(&g->h, 2 * (GMRES_MAXM + 1) * sizeof(double)));
  CKG(cudaMalloc(&g->y, 2 * (GMRES_MAXM + 1) * sizeof(double)));
  g->cap_n = n;
  return 0;
}

// |a|^2 of a device vector through the dot kernel
static int gm_norm2(bem_gmres *g, const double2 *a, int n, double *out, cudaStream_t st) {
  CKG(cudaMemsetAsync(g->h, 0, 2 * sizeof(double), st));
  k_gm_dots<<<blocks_for(n), GM_TH, 0, st>>>(a, n, 1, a, g->h);
  bem_count_launches(1);
  double hv[2];
  CKG(cudaMemcpyAsync(hv, g->h, sizeof(hv), cudaMemcpyDeviceToHost, st));
  CKG(cudaStreamSynchronize(st));
  *out = hv[0];
  return 0;
}

typedef std::complex<double> zc;

extern "C" int bem_gmres_ir(bem_gmres *g, const double *Ad, int n, const double *bd, double *xd, int m, double tol,
                            int max_outer, bem_gmres_precond precond, void *pctx, int *outer_steps, int *inner_steps,
                            double *rel_res, cudaStream_t st) {
  if (m < 1) m = 1;
  if (m > GMRES_MAXM) m = GMRES_MAXM;
  if (gm_grow(g, n)) return -1;
  const double2 *A = (const double2 *)Ad, *b = (const double2 *)bd;
  double2 *x = (double2 *)xd;
  const unsigned nb = blocks_for(n), rows_b = (unsigned)((n + 7) / 8);
  double bnorm2 = 0.0;
  if (gm_norm2(g, b, n, &bnorm2, st)) return -1;
  const double bnorm = sqrt(bnorm2);
  int outer = 0, inner = 0;
  double rr = 1.0;
  for (; outer < max_outer; ++outer) {
    // r = b - A x, its size against b
    k_gm_resid<<<rows_b, 256, 0, st>>>(A, n, x, b, g->r);
    bem_count_launches(1);
    CKG(cudaGetLastError());
    double rn2 = 0.0;
    if (gm_norm2(g, g->r, n, &rn2, st)) return -1;
    rr = bnorm > 0.0 ? sqrt(rn2) / bnorm : 0.0;
    if (!(rr <= DBL_MAX)) break;
    if (rr <= tol) break;
    // z = M^-1 r: the first Krylov vector
    if (precond(pctx, g->r, g->w, st)) {
      snprintf(g->err, sizeof(g->err), "GMRES-IR: preconditioner solve failed");
      return -1;
    }
    double z2 = 0.0;
    if (gm_norm2(g, g->w, n, &z2, st)) return -1;
    const double beta = sqrt(z2);
    if (!(beta > 0.0) || !(beta <= DBL_MAX)) break;
    k_gm_scale<<<nb, GM_TH, 0, st>>>(g->V, g->w, n, 1.0 / beta);
    bem_count_launches(1);
    std::vector<zc> H((size_t)(m + 1) * m), cs(m), sn(m), e(m + 1);
    e[0] = beta;
    int j = 0;
    for (; j < m; ++j) {
      // w = M^-1 A v_j
      k_gm_matvec<<<rows_b, 256, 0, st>>>(A, n, g->V + (size_t)j * n, g->r);
      bem_count_launches(1);
      if (precond(pctx, g->r, g->w, st)) {
        snprintf(g->err, sizeof(g->err), "GMRES-IR: preconditioner solve failed");
        return -1;
      }
      // two passes of classical Gram-Schmidt against v_0 .. v_j
      std::vector<double> hsum(2 * (j + 1), 0.0);
      for (int pass = 0; pass < 2; ++pass) {
        CKG(cudaMemsetAsync(g->h, 0, 2 * (j + 1) * sizeof(double), st));
        k_gm_dots<<<nb, GM_TH, 0, st>>>(g->V, n, j + 1, g->w, g->h);
        bem_count_launches(1);
        k_gm_project<<<nb, GM_TH, 0, st>>>(g->V, n, j + 1, g->h, g->w);
        bem_count_launches(1);
        std::vector<double> hv(2 * (j + 1));
        CKG(cudaMemcpyAsync(hv.data(), g->h, hv.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
        CKG(cudaStreamSynchronize(st));
        for (size_t i = 0; i < hv.size(); ++i) hsum[i] += hv[i];
      }
      double wn2 = 0.0;
      if (gm_norm2(g, g->w, n, &wn2, st)) return -1;
      const double hj1 = sqrt(wn2);
      ++inner;
      for (int i = 0; i <= j; ++i) H[(size_t)i * m + j] = zc(hsum[2 * i], hsum[2 * i + 1]);
      H[(size_t)(j + 1) * m + j] = hj1;
      // Givens rotations: the previous ones on column j, then a new one
      for (int i = 0; i < j; ++i) {
        const zc a = H[(size_t)i * m + j], c = H[(size_t)(i + 1) * m + j];
        H[(size_t)i * m + j] = cs[i] * a + sn[i] * c;
        H[(size_t)(i + 1) * m + j] = -std::conj(sn[i]) * a + cs[i] * c;
      }
      const zc a = H[(size_t)j * m + j], c = H[(size_t)(j + 1) * m + j];
      const double den = sqrt(std::norm(a) + std::norm(c));
      if (den == 0.0) { ++j; break; }
      const zc ca = std::abs(a) > 0.0 ? a / std::abs(a) : zc(1.0, 0.0);
      cs[j] = std::abs(a) / den;
      sn[j] = ca * std::conj(c) / den;
      H[(size_t)j * m + j] = ca * den;
      H[(size_t)(j + 1) * m + j] = 0.0;
      e[j + 1] = -std::conj(sn[j]) * e[j];
      e[j] = cs[j] * e[j];
      const bool done = std::abs(e[j + 1]) <= 0.01 * tol * beta || !(hj1 > 0.0);
      if (j + 1 < m && hj1 > 0.0) {
        k_gm_scale<<<nb, GM_TH, 0, st>>>(g->V + (size_t)(j + 1) * n, g->w, n, 1.0 / hj1);
        bem_count_launches(1);
      }
      if (done) { ++j; break; }
    }
    // y = R^-1 e (back substitution), x += V y
    std::vector<zc> yv(j);
    for (int i = j - 1; i >= 0; --i) {
      zc s = e[i];
      for (int l = i + 1; l < j; ++l) s -= H[(size_t)i * m + l] * yv[l];
      yv[i] = s / H[(size_t)i * m + i];
    }
    std::vector<double> yh(2 * j);
    for (int i = 0; i < j; ++i) { yh[2 * i] = yv[i].real(); yh[2 * i + 1] = yv[i].imag(); }
    CKG(cudaMemcpyAsync(g->y, yh.data(), yh.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    k_gm_combine<<<nb, GM_TH, 0, st>>>(g->V, n, j, g->y, x);
    bem_count_launches(1);
    CKG(cudaGetLastError());
  }
  *outer_steps = outer;
  *inner_steps = inner;
  *rel_res = rr;
  return 0;
}
