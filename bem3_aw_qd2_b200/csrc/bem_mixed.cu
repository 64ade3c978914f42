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
//   rec(j0, w): w <= 32 -> panel factorisation with tournament pivoting
//   (|re|+|im| pivot as LAPACK's icamax within each selection, below), whose
//   row permutation goes to every other column at once; else factor the left
//   half, U12 = L11^-1 A12 (TRSM), A22 -= L21 U12 (GEMM on the tensor cores),
//   factor the right half.
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
#include "bem_refine.h"

#define LEAF_W 32

// ---------------------------------------------------------------- kernels
__global__ void k_round_c32(const double2 *__restrict__ a, cuComplex *__restrict__ m, size_t count) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x) {
    const double2 v = a[i];
    m[i] = make_cuComplex((float)v.x, (float)v.y);
  }
}

// x += d (FP64); norms[0] = max |d|, norms[1] = max |x| (|re| + |im|), +inf in
// norms[0] if any entry is not finite (bem_refine_norms).  Non-negative
// doubles, +inf included, order as their bit patterns, so atomicMax on the
// bits works.
__global__ void k_axpy_norms(double2 *__restrict__ x, const double2 *__restrict__ d, size_t count,
                             unsigned long long *norms) {
  double md = 0.0, mx = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x) {
    const double2 a = d[i];
    double2 v = x[i];
    v.x += a.x;
    v.y += a.y;
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

// ---------------------------------------------------------------- tournament panel
// The panel (rows [j0, n), w <= 32 columns) is factored with tournament
// pivoting (communication-avoiding LU): chunks of at most TS_ROWS rows each
// pick w candidate pivot rows by partial pivoting (many CTAs), the candidates
// are reduced the same way until one set remains, whose partial-pivoting LU
// gives the panel's w pivots in order and the packed top block L11\U11; every
// other row r of the panel becomes L21 = a_r U11^-1.  The pivots are recorded
// as LAPACK's sequential row swaps (piv) and as their net permutation of the
// touched rows, which is applied at once to every other column (the
// right-looking recursion may apply a panel's swaps to any column before that
// column is next used) and to the row map gid (position -> original row) that
// the solves use.  With the FP64 refinement behind it the weaker growth bound
// of tournament pivoting costs nothing measurable; a refinement that does not
// converge falls back to FP64.
#define TS_ROWS 256
#define TS_THREADS 256
#define TS_NP (2 * LEAF_W)          // touched positions of one panel, at most
#define TS_LIST (1 + 2 * TS_NP)     // count, positions, source positions

// Partial-pivoting LU of the rr <= blockDim.x rows held one per thread (row
// t in thread t: values v, original row id), w columns (columns >= w are
// zero).  Afterwards thread k < min(w, rr) holds the k-th pivot row, packed
// (multipliers left of k, U from k on).  Two barriers per step; the shared
// buffers alternate between steps so that no third one is needed.
struct ts_shared {
  float wv[2][TS_THREADS / 32];
  int wi[2][TS_THREADS / 32];
  cuComplex prow[2][LEAF_W], krow[2][LEAF_W];
  int pid[2], kid[2];
};
// The row of each thread is kept rotated: at step k its register 0 holds
// column k, registers 1 .. 31 - k the columns still to be updated and the
// registers after them the finished columns (multipliers, or U for a pivot
// row).  Each step rotates every row left by one, so all register indices are
// compile-time constants while the step stays one short loop body (fully
// unrolled steps, each executed once per launch, stalled on instruction fetch:
// twice the time); after the last step the rows are rotated back.
__device__ __forceinline__ void ts_rotate(cuComplex (&v)[LEAF_W]) {
  const cuComplex f = v[0];
#pragma unroll
  for (int c = 0; c < LEAF_W - 1; ++c) v[c] = v[c + 1];
  v[LEAF_W - 1] = f;
}
__device__ void ts_gepp(cuComplex (&v)[LEAF_W], int &id, int rr, int w, unsigned *status, ts_shared &sh) {
  const int t = threadIdx.x, lane = t & 31, wid = t >> 5, nw = blockDim.x >> 5;
  const int kmax = min(w, rr);
  for (int k = 0; k < kmax; ++k) {
    const int b = k & 1;
    float val = -1.f;
    if (t >= k && t < rr) val = fabsf(v[0].x) + fabsf(v[0].y);
    int bi = t;
    for (int o = 16; o > 0; o >>= 1) {
      const float ov = __shfl_down_sync(0xffffffffu, val, o);
      const int oi = __shfl_down_sync(0xffffffffu, bi, o);
      if (ov > val || (ov == val && oi < bi)) { val = ov; bi = oi; }
    }
    if (lane == 0) { sh.wv[b][wid] = val; sh.wi[b][wid] = bi; }
    __syncthreads();
    float best = sh.wv[b][0];
    int p = sh.wi[b][0];
    for (int q = 1; q < nw; ++q) {
      const float ov = sh.wv[b][q];
      const int oi = sh.wi[b][q];
      if (ov > best || (ov == best && oi < p)) { best = ov; p = oi; }
    }
    if (!(best > 0.f)) {
      if (status && t == 0) atomicOr(status, 0x20u);
      p = k;
    }
    if (t == p) {
#pragma unroll
      for (int c = 0; c < LEAF_W; ++c) sh.prow[b][c] = v[c];
      sh.pid[b] = id;
    }
    if (t == k) {
#pragma unroll
      for (int c = 0; c < LEAF_W; ++c) sh.krow[b][c] = v[c];
      sh.kid[b] = id;
    }
    __syncthreads();
    if (t == k) {
#pragma unroll
      for (int c = 0; c < LEAF_W; ++c) v[c] = sh.prow[b][c];
      id = sh.pid[b];
    } else if (t == p) {
#pragma unroll
      for (int c = 0; c < LEAF_W; ++c) v[c] = sh.krow[b][c];
      id = sh.kid[b];
    }
    const cuComplex d = sh.prow[b][0];
    const float dn = d.x * d.x + d.y * d.y;
    if (t > k && t < rr && dn > 0.f) {
      const cuComplex l = cuCmulf(v[0], make_cuComplex(d.x / dn, -d.y / dn));
      v[0] = l;
#pragma unroll
      for (int c = 1; c < LEAF_W; ++c)
        if (c < LEAF_W - k) v[c] = cuCsubf(v[c], cuCmulf(l, sh.prow[b][c]));
    }
    ts_rotate(v);
  }
  for (int k = kmax; k < LEAF_W; ++k) ts_rotate(v);
  __syncthreads();
}

__device__ __forceinline__ void ts_load_row(const cuComplex *__restrict__ M, int n, int j0, int w, int row,
                                            cuComplex (&v)[LEAF_W]) {
#pragma unroll
  for (int c = 0; c < LEAF_W; ++c)
    v[c] = (row >= 0 && c < w) ? M[(size_t)(j0 + c) * n + row] : make_cuComplex(0.f, 0.f);
}

// Stage 1: chunk b = rows [j0 + b TS_ROWS, ...) picks its candidates cand[b w + k] (-1 past its rows).
__global__ void __launch_bounds__(TS_THREADS) k_ts_chunk(const cuComplex *__restrict__ M, int n, int j0, int w,
                                                         int *__restrict__ cand) {
  __shared__ ts_shared sh;
  const int row0 = j0 + blockIdx.x * TS_ROWS;
  const int rr = min(TS_ROWS, n - row0);
  int id = (int)threadIdx.x < rr ? row0 + (int)threadIdx.x : -1;
  cuComplex v[LEAF_W];
  ts_load_row(M, n, j0, w, id, v);
  ts_gepp(v, id, rr, w, nullptr, sh);
  if (threadIdx.x < w) cand[blockIdx.x * w + threadIdx.x] = threadIdx.x < rr ? id : -1;
}

// Stage 2: group g of `group` (<= blockDim.x) candidate entries (rows of the
// panel; cin == nullptr: all rows [j0, n)) -> its w winners; the last stage
// (one group) also writes the packed top block (top[k w + c], row k = k-th
// pivot), the sequential swaps piv[j0 .. j0+w), the panel's net permutation
// (list: count, positions, source positions), the rows that it moves below
// the top block (disp: count, positions; dval: their original values), and
// updates the row map gid.
__global__ void __launch_bounds__(TS_THREADS) k_ts_reduce(const cuComplex *__restrict__ M, int n, int j0, int w,
                                                          const int *__restrict__ cin, int nin, int group,
                                                          int *__restrict__ cout, int last, cuComplex *__restrict__ top,
                                                          int *__restrict__ piv, int *__restrict__ list,
                                                          int *__restrict__ disp, cuComplex *__restrict__ dval,
                                                          int *__restrict__ gid, unsigned *status) {
  __shared__ ts_shared sh;
  __shared__ int wc[TS_THREADS / 32];
  __shared__ int rows[TS_THREADS];
  __shared__ int win[LEAF_W];
  __shared__ int cnt, nd;
  __shared__ int drow[LEAF_W];
  const unsigned F = 0xffffffffu;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  {  // the group's valid entries, compacted in order
    const int e = blockIdx.x * group + threadIdx.x;
    int r = -1;
    if (threadIdx.x < group && e < nin) r = cin ? cin[e] : j0 + e;
    const unsigned b = __ballot_sync(F, r >= 0);
    if (lane == 0) wc[wid] = __popc(b);
    __syncthreads();
    if (threadIdx.x == 0) {
      int acc = 0;
      for (int q = 0; q < (int)(blockDim.x >> 5); ++q) { const int c = wc[q]; wc[q] = acc; acc += c; }
      cnt = acc;
    }
    __syncthreads();
    if (r >= 0) rows[wc[wid] + __popc(b & ((1u << lane) - 1u))] = r;
    __syncthreads();
  }
  const int rr = cnt;
  int id = threadIdx.x < rr ? rows[threadIdx.x] : -1;
  cuComplex v[LEAF_W];
  ts_load_row(M, n, j0, w, id, v);
  ts_gepp(v, id, rr, w, last ? status : nullptr, sh);
  if (!last) {
    if (threadIdx.x < w) cout[blockIdx.x * w + threadIdx.x] = threadIdx.x < rr ? id : -1;
    return;
  }
  if (threadIdx.x < w) {
#pragma unroll
    for (int c = 0; c < LEAF_W; ++c)
      if (c < w) top[threadIdx.x * w + c] = v[c];
    win[threadIdx.x] = id;
  }
  __syncthreads();
  if (wid == 0) {
    // LAPACK's sequential swaps: at step k the row win[k], wherever the
    // earlier swaps put it, moves to position j0 + k.  The touched positions
    // (at most 2w) are tracked by one warp, two (position, row) entries a lane.
    int pA = -1, rA = -1, pB = -1, rB = -1, np = 0;
    for (int k = 0; k < w; ++k) {
      const int target = j0 + k, want = win[k];
      const unsigned wa = __ballot_sync(F, rA == want), wb = __ballot_sync(F, rB == want);
      int cur = want;
      if (wa) cur = __shfl_sync(F, pA, __ffs(wa) - 1);
      else if (wb) cur = __shfl_sync(F, pB, __ffs(wb) - 1);
      int q2[2];
      const int look[2] = {target, cur};
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const unsigned fa = __ballot_sync(F, pA == look[h]), fb = __ballot_sync(F, pB == look[h]);
        int q = fa ? __ffs(fa) - 1 : (fb ? 32 + __ffs(fb) - 1 : -1);
        if (q < 0) {  // untouched so far: it holds its own row
          q = np++;
          if (lane == (q & 31)) {
            if (q < 32) { pA = look[h]; rA = look[h]; } else { pB = look[h]; rB = look[h]; }
          }
        }
        q2[h] = q;
      }
      if (lane == 0) piv[target] = cur;
      const int rt = __shfl_sync(F, q2[0] < 32 ? rA : rB, q2[0] & 31);
      const int rc = __shfl_sync(F, q2[1] < 32 ? rA : rB, q2[1] & 31);
      if (lane == (q2[0] & 31)) { if (q2[0] < 32) rA = rc; else rB = rc; }
      if (lane == (q2[1] & 31)) { if (q2[1] < 32) rA = rt; else rB = rt; }
    }
    // net permutation: position p now holds the row that was at position r
    if (lane == 0) list[0] = np;
    if (pA >= 0) { list[1 + lane] = pA; list[1 + TS_NP + lane] = rA; }
    if (pB >= 0) { list[1 + 32 + lane] = pB; list[1 + TS_NP + 32 + lane] = rB; }
    // the row map follows: all reads before the writes
    const int gA = pA >= 0 ? gid[rA] : 0, gB = pB >= 0 ? gid[rB] : 0;
    __syncwarp();
    if (pA >= 0) gid[pA] = gA;
    if (pB >= 0) gid[pB] = gB;
    // rows moved below the top block: (position, original position)
    const bool da = pA >= j0 + w && rA != pA, db = pB >= j0 + w && rB != pB;
    const unsigned ba = __ballot_sync(F, da), bb = __ballot_sync(F, db);
    const int na = __popc(ba);
    const unsigned below = (1u << lane) - 1u;
    if (da) { const int q = __popc(ba & below); disp[1 + q] = pA; drow[q] = rA; }
    if (db) { const int q = na + __popc(bb & below); disp[1 + q] = pB; drow[q] = rB; }
    if (lane == 0) { nd = na + __popc(bb); disp[0] = na + __popc(bb); }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < nd * w; t += blockDim.x) {
    const int q = t / w, c = t % w;
    dval[t] = M[(size_t)(j0 + c) * n + drow[q]];
  }
}

// Stage 3: write the top block and L21 = a U11^-1 for every row below it.
__global__ void __launch_bounds__(128) k_ts_apply(cuComplex *__restrict__ M, int n, int j0, int w,
                                                  const cuComplex *__restrict__ top, const int *__restrict__ disp,
                                                  const cuComplex *__restrict__ dval) {
  __shared__ cuComplex U[LEAF_W][LEAF_W + 1];
  __shared__ cuComplex rdiag[LEAF_W];
  __shared__ int dp[LEAF_W + 1];
  for (int t = threadIdx.x; t < w * w; t += blockDim.x) U[t / w][t % w] = top[t];
  if (threadIdx.x <= LEAF_W) dp[threadIdx.x] = threadIdx.x <= disp[0] ? disp[threadIdx.x] : -1;
  __syncthreads();
  if (threadIdx.x < w) {
    const cuComplex d = U[threadIdx.x][threadIdx.x];
    const float dn = d.x * d.x + d.y * d.y;
    rdiag[threadIdx.x] = dn > 0.f ? make_cuComplex(d.x / dn, -d.y / dn) : make_cuComplex(0.f, 0.f);
  }
  __syncthreads();
  const int i = j0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (i < j0 + w) {
    for (int c = 0; c < w; ++c) M[(size_t)(j0 + c) * n + i] = U[i - j0][c];
    return;
  }
  int m = -1;
  for (int q = 0; q < dp[0]; ++q)
    if (dp[1 + q] == i) m = q;
  // all loads first, then the substitution, then the stores
  cuComplex x[LEAF_W];
#pragma unroll
  for (int c = 0; c < LEAF_W; ++c)
    x[c] = c < w ? (m >= 0 ? dval[m * w + c] : M[(size_t)(j0 + c) * n + i]) : make_cuComplex(0.f, 0.f);
#pragma unroll
  for (int c = 0; c < LEAF_W; ++c) {
    cuComplex a = x[c];
#pragma unroll
    for (int k = 0; k < c; ++k) a = cuCsubf(a, cuCmulf(x[k], U[k][c]));
    x[c] = cuCmulf(a, rdiag[c]);
  }
#pragma unroll
  for (int c = 0; c < LEAF_W; ++c)
    if (c < w) M[(size_t)(j0 + c) * n + i] = x[c];
}

// The panel's net row permutation on the columns outside it ([0, j0) and
// [j0 + w, n)): block = TS_NP list entries x 4 columns, all loads before all stores.
__global__ void __launch_bounds__(TS_NP * 4) k_lu_perm(cuComplex *__restrict__ M, int n, int j0, int w,
                                                       const int *__restrict__ list) {
  const int q = threadIdx.x % TS_NP, cc = blockIdx.x * 4 + threadIdx.x / TS_NP;
  const int col = cc < j0 ? cc : cc + w;
  const int np = list[0];
  const bool on = q < np && col < n;
  cuComplex a = make_cuComplex(0.f, 0.f);
  if (on) a = M[(size_t)col * n + list[1 + TS_NP + q]];
  __syncthreads();
  if (on) M[(size_t)col * n + list[1 + q]] = a;
}

__global__ void k_iota(int *__restrict__ g, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) g[i] = i;
}

// x = P v in FP64: D[gid[i]] = v[i] (row i of the factored matrix is row gid[i] of M)
__global__ void k_unpivot_widen(const cuComplex *__restrict__ V, double2 *__restrict__ D, int n, int nrhs,
                                const int *__restrict__ gid) {
  const size_t cnt = (size_t)n * nrhs;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < cnt; e += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(e % n);
    const size_t c = e / n;
    const cuComplex v = V[e];
    D[c * n + gid[i]] = make_double2(v.x, v.y);
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

// candidate-list capacity of one stage for n rows
static size_t ts_ncand(int n) { return (size_t)((n + TS_ROWS - 1) / TS_ROWS) * LEAF_W; }
// ts_i layout: candidates (2 stages), disp, net-permutation list, row map gid
static size_t ts_ints(int n) { return 2 * ts_ncand(n) + 1 + LEAF_W + TS_LIST + (size_t)n; }
static int *ts_gid(bem_mixed *m, int n) { return m->ts_i + 2 * ts_ncand(n) + 1 + LEAF_W + TS_LIST; }

// panel [j0, n) x [j0, j0 + w): chunks -> reductions -> final selection -> L21,
// then the panel's row permutation on every other column
static int ts_panel(bem_mixed *m, int n, int j0, int w, cudaStream_t st) {
  const int rows = n - j0;
  const size_t nc = ts_ncand(n);
  int *in = m->ts_i, *out = m->ts_i + nc, *disp = m->ts_i + 2 * nc, *list = disp + 1 + LEAF_W;
  cuComplex *top = m->ts_c, *dval = m->ts_c + LEAF_W * LEAF_W;
  int nin = rows;
  if (rows > TS_ROWS) {
    const int nb = (rows + TS_ROWS - 1) / TS_ROWS;
    k_ts_chunk<<<nb, TS_THREADS, 0, st>>>(m->M, n, j0, w, in);
    CKC(cudaGetLastError());
    nin = nb * w;
    while (nin > TS_ROWS) {
      const int ng = (nin + TS_ROWS - 1) / TS_ROWS;
      k_ts_reduce<<<ng, TS_THREADS, 0, st>>>(m->M, n, j0, w, in, nin, TS_ROWS, out, 0, nullptr, nullptr, nullptr,
                                             nullptr, nullptr, nullptr, nullptr);
      CKC(cudaGetLastError());
      nin = ng * w;
      int *t = in; in = out; out = t;
    }
  } else {
    in = nullptr;  // all rows of the panel are the candidates
  }
  // the final selection with as many warps as it has candidate rows: its 32
  // steps cost barriers and instructions per warp, not per row
  const int fthreads = nin >= TS_THREADS ? TS_THREADS : ((nin + 31) / 32 * 32 < 64 ? 64 : (nin + 31) / 32 * 32);
  k_ts_reduce<<<1, fthreads, 0, st>>>(m->M, n, j0, w, in, nin, fthreads, nullptr, 1, top, m->piv, list, disp, dval,
                                      ts_gid(m, n), m->status);
  CKC(cudaGetLastError());
  k_ts_apply<<<(rows + 127) / 128, 128, 0, st>>>(m->M, n, j0, w, top, disp, dval);
  CKC(cudaGetLastError());
  if (n > w) {
    k_lu_perm<<<(n - w + 3) / 4, TS_NP * 4, 0, st>>>(m->M, n, j0, w, list);
    CKC(cudaGetLastError());
  }
  return 0;
}

static int rec_lu(bem_mixed *m, int n, int j0, int w, cudaStream_t st) {
  cuComplex *M = m->M;
  if (w <= LEAF_W) return ts_panel(m, n, j0, w, st);
  int w1 = (w / 2 + LEAF_W - 1) / LEAF_W * LEAF_W;
  if (w1 >= w) w1 = w - LEAF_W;
  const int w2 = w - w1;
  if (rec_lu(m, n, j0, w1, st)) return -1;  // its row swaps are already on every column
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
  return rec_lu(m, n, j0 + w1, w2, st);
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
  // cuBLAS gets its workspace up front: a captured factorisation may not allocate
  CKC(cudaMalloc(&m->blas_ws, BEM_MIXED_BLAS_WS));
  CKB(cublasSetWorkspace(m->blas, m->blas_ws, BEM_MIXED_BLAS_WS));
  CKC(cudaMalloc(&m->status, sizeof(unsigned)));
  CKC(cudaMalloc(&m->norms, 2 * sizeof(unsigned long long)));
  CKC(cudaMemsetAsync(m->status, 0, sizeof(unsigned), st));
  return 0;
}

extern "C" void bem_mixed_free(bem_mixed *m) {
  if (m->gexec) cudaGraphExecDestroy(m->gexec);
  if (m->graph) cudaGraphDestroy(m->graph);
  if (m->blas) cublasDestroy(m->blas);
  cudaFree(m->M); cudaFree(m->piv); cudaFree(m->R32); cudaFree(m->X); cudaFree(m->R); cudaFree(m->D);
  cudaFree(m->ts_i); cudaFree(m->ts_c); cudaFree(m->blas_ws);
  cudaFree(m->status); cudaFree(m->norms);
  *m = bem_mixed();
}

extern "C" int bem_mixed_factor(bem_mixed *m, const double *A, int n, cudaStream_t st) {
  CKB(cublasSetStream(m->blas, st));
  if (grow(m, &m->M, &m->M_cap, (size_t)n * n) || grow(m, &m->piv, &m->piv_cap, (size_t)n) ||
      grow(m, &m->ts_i, &m->ts_i_cap, ts_ints(n)) ||
      grow(m, &m->ts_c, &m->ts_c_cap, (size_t)2 * LEAF_W * LEAF_W))
    return -1;
  // The factorisation of a size is a fixed sequence of several hundred short
  // launches (panels, TRSM, GEMM); it is captured once as a CUDA graph per
  // (size, matrix and buffer addresses, arithmetic) and replayed, which takes
  // the per-launch cost off the critical path.
  const bool same = m->gexec && m->g_n == n && m->g_A == (const void *)A && m->g_M == (const void *)m->M &&
                    m->g_ts == (const void *)m->ts_i && m->g_mode == m->mode;
  if (!same) {
    if (m->gexec) cudaGraphExecDestroy(m->gexec);
    if (m->graph) cudaGraphDestroy(m->graph);
    m->gexec = nullptr;
    m->graph = nullptr;
    CKC(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    const size_t count = (size_t)n * n;
    k_round_c32<<<grid_for(count), 256, 0, st>>>((const double2 *)A, m->M, count);
    k_iota<<<(n + 255) / 256, 256, 0, st>>>(ts_gid(m, n), n);
    int rc = cudaGetLastError() == cudaSuccess ? rec_lu(m, n, 0, n, st) : -1;
    cudaGraph_t g = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(st, &g);
    if (rc == 0 && ec != cudaSuccess) {
      snprintf(m->err, sizeof(m->err), "capture of the factorisation: %s", cudaGetErrorString(ec));
      rc = -1;
    }
    if (rc != 0) {
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      return -1;
    }
    m->graph = g;
    CKC(cudaGraphInstantiate(&m->gexec, m->graph, 0));
    m->g_n = n;
    m->g_A = A;
    m->g_M = m->M;
    m->g_ts = m->ts_i;
    m->g_mode = m->mode;
  }
  CKC(cudaGraphLaunch(m->gexec, st));
  return 0;
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
    k_unpivot_widen<<<grid_for(cnt), 256, 0, st>>>(m->R32, m->D, n, nrhs, ts_gid(m, n));
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

extern "C" unsigned bem_mixed_status(bem_mixed *m, cudaStream_t st) {
  unsigned s = 0;
  cudaMemcpyAsync(&s, m->status, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
  cudaStreamSynchronize(st);
  cudaMemsetAsync(m->status, 0, sizeof(unsigned), st);
  return s;
}
