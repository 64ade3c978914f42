// Dense complex FP64 LU factorisation with row pivoting, and the triangular
// solves, written for B200 with no library: the device replacement of the
// reference's dense solves (PARDISO mtype 13 on the global system,
// b_mkl_solver_pardiso_d, d3qd2_mkl_solver.c:18-148, called at
// bem3_aw_qd2_solve_bieq.c:347-368; LAPACKE_zgesv on each domain's dpv system,
// solve_dpv_bv, bem3_aw_qd2_solve_bieq.c:533-653).
//
// The matrix is row-major (the layout the assembly writes), factored in place
// as P A = L U, right-looking, 32 columns per panel.  Per panel three kernels:
//
//  k_lu_panel   one thread-block cluster of 8 CTAs picks the panel's 32 pivot
//               rows by tournament pivoting (communication-avoiding LU): each
//               CTA runs partial pivoting on its slice of rows, one row per
//               thread in registers, and passes its winners on; CTA 0 runs
//               partial pivoting on the winners, which gives the pivot order
//               and the packed L11\U11, inverts U11 and L11, and lists the row
//               moves (at most 64 touched positions).  The matrix is not
//               written here.
//  k_lu_apply   all SMs: L21 = A21 U11^-1 for every row below the panel,
//               the row moves on the columns outside the panel, and
//               U12 = L11^-1 A12 on the pivot rows.
//  k_lu_update  all SMs: A22 -= L21 U12 on the FP64 tensor cores
//               (mma.sync m8n8k4 f64; Blackwell's tcgen05 has no FP64 kind),
//               64 x 64 complex tiles, the complex product as four real ones.
//
// The sequence of a size and matrix is captured once as a CUDA graph and
// replayed.  Solves: forward substitution L y = P b and back substitution
// U x = y in one launch each, one CTA per 32-row block; blocks are written in
// dependency order and a block folds in each block it needs as soon as a
// progress counter in global memory has passed it (bounded waits: a wait that
// gives up sets BEM_LU_ST_WAIT and the call reports it; nothing hangs).  The
// launches are cooperative, so every CTA is resident and blocks are taken in
// order: the waits cannot deadlock.
#include "bem_count.h"
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include "bem_lu.h"

#define LU_W BEM_LU_W
#define LU_OB BEM_LU_OB  // outer block: panels whose updates right of it are delayed and applied at once
#define LU_NSLOT (LU_OB / LU_W)
#define LU_ONE_BLOCK_N 2048  // default of bem_lu.one_block_max
static_assert(LU_OB == LU_OUTER_W, "the tensor-core update depth is the outer block");
#define LU_TH 256        // threads of a panel CTA: one row each
#define LU_CL 8          // CTAs of the panel cluster
#define LU_MAXP (2 * LU_W)
#define FULL 0xffffffffu

// integer scratch (bem_lu.piv)
#define PV_CAND 0                    // [LU_CL][LU_W] candidate rows of each leaf
#define PV_CCNT (LU_CL * LU_W)       // [LU_CL] candidates per leaf
#define PV_SEL (PV_CCNT + LU_CL)     // [LU_W] pivot rows in order
#define PV_PERM (PV_SEL + LU_W)      // count, then (dst, src) pairs of the row moves
#define PV_INTS (PV_PERM + 1 + 2 * LU_MAXP)
// complex scratch (bem_lu.u11)
#define U_LU 0                       // [LU_W][LU_W] packed L11\U11, row i = pivot row i
#define U_UINV (LU_W * LU_W)         // U11^-1 (upper)
#define U_STAGE (2 * LU_W * LU_W)    // panel values of the rows moved out of the pivot block
#define U_LINV (3 * LU_W * LU_W)     // [LU_NSLOT] L11^-1 (unit lower) of each panel of the outer block
#define U_COUNT ((3 + LU_NSLOT) * LU_W * LU_W)

// ---------------------------------------------------------------- complex helpers
// complex double (double2) and complex float (float2): the same code in both
// precisions
template <class C2> struct cx;
template <> struct cx<double2> {
  using R = double;
  static __device__ __forceinline__ double2 mk(double a, double b) { return make_double2(a, b); }
};
template <> struct cx<float2> {
  using R = float;
  static __device__ __forceinline__ float2 mk(float a, float b) { return make_float2(a, b); }
};
template <class C2> __device__ __forceinline__ C2 czero() { return cx<C2>::mk(0, 0); }
template <class C2> __device__ __forceinline__ C2 cone() { return cx<C2>::mk(1, 0); }
template <class C2> __device__ __forceinline__ C2 cneg(C2 a) { return cx<C2>::mk(-a.x, -a.y); }
__device__ __forceinline__ double2 cz() { return make_double2(0.0, 0.0); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
// c + a b
__device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 c) {
  return make_double2(fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y)));
}
// c - a b
__device__ __forceinline__ double2 cfms(double2 a, double2 b, double2 c) {
  return make_double2(fma(-a.x, b.x, fma(a.y, b.y, c.x)), fma(-a.x, b.y, fma(-a.y, b.x, c.y)));
}
__device__ __forceinline__ double2 crcp(double2 a) {
  const double d = 1.0 / fma(a.x, a.x, a.y * a.y);
  return make_double2(a.x * d, -a.y * d);
}
__device__ __forceinline__ double cabs1(double2 a) { return fabs(a.x) + fabs(a.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cfma(float2 a, float2 b, float2 c) {
  return make_float2(fmaf(a.x, b.x, fmaf(-a.y, b.y, c.x)), fmaf(a.x, b.y, fmaf(a.y, b.x, c.y)));
}
__device__ __forceinline__ float2 cfms(float2 a, float2 b, float2 c) {
  return make_float2(fmaf(-a.x, b.x, fmaf(a.y, b.y, c.x)), fmaf(-a.x, b.y, fmaf(-a.y, b.x, c.y)));
}
__device__ __forceinline__ float2 crcp(float2 a) {
  const float d = 1.0f / fmaf(a.x, a.x, a.y * a.y);
  return make_float2(a.x * d, -a.y * d);
}
__device__ __forceinline__ float cabs1(float2 a) { return fabsf(a.x) + fabsf(a.y); }

// ---------------------------------------------------------------- partial pivoting in one CTA
template <class C2>
struct gepp_sh {
  unsigned wk[2][LU_TH / 32];  // each warp's pivot key
  C2 prow[2][LU_W], krow[2][LU_W];
  C2 prcp[2];                  // reciprocal of the pivot
  int pid[2], kid[2];
};

// Pivot key of a candidate: the float bits of |re| + |im| (non-negative floats
// order as their bits) with the low 8 bits replaced by 255 - t, so that one
// integer maximum gives the largest value and, among values equal to 2^-15,
// the lowest row; 0 for a row that takes no part.
__device__ __forceinline__ unsigned pivot_key(float a, int t) {
  return (__float_as_uint(a) & 0xFFFFFF00u) | (unsigned)(255 - t);
}

// rotate the first L registers by one: v[0] (the finished pivot column)
// goes to v[L - 1]
template <int L, class C2>
__device__ __forceinline__ void rotl(C2 (&v)[LU_W]) {
  const C2 f = v[0];
#pragma unroll
  for (int c = 0; c < L - 1; ++c) v[c] = v[c + 1];
  v[L - 1] = f;
}

// One elimination step j of gepp: v[0] holds column j and v[1 .. 31 - j] the
// columns still to update; L >= 32 - j is the step's compile-time bound, so
// that the update and the rotation touch only the live window (the finished
// columns beyond it stay where they are).
template <int L, class C2>
__device__ __forceinline__ void gepp_step(C2 (&v)[LU_W], int &id, int j, int steps, int rr, gepp_sh<C2> &sh,
                                          unsigned *status) {
  const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
  if (j < steps) {
    const int b = j & 1;
    // the pivot: one integer maximum per warp, then over the warps (the
    // 2^-15 resolution of the key only picks among rows within that much of
    // the largest, which keeps partial pivoting's growth bound)
    const unsigned key = __reduce_max_sync(FULL, (t >= j && t < rr) ? pivot_key((float)cabs1(v[0]), t) : 0u);
    if (lane == 0) sh.wk[b][wid] = key;
    __syncthreads();
    unsigned best = sh.wk[b][0];
#pragma unroll
    for (int q = 1; q < LU_TH / 32; ++q) best = max(best, sh.wk[b][q]);
    int p = 255 - (int)(best & 255u);
    if ((best >> 8) == 0u) {  // no non-zero entry left in the column
      if (status && t == 0) atomicOr(status, BEM_LU_ST_ZERO);
      p = j;
    }
    if (t == p) {
#pragma unroll
      for (int c = 0; c < LU_W; ++c) sh.prow[b][c] = v[c];
      sh.pid[b] = id;
      sh.prcp[b] = crcp(v[0]);
    }
    if (t == j) {
#pragma unroll
      for (int c = 0; c < LU_W; ++c) sh.krow[b][c] = v[c];
      sh.kid[b] = id;
    }
    __syncthreads();
    if (t == j) {
#pragma unroll
      for (int c = 0; c < LU_W; ++c) v[c] = sh.prow[b][c];
      id = sh.pid[b];
    } else if (t == p) {
#pragma unroll
      for (int c = 0; c < LU_W; ++c) v[c] = sh.krow[b][c];
      id = sh.kid[b];
    }
    if (t > j && t < rr) {
      const C2 l = cmul(v[0], sh.prcp[b]);
      v[0] = l;
#pragma unroll
      for (int c = 1; c < L; ++c)
        if (c < LU_W - j) v[c] = cfms(l, sh.prow[b][c], v[c]);
    }
  }
  rotl<L>(v);
}

// Partial pivoting (|re| + |im| as LAPACK's izamax, lowest row on ties) over
// the rr <= LU_TH rows held one per thread (thread t < rr: values v, matrix
// row id), w columns.  Afterwards thread i < min(w, rr) holds the i-th pivot
// row and its id, its values packed (multipliers left of column i, U from i
// on), columns in order.  A row is kept rotated while it is eliminated: at
// step j its register 0 holds column j, registers 1 .. 31 - j the columns
// still to update and the rest the finished ones, so that every register
// index is a compile-time constant inside one short loop body.
//
// The steps run in four groups of eight with a shrinking live window of 32,
// 24, 16 and 8 registers: each group's finished columns end up in the eight
// registers just past the next group's window (group g's at 24 - 8 g ..
// 31 - 8 g), which a fixed permutation puts back in order at the end.
template <class C2>
__device__ void gepp(C2 (&v)[LU_W], int &id, int rr, int w, gepp_sh<C2> &sh, unsigned *status) {
  const int steps = min(w, rr);
  for (int j = 0; j < 8; ++j) gepp_step<32>(v, id, j, steps, rr, sh, status);
  for (int j = 8; j < 16; ++j) gepp_step<24>(v, id, j, steps, rr, sh, status);
  for (int j = 16; j < 24; ++j) gepp_step<16>(v, id, j, steps, rr, sh, status);
  for (int j = 24; j < 32; ++j) gepp_step<8>(v, id, j, steps, rr, sh, status);
  // registers 24 - 8 g .. 31 - 8 g hold columns 8 g .. 8 g + 7
  C2 o[LU_W];
#pragma unroll
  for (int g = 0; g < 4; ++g)
#pragma unroll
    for (int i = 0; i < 8; ++i) o[8 * g + i] = v[24 - 8 * g + i];
#pragma unroll
  for (int c = 0; c < LU_W; ++c) v[c] = o[c];
}

template <class C2>
__device__ __forceinline__ void load_row(C2 (&v)[LU_W], const C2 *A, long lda, int row, int k, int w) {
  const C2 *p = A + (size_t)(row < 0 ? 0 : row) * lda + k;
#pragma unroll
  for (int c = 0; c < LU_W; ++c) v[c] = (row >= 0 && c < w) ? p[c] : czero<C2>();
}

__device__ __forceinline__ unsigned cluster_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
// all threads of all CTAs of the cluster; orders global-memory writes before it
// with reads after it (release / acquire at cluster scope)
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// ---------------------------------------------------------------- panel
// the leaves' partial pivoting only selects candidate rows (the root factors
// the winners from their stored values), so it runs in complex FP32 for
// either precision of the factorisation
template <class C2> struct leaf_of { using T = float2; };

__device__ __forceinline__ void load_row_leaf(float2 (&v)[LU_W], const double2 *A, long lda, int row, int k, int w) {
  const double2 *p = A + (size_t)(row < 0 ? 0 : row) * lda + k;
#pragma unroll
  for (int c = 0; c < LU_W; ++c) {
    const double2 x = (row >= 0 && c < w) ? p[c] : make_double2(0.0, 0.0);
    v[c] = make_float2((float)x.x, (float)x.y);
  }
}
__device__ __forceinline__ void load_row_leaf(float2 (&v)[LU_W], const float2 *A, long lda, int row, int k, int w) {
  load_row(v, A, lda, row, k, w);
}

template <class C2>
struct panel_sh {
  gepp_sh<C2> g;
  gepp_sh<float2> gl;
  C2 lu[LU_W][LU_W + 1];
  C2 rd[LU_W];  // reciprocals of U11's diagonal
  int sel[LU_W], la[LU_W], lb[LU_W];
};

template <class C2>
__global__ void __cluster_dims__(LU_CL, 1, 1) __launch_bounds__(LU_TH, 1)
    k_lu_panel(C2 *A, long lda, int n, int k, int *pv, C2 *u, unsigned *status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  panel_sh<C2> &S = *reinterpret_cast<panel_sh<C2> *>(smem_raw);
  const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
  const int crank = (int)cluster_rank();
  const int w = min(LU_W, n - k), m = n - k;
  int id = -1;
  if (m > LU_TH) {
    // leaves: each CTA a contiguous slice of the panel's rows, in rounds of
    // LU_TH rows: the winners of a round stay, fresh rows fill the other slots
    const int q = (m + LU_CL - 1) / LU_CL;
    const int lo = k + crank * q, hi = min(n, lo + q);
    int ncand = 0, next = lo;
    while (next < hi) {
      const int fresh = min(LU_TH - ncand, hi - next);
      int row = -1;
      if (t < ncand) row = id;
      else if (t < ncand + fresh) row = next + (t - ncand);
      next += fresh;
      id = row;
      float2 vl[LU_W];
      load_row_leaf(vl, A, lda, row, k, w);
      const int rr = ncand + fresh;
      gepp(vl, id, rr, w, S.gl, nullptr);
      ncand = min(w, rr);
      __syncthreads();
    }
    if (t < ncand) pv[PV_CAND + crank * LU_W + t] = id;
    if (t == 0) pv[PV_CCNT + crank] = ncand;
    __threadfence();
  }
  cluster_sync_all();
  if (crank != 0) return;
  // root: partial pivoting over the leaves' winners (or over all rows of a
  // short panel), with the values kept: the pivot order and L11\U11
  int rr;
  if (m > LU_TH) {
    int total = 0, mine = -1;
    for (int cc = 0; cc < LU_CL; ++cc) {
      const int cnt = __ldcg(pv + PV_CCNT + cc);
      if (t >= total && t < total + cnt) mine = __ldcg(pv + PV_CAND + cc * LU_W + (t - total));
      total += cnt;
    }
    rr = total;
    id = mine;
  } else {
    rr = m;
    id = t < m ? k + t : -1;
  }
  C2 v[LU_W];
  load_row(v, A, lda, id, k, w);
  gepp(v, id, rr, w, S.g, status);
  if (t < LU_W) {
#pragma unroll
    for (int c = 0; c < LU_W; ++c) {
      const C2 x = (t < w) ? v[c] : czero<C2>();
      S.lu[t][c] = x;
      u[U_LU + t * LU_W + c] = x;
    }
    S.sel[t] = t < w ? id : -1;
    if (t < w) pv[PV_SEL + t] = id;
  }
  if (t < LU_W) S.rd[t] = t < w ? crcp(S.lu[t][t]) : czero<C2>();
  __syncthreads();
  // U11^-1 (warps 0-3) and L11^-1 (warps 4-7), 8 columns a warp, 4 at a
  // time, column-oriented substitution with lane = row: at step l lane l
  // finishes x_l, a shuffle hands it to the other lanes, and each lane
  // removes its u_il x_l (l_il x_l): one short dependent step per row, all
  // rows of four columns at once
  {
    const int i = lane;
    const bool upper = wid < 4;
    const int jb = (wid & 3) * 8;
    for (int half = 0; half < 2; ++half) {
      C2 x[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) x[q] = (i == jb + half * 4 + q && i < w) ? cone<C2>() : czero<C2>();
      if (upper) {
        for (int l = LU_W - 1; l >= 0; --l) {
          const C2 a = S.lu[i][l], d = S.rd[l];
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            if (i == l) x[q] = cmul(x[q], d);
            const C2 xl = cx<C2>::mk(__shfl_sync(FULL, x[q].x, l), __shfl_sync(FULL, x[q].y, l));
            if (i < l) x[q] = cfms(a, xl, x[q]);
          }
        }
      } else {
        for (int l = 0; l < LU_W; ++l) {
          const C2 a = S.lu[i][l];
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const C2 xl = cx<C2>::mk(__shfl_sync(FULL, x[q].x, l), __shfl_sync(FULL, x[q].y, l));
            if (i > l) x[q] = cfms(a, xl, x[q]);
          }
        }
      }
      C2 *dst = upper ? u + U_UINV : u + U_LINV + (k % LU_OB) / LU_W * (LU_W * LU_W);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int j = jb + half * 4 + q;
        // entries outside a short panel (w < 32) are zero
        dst[i * LU_W + j] = (i < w && j < w) ? x[q] : czero<C2>();
      }
    }
  }
  if (wid == 2) {
    // row moves: pivot row i goes to position k + i; the rows of the pivot
    // block that were not picked (displaced) go to the positions the pivot
    // rows from below left, paired in lane order
    const int i = lane;
    const int p = (i < w) ? S.sel[i] : -1;
    const bool below = (i < w) && (p >= k + w);
    bool picked = false;
    for (int jj = 0; jj < w; ++jj) picked |= (S.sel[jj] == k + i);
    const bool displaced = (i < w) && !picked;
    const unsigned ba = __ballot_sync(FULL, below), bb = __ballot_sync(FULL, displaced);
    const unsigned lt = (1u << lane) - 1u;
    if (below) S.la[__popc(ba & lt)] = p;
    if (displaced) S.lb[__popc(bb & lt)] = k + i;
    __syncwarp();
    const int cnt = __popc(ba);
    int *perm = pv + PV_PERM;
    if (lane == 0) perm[0] = w + cnt;
    if (i < w) { perm[1 + 2 * i] = k + i; perm[2 + 2 * i] = p; }
    if (lane < cnt) { perm[1 + 2 * (w + lane)] = S.la[lane]; perm[2 + 2 * (w + lane)] = S.lb[lane]; }
    // the displaced rows' panel values, before anything overwrites them
    for (int r = 0; r < cnt; ++r)
      u[U_STAGE + r * LU_W + lane] = lane < w ? A[(size_t)S.lb[r] * lda + k + lane] : czero<C2>();
  }
}

// ---------------------------------------------------------------- row moves, L21, U12
#define AP_TH 128
#define AP_ROWS 32   // rows of an L21 block (4 threads per row)
#define AP_COLS 16   // columns of a row-move block

template <class C2>
__global__ void __launch_bounds__(AP_TH) k_lu_apply(C2 *A, long lda, int n, int k, int cend, const int *pv, const C2 *u,
                                                    int *rowmap, unsigned *status) {
  __shared__ C2 sm[LU_W][LU_W + 1];
  __shared__ C2 srow[LU_MAXP][AP_COLS + 1];
  __shared__ int sdst[LU_MAXP], ssrc[LU_MAXP];
  const int t = threadIdx.x;
  const int w = min(LU_W, n - k);
  const int r0 = k + w;
  int nperm = __ldcg(pv + PV_PERM);
  if (nperm < 0 || nperm > LU_MAXP) {
    if (t == 0) atomicOr(status, BEM_LU_ST_INTERNAL);
    nperm = 0;
  }
  for (int e = t; e < nperm; e += AP_TH) {
    int d = __ldcg(pv + PV_PERM + 1 + 2 * e), sr = __ldcg(pv + PV_PERM + 2 + 2 * e);
    if (d < k || d >= n || sr < k || sr >= n) {  // a row move out of range: report, keep the row
      if (blockIdx.x == 0) atomicOr(status, BEM_LU_ST_INTERNAL);
      d = sr = k + (e < w ? e : 0);
    }
    sdst[e] = d;
    ssrc[e] = sr;
  }
  const int nL = (n - r0 + AP_ROWS - 1) / AP_ROWS;
  const int nCl = (k + AP_COLS - 1) / AP_COLS, nCr = (n - r0 + AP_COLS - 1) / AP_COLS;
  const int b = blockIdx.x;
  if (b < nL) {
    // L21 = A21 U11^-1 in place, for the rows below the pivot block that no move touches
    for (int e = t; e < LU_W * LU_W; e += AP_TH) sm[e / LU_W][e % LU_W] = __ldcg(u + U_UINV + e);
    const int row = r0 + b * AP_ROWS + (t >> 2), part = t & 3;
    // the row's panel values, loaded at once (independent loads, not a chain)
    C2 a[LU_W];
    {
      const C2 *ap = A + (size_t)(row < n ? row : r0) * lda + k;
#pragma unroll
      for (int l = 0; l < LU_W; ++l) a[l] = (row < n && l < w) ? ap[l] : czero<C2>();
    }
    __syncthreads();
    bool live = row < n;
    for (int e = w; e < nperm && live; ++e) live = sdst[e] != row;
    C2 x[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) x[c] = czero<C2>();
#pragma unroll
    for (int l = 0; l < LU_W; ++l)
#pragma unroll
      for (int c = 0; c < 8; ++c) x[c] = cfma(a[l], sm[l][part * 8 + c], x[c]);
    __syncthreads();  // every read of the row before any write to it
    if (live) {
      C2 *ap = A + (size_t)row * lda + k;
#pragma unroll
      for (int c = 0; c < 8; ++c)
        if (part * 8 + c < w) ap[part * 8 + c] = x[c];
    }
    return;
  }
  if (b < nL + nCl + nCr) {
    // the row moves on AP_COLS columns outside the panel; right of the panel
    // and left of cend (the end of the outer block) also U12 = L11^-1 A12 on
    // the pivot block; right of cend the moves alone (U12 there is formed for
    // the whole outer block at once, k_lu_trsm)
    const int i = b - nL;
    const bool right = i >= nCl;
    const int c0 = right ? r0 + (i - nCl) * AP_COLS : i * AP_COLS;
    const int c1 = min(right ? n : k, c0 + AP_COLS);
    const int nc = c1 - c0;
    const bool u12 = right && c0 < cend;
    if (u12) {
      const C2 *linv = u + U_LINV + (k % LU_OB) / LU_W * (LU_W * LU_W);
      for (int e = t; e < LU_W * LU_W; e += AP_TH) sm[e / LU_W][e % LU_W] = __ldcg(linv + e);
    }
    __syncthreads();  // sdst / ssrc
    for (int e = t; e < nperm * AP_COLS; e += AP_TH) {
      const int pr = e / AP_COLS, cc = e % AP_COLS;
      srow[pr][cc] = cc < nc ? A[(size_t)ssrc[pr] * lda + c0 + cc] : czero<C2>();
    }
    __syncthreads();
    const int cc = t % AP_COLS, grp = t / AP_COLS;  // 8 groups of 16 columns
    if (cc < nc) {
      if (u12) {
        for (int ii = grp; ii < w; ii += AP_TH / AP_COLS) {
          C2 s = czero<C2>();
          for (int l = 0; l <= ii; ++l) s = cfma(sm[ii][l], srow[l][cc], s);
          A[(size_t)(k + ii) * lda + c0 + cc] = s;
        }
        for (int e = w + grp; e < nperm; e += AP_TH / AP_COLS) A[(size_t)sdst[e] * lda + c0 + cc] = srow[e][cc];
      } else {
        for (int e = grp; e < nperm; e += AP_TH / AP_COLS) A[(size_t)sdst[e] * lda + c0 + cc] = srow[e][cc];
      }
    }
    return;
  }
  // last block: the panel columns of the moved rows (the pivot block gets
  // L11\U11, a row moved below it its L21), and the row map
  for (int e = t; e < LU_W * LU_W; e += AP_TH) sm[e / LU_W][e % LU_W] = __ldcg(u + U_UINV + e);
  __syncthreads();
  for (int e = t; e < w * LU_W; e += AP_TH) {
    const int ii = e / LU_W, c = e % LU_W;
    if (c < w) A[(size_t)(k + ii) * lda + k + c] = __ldcg(u + U_LU + ii * LU_W + c);
  }
  {
    const int r = t >> 2, part = t & 3, e = w + r;
    if (e < nperm) {
      C2 a[LU_W];
#pragma unroll
      for (int l = 0; l < LU_W; ++l) a[l] = l < w ? __ldcg(u + U_STAGE + r * LU_W + l) : czero<C2>();
      C2 x[8];
#pragma unroll
      for (int c = 0; c < 8; ++c) x[c] = czero<C2>();
#pragma unroll
      for (int l = 0; l < LU_W; ++l)
#pragma unroll
        for (int c = 0; c < 8; ++c) x[c] = cfma(a[l], sm[l][part * 8 + c], x[c]);
      C2 *ap = A + (size_t)sdst[e] * lda + k;
#pragma unroll
      for (int c = 0; c < 8; ++c)
        if (part * 8 + c < w) ap[part * 8 + c] = x[c];
    }
  }
  int old = 0;
  if (t < nperm) old = rowmap[ssrc[t]];
  __syncthreads();
  if (t < nperm) rowmap[sdst[t]] = old;
}

// ---------------------------------------------------------------- trailing update
#define UP_BM 64
#define UP_BN 64
#define UP_TH 256
#define UP_LDA 36   // shared-memory row strides (doubles) of the L21 and U12 tiles:
#define UP_LDB 68   // conflict-free fragment loads
#define UP_SMEM ((2 * UP_BM * UP_LDA + 2 * LU_W * UP_LDB) * sizeof(double))

// d = a b + d on an 8 x 8 x 4 FP64 tile: a (8 x 4, row) holds a[g][q], b (4 x 8,
// col) b[q][g], d (8 x 8) d[g][2 q .. 2 q + 1], with g = lane / 4, q = lane % 4
__device__ __forceinline__ void dmma(double a, double b, double (&d)[2]) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

// C -= L U on the FP64 tensor cores: C = A[r0:n, c0:cend), L = A[r0:n, kk:kk+kw),
// U = A[kk:kk+kw, c0:cend); kw in steps of LU_W staged through shared memory.
// A panel's update (kk = k, kw = 32, cend = the end of its outer block) and an
// outer block's (kk = its first column, kw = LU_OB, cend = n) alike.
__global__ void __launch_bounds__(UP_TH, 2) k_lu_update(double2 *A, long lda, int n, int kk, int kw, int r0,
                                                        int c0, int cend) {
  extern __shared__ __align__(16) double up_smem[];
  double *Ar = up_smem, *Ai = Ar + UP_BM * UP_LDA, *Br = Ai + UP_BM * UP_LDA, *Bi = Br + LU_W * UP_LDB;
  const int t = threadIdx.x;
  const int rb = r0 + blockIdx.y * UP_BM, cb = c0 + blockIdx.x * UP_BN;
  const int lane = t & 31, wid = t >> 5, g = lane >> 2, q = lane & 3;
  const int wm = wid & 1, wn = wid >> 1;  // warp tile: 32 rows x 16 columns
  double cr[4][2][2], ci[4][2][2];
#pragma unroll
  for (int mt = 0; mt < 4; ++mt)
#pragma unroll
    for (int nt = 0; nt < 2; ++nt) {
      const int row = rb + wm * 32 + mt * 8 + g, col = cb + wn * 16 + nt * 8 + 2 * q;
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const double2 x = (row < n && col + i < cend) ? A[(size_t)row * lda + col + i] : cz();
        cr[mt][nt][i] = x.x;
        ci[mt][nt][i] = x.y;
      }
    }
  for (int q0 = 0; q0 < kw; q0 += LU_W) {
    const int wq = min(LU_W, kw - q0), kc = kk + q0;
    if (q0) __syncthreads();  // the previous chunk's fragment loads are done
    for (int e = t; e < UP_BM * LU_W; e += UP_TH) {
      const int r = e / LU_W, c = e % LU_W;
      const double2 x = (rb + r < n && c < wq) ? A[(size_t)(rb + r) * lda + kc + c] : cz();
      Ar[r * UP_LDA + c] = x.x;
      Ai[r * UP_LDA + c] = x.y;
    }
    for (int e = t; e < LU_W * UP_BN; e += UP_TH) {
      const int r = e / UP_BN, c = e % UP_BN;
      const double2 x = (r < wq && cb + c < cend) ? A[(size_t)(kc + r) * lda + cb + c] : cz();
      Br[r * UP_LDB + c] = x.x;
      Bi[r * UP_LDB + c] = x.y;
    }
    __syncthreads();
#pragma unroll
    for (int k4 = 0; k4 < LU_W; k4 += 4) {
      double ar[4], ai[4], br[2], bi[2];
#pragma unroll
      for (int mt = 0; mt < 4; ++mt) {
        ar[mt] = Ar[(wm * 32 + mt * 8 + g) * UP_LDA + k4 + q];
        ai[mt] = Ai[(wm * 32 + mt * 8 + g) * UP_LDA + k4 + q];
      }
#pragma unroll
      for (int nt = 0; nt < 2; ++nt) {
        br[nt] = Br[(k4 + q) * UP_LDB + wn * 16 + nt * 8 + g];
        bi[nt] = Bi[(k4 + q) * UP_LDB + wn * 16 + nt * 8 + g];
      }
#pragma unroll
      for (int mt = 0; mt < 4; ++mt)
#pragma unroll
        for (int nt = 0; nt < 2; ++nt) {
          // (cr, ci) -= (ar + i ai)(br + i bi)
          dmma(-ar[mt], br[nt], cr[mt][nt]);
          dmma(ai[mt], bi[nt], cr[mt][nt]);
          dmma(-ar[mt], bi[nt], ci[mt][nt]);
          dmma(-ai[mt], br[nt], ci[mt][nt]);
        }
    }
  }
#pragma unroll
  for (int mt = 0; mt < 4; ++mt)
#pragma unroll
    for (int nt = 0; nt < 2; ++nt) {
      const int row = rb + wm * 32 + mt * 8 + g, col = cb + wn * 16 + nt * 8 + 2 * q;
#pragma unroll
      for (int i = 0; i < 2; ++i)
        if (row < n && col + i < cend) A[(size_t)row * lda + col + i] = make_double2(cr[mt][nt][i], ci[mt][nt][i]);
    }
}

// complex FP32: the same update on the CUDA cores, 64 x 64 tiles, 4 x 4
// outputs per thread (rows ty*4 + i, columns tx + 16 j: conflict-free shared
// loads and 128-byte runs of C per 16 threads)
#define UF_TH 256
__global__ void __launch_bounds__(UF_TH) k_lu_update_c32(float2 *A, long lda, int n, int kk, int kw, int r0,
                                                         int c0, int cend) {
  __shared__ float2 As[UP_BM][LU_W + 1];
  __shared__ float2 Bs[LU_W][UP_BN + 1];
  const int t = threadIdx.x;
  const int rb = r0 + blockIdx.y * UP_BM, cb = c0 + blockIdx.x * UP_BN;
  const int ty = t >> 4, tx = t & 15;
  float2 acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int row = rb + ty * 4 + i, col = cb + tx + 16 * j;
      acc[i][j] = (row < n && col < cend) ? A[(size_t)row * lda + col] : make_float2(0.f, 0.f);
    }
  for (int q0 = 0; q0 < kw; q0 += LU_W) {
    const int wq = min(LU_W, kw - q0), kc = kk + q0;
    if (q0) __syncthreads();
    for (int e = t; e < UP_BM * LU_W; e += UF_TH) {
      const int r = e / LU_W, c = e % LU_W;
      As[r][c] = (rb + r < n && c < wq) ? A[(size_t)(rb + r) * lda + kc + c] : make_float2(0.f, 0.f);
    }
    for (int e = t; e < LU_W * UP_BN; e += UF_TH) {
      const int r = e / UP_BN, c = e % UP_BN;
      Bs[r][c] = (r < wq && cb + c < cend) ? A[(size_t)(kc + r) * lda + cb + c] : make_float2(0.f, 0.f);
    }
    __syncthreads();
#pragma unroll 4
    for (int k1 = 0; k1 < LU_W; ++k1) {
      float2 a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[ty * 4 + i][k1];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[k1][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = cfms(a[i], b[j], acc[i][j]);
    }
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int row = rb + ty * 4 + i, col = cb + tx + 16 * j;
      if (row < n && col < cend) A[(size_t)row * lda + col] = acc[i][j];
    }
}

// ---------------------------------------------------------------- U12 of an outer block
// U12 = L11^-1 A12 in place for the outer block's rows K .. K + ob - 1 and the
// columns right of it (L11 unit lower, in A's strictly lower part, its
// diagonal blocks' inverses in the LINV slots): block row ib gets
// Linv_ib (A12_ib - sum_{jb < ib} L_ib,jb U12_jb).  One CTA per TR_NC
// columns; thread (i, c) holds row i of a block row and columns c, c + 4,
// c + 8, c + 12 (conflict-free shared-memory reads: a warp reads 8 rows of L
// at one column and 4 consecutive columns of X).
#define TR_TH 128
#define TR_NC 16
template <class C2>
struct trsm_sh {
  C2 X[LU_OB][TR_NC + 1];
  C2 L[LU_W][LU_W + 1];
  C2 Y[LU_W][TR_NC + 1];
};
template <class C2>
__global__ void __launch_bounds__(TR_TH) k_lu_trsm(C2 *A, long lda, int n, int K, int ob, const C2 *u) {
  extern __shared__ __align__(16) unsigned char tr_raw[];
  trsm_sh<C2> &S = *reinterpret_cast<trsm_sh<C2> *>(tr_raw);
  const int t = threadIdx.x;
  const int c0 = K + ob + blockIdx.x * TR_NC;
  const int nbk = ob / LU_W;
  for (int e = t; e < ob * TR_NC; e += TR_TH) {
    const int r = e / TR_NC, c = e % TR_NC;
    S.X[r][c] = c0 + c < n ? A[(size_t)(K + r) * lda + c0 + c] : czero<C2>();
  }
  const int i = t >> 2, cq = t & 3;  // row i of a block row, columns cq + 4 j
  for (int ib = 0; ib < nbk; ++ib) {
    C2 acc[4];
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[j] = S.X[ib * LU_W + i][cq + 4 * j];
    for (int jb = 0; jb < ib; ++jb) {
      for (int e = t; e < LU_W * LU_W; e += TR_TH) {
        const int r = e / LU_W, c = e % LU_W;
        S.L[r][c] = A[(size_t)(K + ib * LU_W + r) * lda + K + jb * LU_W + c];
      }
      __syncthreads();
#pragma unroll 8
      for (int l = 0; l < LU_W; ++l) {
        const C2 lv = S.L[i][l];
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[j] = cfms(lv, S.X[jb * LU_W + l][cq + 4 * j], acc[j]);
      }
      __syncthreads();
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) S.Y[i][cq + 4 * j] = acc[j];
    const C2 *linv = u + U_LINV + ib * (LU_W * LU_W);
    for (int e = t; e < LU_W * LU_W; e += TR_TH) S.L[e / LU_W][e % LU_W] = __ldcg(linv + e);
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[j] = czero<C2>();
#pragma unroll 8
    for (int l = 0; l < LU_W; ++l) {
      const C2 lv = S.L[i][l];
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[j] = cfma(lv, S.Y[l][cq + 4 * j], acc[j]);
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) S.X[ib * LU_W + i][cq + 4 * j] = acc[j];
    __syncthreads();  // Y and L are rewritten by the next block row
  }
  __syncthreads();
  for (int e = t; e < ob * TR_NC; e += TR_TH) {
    const int r = e / TR_NC, c = e % TR_NC;
    if (c0 + c < n) A[(size_t)(K + r) * lda + c0 + c] = S.X[r][c];
  }
}

// R = B - A X in FP64 (refinement residual): A row-major n x n, X, B, R
// column-major n x NR; one warp per row
template <int NR>
__global__ void __launch_bounds__(256) k_resid_z(const double2 *A, int n, const double2 *X, const double2 *B,
                                                 double2 *R) {
  const int lane = threadIdx.x & 31;
  const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (row >= n) return;
  double2 acc[NR];
#pragma unroll
  for (int q = 0; q < NR; ++q) acc[q] = cz();
  const double2 *a = A + (size_t)row * n;
  for (int col = lane; col < n; col += 32) {
    const double2 av = a[col];
#pragma unroll
    for (int q = 0; q < NR; ++q) acc[q] = cfma(av, X[(size_t)q * n + col], acc[q]);
  }
#pragma unroll
  for (int q = 0; q < NR; ++q)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      acc[q].x += __shfl_down_sync(FULL, acc[q].x, o);
      acc[q].y += __shfl_down_sync(FULL, acc[q].y, o);
    }
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < NR; ++q) {
      const double2 b = B[(size_t)q * n + row];
      R[(size_t)q * n + row] = make_double2(b.x - acc[q].x, b.y - acc[q].y);
    }
}

__global__ void k_lu_iota(int *rowmap, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) rowmap[i] = i;
}

// ---------------------------------------------------------------- triangular solves
#define TS_TH 128
#define TS_WAIT_NS 1000000000ull  // one second

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(unsigned *p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ unsigned ld_relaxed(const unsigned *p) {
  unsigned v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
// the two counters (lower, upper solve) sit 128 bytes apart
#define TS_FSTRIDE 32
// wait until *cnt > k and return the count seen: a spin of relaxed loads with
// an acquire fence once it has moved past k; after one second it gives up with
// BEM_LU_ST_WAIT set (and returns k + 1), and once any wait has given up later
// waits return at once
__device__ __forceinline__ unsigned wait_count(const unsigned *cnt, unsigned k, unsigned *status) {
  unsigned c = ld_acquire(cnt);
  if (c > k) return c;
  const unsigned long long t0 = gtimer();
  for (unsigned it = 1;; ++it) {
    c = ld_relaxed(cnt);
    if (c > k) {
      asm volatile("fence.acq_rel.gpu;" ::: "memory");
      return c;
    }
    if ((it & 255) == 0 && (gtimer() - t0 > TS_WAIT_NS || (ld_relaxed(status) & BEM_LU_ST_WAIT))) {
      atomicOr(status, BEM_LU_ST_WAIT);
      return k + 1;
    }
  }
}

// lower = 1: out = L^-1 (P in), in read through rowmap (unit lower L);
// lower = 0: out = U^-1 in.  in / out are n x NR column-major.  The 32-row
// blocks are solved in dependency order (top down for L, bottom up for U): the
// block of position it needs the blocks of positions 0 .. it-1, each of which
// it folds in as soon as *cnt (the number of blocks written so far, which
// grows in position order) has passed it.
template <class C2, int NR>
__global__ void __launch_bounds__(TS_TH) k_lu_trsv(const C2 *LU, long lda, int n, const int *rowmap, const C2 *in,
                                                   C2 *out, unsigned *cnt, int lower, unsigned *status) {
  __shared__ C2 sd[32][33];
  __shared__ C2 sacc[4][32][NR];
  __shared__ unsigned sready[2];
  const int nb = (n + 31) / 32;
  const int t = threadIdx.x, r = t & 31, s = t >> 5;
  unsigned nwait = 0;
  for (int it = blockIdx.x; it < nb; it += gridDim.x) {
    const int b = lower ? it : nb - 1 - it;
    const int r0 = b * 32, rows = min(32, n - r0);
    for (int e = t; e < 32 * 32; e += TS_TH) {
      const int i = e >> 5, j = e & 31;
      sd[i][j] = (i < rows && j < rows) ? LU[(size_t)(r0 + i) * lda + r0 + j] : czero<C2>();
    }
    const int row = r0 + r;
    C2 acc[NR];
#pragma unroll
    for (int q = 0; q < NR; ++q) acc[q] = czero<C2>();
    if (s == 0 && r < rows) {
      const int src = lower ? rowmap[row] : row;
#pragma unroll
      for (int q = 0; q < NR; ++q) acc[q] = in[(size_t)q * n + src];
    }
    // dependency k is the block of position k: rows/columns jb * 32 ..
    // jb * 32 + 31 with jb = k (lower) or nb - 1 - k (upper).  The factor's
    // entries do not depend on the other blocks, so dependency k + 1's eight
    // are loaded before the wait for dependency k.
    const C2 *arow = LU + (size_t)(r < rows ? row : r0) * lda;
    C2 ac[8], an[8];
    {
      const int jb = lower ? 0 : nb - 1;
#pragma unroll
      for (int cc = 0; cc < 8; ++cc) {
        const int col = jb * 32 + s * 8 + cc;
        ac[cc] = (it > 0 && r < rows && col < n) ? arow[col] : czero<C2>();
      }
    }
    unsigned ready = 0;
    for (int k = 0; k < it; ++k) {
      const int jb = lower ? k : nb - 1 - k, jn = lower ? k + 1 : nb - 2 - k;
#pragma unroll
      for (int cc = 0; cc < 8; ++cc) {
        const int col = jn * 32 + s * 8 + cc;
        an[cc] = (k + 1 < it && r < rows && col < n) ? arow[col] : czero<C2>();
      }
      if ((unsigned)k >= ready) {
        // one thread polls (all threads polling one line starve the block
        // that publishes it); the barrier passes its acquire on.  The two
        // slots alternate so a slot is rewritten only after every thread has
        // passed the barrier that follows its read.
        if (t == 0) sready[nwait & 1] = wait_count(cnt, (unsigned)k, status);
        __syncthreads();
        ready = sready[nwait & 1];
        ++nwait;
      }
      const int c0 = jb * 32 + s * 8;
#pragma unroll
      for (int cc = 0; cc < 8; ++cc) {
        const int col = c0 + cc;
        if (col < n)
#pragma unroll
          for (int q = 0; q < NR; ++q) acc[q] = cfms(ac[cc], __ldcg(out + (size_t)q * n + col), acc[q]);
        ac[cc] = an[cc];
      }
    }
#pragma unroll
    for (int q = 0; q < NR; ++q) sacc[s][r][q] = acc[q];
    __syncthreads();
    if (s == 0) {
#pragma unroll
      for (int q = 0; q < NR; ++q) {
        C2 x = sacc[0][r][q];
        for (int ss = 1; ss < 4; ++ss) x = cx<C2>::mk(x.x + sacc[ss][r][q].x, x.y + sacc[ss][r][q].y);
        acc[q] = x;
      }
      if (lower) {
        for (int i = 0; i < rows; ++i) {
#pragma unroll
          for (int q = 0; q < NR; ++q) {
            const C2 yi = cx<C2>::mk(__shfl_sync(FULL, acc[q].x, i), __shfl_sync(FULL, acc[q].y, i));
            if (r > i && r < rows) acc[q] = cfms(sd[r][i], yi, acc[q]);
          }
        }
      } else {
        for (int i = rows - 1; i >= 0; --i) {
          if (r == i) {
            const C2 d = crcp(sd[i][i]);
#pragma unroll
            for (int q = 0; q < NR; ++q) acc[q] = cmul(acc[q], d);
          }
#pragma unroll
          for (int q = 0; q < NR; ++q) {
            const C2 xi = cx<C2>::mk(__shfl_sync(FULL, acc[q].x, i), __shfl_sync(FULL, acc[q].y, i));
            if (r < i) acc[q] = cfms(sd[r][i], xi, acc[q]);
          }
        }
      }
      if (r < rows)
#pragma unroll
        for (int q = 0; q < NR; ++q) out[(size_t)q * n + row] = acc[q];
      __threadfence();
      __syncwarp();
      if (r == 0) st_release(cnt, (unsigned)it + 1u);
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------- host side
#define CKL(call, what)                                                                     \
  do {                                                                                     \
    cudaError_t _e = (call);                                                               \
    if (_e != cudaSuccess) {                                                               \
      snprintf(w->err, sizeof(w->err), "%s: %s", what, cudaGetErrorString(_e));            \
      return -1;                                                                           \
    }                                                                                      \
  } while (0)

extern "C" int bem_lu_init(bem_lu *w, int device) {
  CKL(cudaDeviceGetAttribute(&w->sms, cudaDevAttrMultiProcessorCount, device), "SM count");
  CKL(cudaFuncSetAttribute(k_lu_panel<double2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)sizeof(panel_sh<double2>)),
      "panel smem");
  CKL(cudaFuncSetAttribute(k_lu_panel<float2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)sizeof(panel_sh<float2>)),
      "panel smem");
  CKL(cudaFuncSetAttribute(k_lu_update, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)UP_SMEM), "update smem");
  CKL(cudaFuncSetAttribute(k_lu_trsm<double2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)sizeof(trsm_sh<double2>)),
      "U12 smem");
  CKL(cudaFuncSetAttribute(k_lu_trsm<float2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)sizeof(trsm_sh<float2>)),
      "U12 smem");
  int per_sm = 0;
  CKL(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_lu_trsv<double2, 4>, TS_TH, 0), "solve occupancy");
  w->coop_blocks = per_sm * w->sms;
  if (w->coop_blocks <= 0) {
    snprintf(w->err, sizeof(w->err), "triangular solve: no resident block");
    return -1;
  }
  CKL(cudaStreamCreateWithFlags(&w->side, cudaStreamNonBlocking), "LU side stream");
  CKL(cudaEventCreateWithFlags(&w->ev_fork, cudaEventDisableTiming), "LU events");
  CKL(cudaEventCreateWithFlags(&w->ev_join, cudaEventDisableTiming), "LU events");
  CKL(cudaMalloc(&w->piv, PV_INTS * sizeof(int)), "LU scratch");
  CKL(cudaMalloc(&w->u11, U_COUNT * sizeof(double2)), "LU scratch");
  CKL(cudaMalloc(&w->status, sizeof(unsigned)), "LU status");
  CKL(cudaMemset(w->status, 0, sizeof(unsigned)), "LU status");
  return 0;
}

extern "C" void bem_lu_free(bem_lu *w) {
  if (w->gexec) cudaGraphExecDestroy(w->gexec);
  if (w->graph) cudaGraphDestroy(w->graph);
  cudaFree(w->rowmap);
  cudaFree(w->piv);
  cudaFree(w->u11);
  cudaFree(w->status);
  cudaFree(w->flags);
  cudaFree(w->y);
  if (w->ev_fork) cudaEventDestroy(w->ev_fork);
  if (w->ev_join) cudaEventDestroy(w->ev_join);
  if (w->side) cudaStreamDestroy(w->side);
  *w = bem_lu();
}

static int grow_bytes(bem_lu *w, void **p, size_t *cap, size_t bytes, const char *what) {
  if (*cap >= bytes) return 0;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  CKL(cudaMalloc(p, bytes), what);
  *cap = bytes;
  return 0;
}

// C = A[r0:n, c0:cend) -= A[r0:n, kk:kk+kw) A[kk:kk+kw, c0:cend)
static void launch_update(double2 *A, int n, int kk, int kw, int r0, int c0, int cend, cudaStream_t st) {
  const dim3 grid((cend - c0 + UP_BN - 1) / UP_BN, (n - r0 + UP_BM - 1) / UP_BM);
  k_lu_update<<<grid, UP_TH, UP_SMEM, st>>>(A, n, n, kk, kw, r0, c0, cend);
}
static void launch_update(float2 *A, int n, int kk, int kw, int r0, int c0, int cend, cudaStream_t st) {
  const dim3 grid((cend - c0 + UP_BN - 1) / UP_BN, (n - r0 + UP_BM - 1) / UP_BM);
  k_lu_update_c32<<<grid, UF_TH, 0, st>>>(A, n, n, kk, kw, r0, c0, cend);
}

// an outer block's update of a complex FP32 factorisation on the tensor cores
// when the LU has them (returns 1 when launched)
static int tc_update(bem_lu *w, double2 *, int, int, cudaStream_t) { (void)w; return 0; }
static int tc_update(bem_lu *w, float2 *A, int n, int K, cudaStream_t st) {
  if (!w->tc || !w->tc->ready) return 0;
  bem_tc_launch(w->tc, A, n, n, K, w->status, st);
  return 1;
}

// the launches of one factorisation, in order (captured into the graph, whose
// replays count them).  Outer blocks of LU_OB columns: each panel's update
// covers only the rest of its outer block; the columns right of the block get
// the row moves as the panels go, then U12 (k_lu_trsm) and one rank-LU_OB
// update, so the trailing matrix is read and written once per outer block
// instead of once per panel.  Look-ahead: a panel's update is split into the
// next panel's 32 columns (on st, before the next panel) and the rest (on the
// side stream, beside the next panel); the next row moves wait for the rest.
template <class C2>
static int factor_launches(bem_lu *w, C2 *A, int n, cudaStream_t st) {
  k_lu_iota<<<(n + 255) / 256, 256, 0, st>>>(w->rowmap, n);
  // up to one_block_max the whole matrix is one outer block (every panel
  // updates the whole trailing matrix: fewer, shorter launches on the
  // critical path of a small factorisation)
  const int one_block = w->one_block_max > 0 ? w->one_block_max : LU_ONE_BLOCK_N;
  const int obw = n <= one_block ? n : LU_OB;
  bool pending = false;  // update work on the side stream not yet joined
  for (int K = 0; K < n; K += obw) {
    const int cend = n - K < obw ? n : K + obw;
    for (int k = K; k < cend; k += LU_W) {
      const int wd = n - k < LU_W ? n - k : LU_W;
      const int r0 = k + wd;
      k_lu_panel<C2><<<LU_CL, LU_TH, sizeof(panel_sh<C2>), st>>>(A, n, n, k, w->piv, (C2 *)w->u11, w->status);
      if (pending) {
        CKL(cudaStreamWaitEvent(st, w->ev_join, 0), "LU join");
        pending = false;
      }
      const int nL = (n - r0 + AP_ROWS - 1) / AP_ROWS;
      const int nC = (k + AP_COLS - 1) / AP_COLS + (n - r0 + AP_COLS - 1) / AP_COLS;
      k_lu_apply<C2><<<nL + nC + 1, AP_TH, 0, st>>>(A, n, n, k, cend, w->piv, (const C2 *)w->u11, w->rowmap,
                                                    w->status);
      if (r0 < cend) {
        const int nxt = cend - r0 < LU_W ? cend : r0 + LU_W;
        launch_update(A, n, k, wd, r0, r0, nxt, st);
        if (nxt < cend) {
          CKL(cudaEventRecord(w->ev_fork, st), "LU fork");
          CKL(cudaStreamWaitEvent(w->side, w->ev_fork, 0), "LU fork");
          launch_update(A, n, k, wd, r0, nxt, cend, w->side);
          CKL(cudaEventRecord(w->ev_join, w->side), "LU join");
          pending = true;
        }
      }
    }
    if (pending) {
      CKL(cudaStreamWaitEvent(st, w->ev_join, 0), "LU join");
      pending = false;
    }
    if (cend < n) {
      k_lu_trsm<C2><<<(n - cend + TR_NC - 1) / TR_NC, TR_TH, sizeof(trsm_sh<C2>), st>>>(A, n, n, K, cend - K,
                                                                                         (const C2 *)w->u11);
      if (tc_update(w, A, n, K, st) == 0) launch_update(A, n, K, cend - K, cend, cend, n, st);
    }
  }
  CKL(cudaGetLastError(), "LU launch");
  return 0;
}

template <class C2>
static int lu_factor(bem_lu *w, void *Av, int n, cudaStream_t st) {
  if (n <= 0) return 0;
  C2 *A = (C2 *)Av;
  if (grow_bytes(w, (void **)&w->rowmap, &w->rowmap_cap, (size_t)n * sizeof(int), "row map")) return -1;
  const int tcmode = (sizeof(C2) == sizeof(float2) && w->tc && w->tc->ready) ? w->tc->nprod : 0;
  if (!(w->gexec && w->g_A == Av && w->g_n == n && w->g_tc == tcmode && w->g_obm == w->one_block_max)) {
    if (w->gexec) cudaGraphExecDestroy(w->gexec);
    if (w->graph) cudaGraphDestroy(w->graph);
    w->gexec = nullptr;
    w->graph = nullptr;
    CKL(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "LU capture");
    const int rc = factor_launches(w, A, n, st);
    cudaGraph_t g = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(st, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    CKL(ce, "LU capture");
    w->graph = g;
    CKL(cudaGraphInstantiate(&w->gexec, g, 0), "LU graph");
    size_t nodes = 0;
    CKL(cudaGraphGetNodes(g, nullptr, &nodes), "LU graph");
    w->g_nodes = nodes;
    w->g_obm = w->one_block_max;
    w->g_A = Av;
    w->g_n = n;
    w->g_tc = tcmode;
  }
  CKL(cudaGraphLaunch(w->gexec, st), "LU graph launch");
  bem_count_launches(w->g_nodes);
  return 0;
}

extern "C" void bem_lu_set_one_block(bem_lu *w, int nmax) { w->one_block_max = nmax; }
extern "C" int bem_lu_factor_z(bem_lu *w, double *A, int n, cudaStream_t st) { return lu_factor<double2>(w, A, n, st); }
extern "C" int bem_lu_factor_c(bem_lu *w, float *A, int n, cudaStream_t st) { return lu_factor<float2>(w, A, n, st); }

template <class C2, int NR>
static int launch_trsv(bem_lu *w, const C2 *LU, int n, const C2 *in, C2 *out, unsigned *flags, int lower,
                       cudaStream_t st) {
  const int nb = (n + 31) / 32;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(nb < w->coop_blocks ? nb : w->coop_blocks);
  cfg.blockDim = dim3(TS_TH);
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  CKL(cudaLaunchKernelEx(&cfg, k_lu_trsv<C2, NR>, LU, (long)n, n, (const int *)w->rowmap, in, out, flags, lower,
                         w->status),
      "triangular solve");
  bem_count_launches(1);
  return 0;
}

template <class C2>
static int lu_solve(bem_lu *w, const void *LUv, int n, int nrhs, void *Bv, cudaStream_t st) {
  if (n <= 0) return 0;
  if (nrhs < 1 || nrhs > 4) {
    snprintf(w->err, sizeof(w->err), "LU solve: %d right-hand sides (1..4)", nrhs);
    return -1;
  }
  if (grow_bytes(w, (void **)&w->flags, &w->flags_cap, 2 * TS_FSTRIDE * sizeof(unsigned), "solve flags") ||
      grow_bytes(w, &w->y, &w->y_cap, (size_t)n * nrhs * sizeof(C2), "solve scratch"))
    return -1;
  const C2 *LU = (const C2 *)LUv;
  C2 *B = (C2 *)Bv, *Y = (C2 *)w->y;
  CKL(cudaMemsetAsync(w->flags, 0, 2 * TS_FSTRIDE * sizeof(unsigned), st), "solve flags");
  int rc = 0;
  switch (nrhs) {
    case 1: rc = launch_trsv<C2, 1>(w, LU, n, B, Y, w->flags, 1, st) || launch_trsv<C2, 1>(w, LU, n, Y, B, w->flags + TS_FSTRIDE, 0, st); break;
    case 2: rc = launch_trsv<C2, 2>(w, LU, n, B, Y, w->flags, 1, st) || launch_trsv<C2, 2>(w, LU, n, Y, B, w->flags + TS_FSTRIDE, 0, st); break;
    case 3: rc = launch_trsv<C2, 3>(w, LU, n, B, Y, w->flags, 1, st) || launch_trsv<C2, 3>(w, LU, n, Y, B, w->flags + TS_FSTRIDE, 0, st); break;
    default: rc = launch_trsv<C2, 4>(w, LU, n, B, Y, w->flags, 1, st) || launch_trsv<C2, 4>(w, LU, n, Y, B, w->flags + TS_FSTRIDE, 0, st); break;
  }
  return rc ? -1 : 0;
}

extern "C" int bem_lu_solve_z(bem_lu *w, const double *LU, int n, int nrhs, double *B, cudaStream_t st) {
  return lu_solve<double2>(w, LU, n, nrhs, B, st);
}
extern "C" int bem_lu_solve_c(bem_lu *w, const float *LU, int n, int nrhs, float *B, cudaStream_t st) {
  return lu_solve<float2>(w, LU, n, nrhs, B, st);
}

extern "C" int bem_lu_resid_z(const double *A, int n, int nrhs, const double *X, const double *B, double *R,
                              cudaStream_t st) {
  const int blocks = (n + 7) / 8;
  const double2 *a = (const double2 *)A, *x = (const double2 *)X, *b = (const double2 *)B;
  double2 *r = (double2 *)R;
  switch (nrhs) {
    case 1: k_resid_z<1><<<blocks, 256, 0, st>>>(a, n, x, b, r); bem_count_launches(1); break;
    case 2: k_resid_z<2><<<blocks, 256, 0, st>>>(a, n, x, b, r); bem_count_launches(1); break;
    case 3: k_resid_z<3><<<blocks, 256, 0, st>>>(a, n, x, b, r); bem_count_launches(1); break;
    case 4: k_resid_z<4><<<blocks, 256, 0, st>>>(a, n, x, b, r); bem_count_launches(1); break;
    default: return -1;
  }
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" unsigned bem_lu_status(bem_lu *w, cudaStream_t st) {
  unsigned s = 0;
  if (cudaMemcpyAsync(&s, w->status, sizeof(unsigned), cudaMemcpyDeviceToHost, st) != cudaSuccess) return 0xffffffffu;
  if (cudaStreamSynchronize(st) != cudaSuccess) return 0xffffffffu;
  cudaMemsetAsync(w->status, 0, sizeof(unsigned), st);
  return s;
}
