// Boundary-integral coefficient matrices of one domain on the device.
//
// Replaces create_cmatrix_domain (d3qd2_src/bem3_aw_qd2_solve_bieq.c:133-218)
// and the element integrals it calls.  Outputs use the reference's layout so
// they can be compared with its temporary files entry by entry:
//   G[p][4 s + i], H[p][4 s + i]   (N x N, row-major complex128, p = 4 t + tn)
//   dG[2 p + {0,1}][4 s + i], dH   (2N x N, tangential derivatives, interior only)
//   dF[p][3] = {(1+)F, dF/dt_zeta, dF/dt_eta}
//
// Work is split by pair class, each class in its own kernel:
//   classify  geometric F, dF/dt on 12x12 points for every (p, s); flags the
//             near-singular pairs (|dF/dt| > 0.5, d3qd2_elem.c:851,537)
//   regular   12x12 points: periodic domain one thread per point (each point is
//             a full quasi-periodic Green's function, ~100 lattice terms);
//             free-space domain one thread per pair (cheap integrand)
//   near      64x64 points for flagged pairs, one block per pair
//   self      singular polar quadrature on the collocation element, one block
//             per collocation node
//   diag      adds (1+)F to the diagonal of H and writes dF
#include "bem_count.h"
#include <cuda_runtime.h>
#include <stdint.h>
#include "bem_qpgf.cuh"
#include "bem_geom.cuh"
#include "bem_kernels.h"


// ------------------------------------------------------------------ helpers
struct bem_node { double rt[3], vz[3], vt[3]; };  // collocation point, unit tangents

__device__ __forceinline__ void bem_load_node(const bem_dom_dev &D, int p, bem_node &n, int &t, int &te) {
  t = p >> 2;
  const int tn = p & 3;
  te = abs(D.sid[t]) - 1;
#pragma unroll
  for (int d = 0; d < 3; ++d) n.rt[d] = __ldg(D.ren + (size_t)te * 12 + tn * 3 + d);
  // tz_te_bd_node (d3qd2_elem.c:125)
  double az = 0, ae = 0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    n.vz[d] = __ldg(D.cr + (size_t)te * 12 + d * 4 + 1) + __ldg(D.cr + (size_t)te * 12 + d * 4 + 3) * c_q.et[tn];
    n.vt[d] = __ldg(D.cr + (size_t)te * 12 + d * 4 + 2) + __ldg(D.cr + (size_t)te * 12 + d * 4 + 3) * c_q.zt[tn];
    az += n.vz[d] * n.vz[d];
    ae += n.vt[d] * n.vt[d];
  }
  az = sqrt(az);
  ae = sqrt(ae);
#pragma unroll
  for (int d = 0; d < 3; ++d) { n.vz[d] /= az; n.vt[d] /= ae; }
}

__device__ __forceinline__ double dot3(const double a[3], const double b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// element e (0-based) is a linear triangle
__device__ __forceinline__ bool bem_is_tri(const bem_dom_dev &D, int e) { return D.has_tri && __ldg(D.npe + e) == 3; }
// row p = 4 t + 3 of a triangle t is padding: the reference leaves it zero
// (create_cmatrix_domain computes tn < 3 for triangles, bem3_aw_qd2_solve_bieq.c:160-161)
__device__ __forceinline__ bool bem_pad_row(const bem_dom_dev &D, int p) {
  return (p & 3) == 3 && bem_is_tri(D, abs(D.sid[p >> 2]) - 1);
}

__device__ __forceinline__ void set_status(unsigned *st, unsigned bits) { if (bits) atomicOr(st, bits); }

// warp-aggregated work counters (lattice terms and Green's-function points);
// every lane of the warp must call it
__device__ __forceinline__ void count_work(unsigned long long *ctr, unsigned long long terms, unsigned long long pts) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    terms += __shfl_down_sync(0xffffffffu, terms, o);
    pts += __shfl_down_sync(0xffffffffu, pts, o);
  }
  if ((threadIdx.x & 31) == 0 && pts) {
    atomicAdd(ctr, terms);
    atomicAdd(ctr + 3, pts);
  }
}

// geometric F and its tangential derivatives at one quadrature point:
// tD = (R.W)/R^3, dF_v = (3 (R.v)(R.W)/R^2 - W.v)/R^3   (q0_bil_dcoef_v2_cc.c:165-200)
__device__ __forceinline__ void geomF(const double vR[3], const double vW[3], const bem_node &n, double &f, double &fz, double &fe) {
  const double aR = sqrt(vR[0] * vR[0] + vR[1] * vR[1] + vR[2] * vR[2]);
  const double iR = 1.0 / aR;
  const double rdW = dot3(vR, vW) * iR;
  const double rdz = dot3(vR, n.vz) * iR, rde = dot3(vR, n.vt) * iR;
  const double Wdz = dot3(vW, n.vz), Wde = dot3(vW, n.vt);
  const double i3 = iR * iR * iR;
  f = rdW * iR * iR;
  fz = i3 * (3.0 * rdz * rdW - Wdz);
  fe = i3 * (3.0 * rde * rdW - Wde);
}

// ------------------------------------------------------------------ classify
// One block per collocation node p; threads stride over source elements.
// Regular pairs of the periodic domain on a shorter rule (flag 3 + t, tier t):
// a source element whose centre is at least d_t circumradii R from the nearest
// lattice image of the collocation node, with k R <= kR_t, is integrated with
// the n_t x n_t Gauss rule on a quad (the collapsed rule over the whole
// triangle on a triangle) instead of the reference's 12 x 12 per quad or
// triangle part.  There the integrand is analytic well beyond the element (its
// nearest singularity is that image) and turns by at most k R in phase across it:
//    t   n_t   d_t   kR_t   (triangles: d_t, kR_t)
//    0   10    3     1
//    1    9    3.5   1
//    2    8    5     1
//    3    7    8     0.5    (6, 0.5)
//    4    6    25    0.2    (12, 0.5)
// Each rule gives the converged integral (and so the reference's 12 x 12,
// itself converged there) to about 1e-13 of the pair's largest entry: checked
// against 40 x 40 on curved and on twisted quads, on triangles with angles of
// 25 degrees and more, and on the cube-sphere and spheroid elements.  Tiers
// 0, 1, 3 and 4 also need a quad that is nearly flat and not long: the part of
// its twist c3 along the normal c1 x c2 at most a tenth of its shorter
// half-side |c1| or |c2| (cube-sphere and spheroid quads: under 0.05), and the
// longer half-side at most 3 times the shorter (a twisted quad's area element
// |W| has complex zeros near the element, which the shorter rules feel first;
// at a quarter the 6-point tier is off by 1e-11); other quads keep tier 2 or
// the reference rule.
struct bem_far { int on; double d1x, d1y, d2x, d2y, idet, k; };
__device__ __forceinline__ bool quad_tier_shape(const bem_el &el) {
  double c1[3], c2[3], c3[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) { c1[d] = el.cr[d][1]; c2[d] = el.cr[d][2]; c3[d] = el.cr[d][3]; }
  const double n0 = c1[1] * c2[2] - c1[2] * c2[1], n1 = c1[2] * c2[0] - c1[0] * c2[2], n2 = c1[0] * c2[1] - c1[1] * c2[0];
  const double nn = sqrt(n0 * n0 + n1 * n1 + n2 * n2);
  const double l1 = sqrt(dot3(c1, c1)), l2 = sqrt(dot3(c2, c2));
  const double lmin = fmin(l1, l2), lmax = fmax(l1, l2);
  return nn > 0.0 && fabs(c3[0] * n0 + c3[1] * n1 + c3[2] * n2) <= 0.1 * lmin * nn && lmax <= 3.0 * lmin;
}
// (distance from the element's centre (a triangle's centroid) to the nearest
// lattice image of rt) / (the element's circumradius R about that centre),
// squared, and (k R)^2.
__device__ __forceinline__ double pair_ratio2(const bem_far &fr, const bem_el &el, const double rt[3], bool tri,
                                              double &kR2) {
  // corners (+-1, +-1) of a quad, (1, 0), (-1/2, +-sqrt3/2) of a triangle
  double R2 = 0.0;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    double sz = (c == 1 || c == 2) ? 1.0 : -1.0, se = c >= 2 ? 1.0 : -1.0;
    if (tri) {
      sz = c == 0 ? 1.0 : -0.5;
      se = c == 0 ? 0.0 : (c == 1 ? 0.5 * BEM_SQ3 : -0.5 * BEM_SQ3);
    }
    double v2 = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double v = el.cr[d][1] * sz + el.cr[d][2] * se + el.cr[d][3] * sz * se;
      v2 += v * v;
    }
    R2 = fmax(R2, v2);
  }
  kR2 = fr.k * fr.k * R2;
  const double vz = rt[2] - el.cr[2][0];
  const double vx = rt[0] - el.cr[0][0], vy = rt[1] - el.cr[1][0];
  const double l1 = floor((vx * fr.d2y - vy * fr.d2x) * fr.idet + 0.5);
  const double l2 = floor(-(vx * fr.d1y - vy * fr.d1x) * fr.idet + 0.5);
  double dmin2 = 1e300;
  for (int a = -1; a <= 1; ++a)
    for (int b = -1; b <= 1; ++b) {
      const double x = vx - (l1 + a) * fr.d1x - (l2 + b) * fr.d2x, y = vy - (l1 + a) * fr.d1y - (l2 + b) * fr.d2y;
      dmin2 = fmin(dmin2, x * x + y * y + vz * vz);
    }
  return dmin2 / R2;
}
// Quadrature points closer than this to the lattice plane through the node
// keep a pair on the reference's rule: there the reference's lattice sums
// stop on rounding-decided zeros, so its values at its own points are not a
// smooth function that another rule could reproduce.
#define BEM_FAR_PLANE_TOL 1e-10
// point (i, j) of tier t's rule: Gauss on a quad; on a triangle the collapsed
// (Duffy) rule over the whole reference triangle, (z, e) = (1 - 3u/2,
// sqrt3/2 u (1 - 2v)) for (u, v) in [0, 1]^2, weight u w_u w_v
__device__ __forceinline__ void tier_point(int t, bool tri, int i, int j, double &z, double &e) {
  if (tri) {
    const double u = 0.5 * (c_q.xt[t][i] + 1.0), v = 0.5 * (c_q.xt[t][j] + 1.0);
    z = 1.0 - 1.5 * u;
    e = 0.5 * BEM_SQ3 * u * (1.0 - 2.0 * v);
  } else {
    z = c_q.xt[t][i];
    e = c_q.xt[t][j];
  }
}
// tier of a regular pair, or -1 for the reference's rule (whose points the
// caller has checked against the lattice plane); none of the tier's points
// may lie within BEM_FAR_PLANE_TOL of rt's lattice plane either
__device__ __forceinline__ int far_tier(const bem_far &fr, const bem_el &el, const double rt[3], bool tri) {
  double kR2;
  const double r2 = pair_ratio2(fr, el, rt, tri, kR2);
  if (kR2 > 1.0) return -1;
  int t;
  if (tri)  // flat triangles converge faster: 7 points from 6 R, 6 from 12 R (k R <= 0.5)
    t = r2 >= 144.0 && kR2 <= 0.25 ? 4 : r2 >= 36.0 && kR2 <= 0.25 ? 3 : r2 >= 25.0 ? 2 : r2 >= 12.25 ? 1 : r2 >= 9.0 ? 0 : -1;
  else if (!quad_tier_shape(el))
    t = r2 >= 25.0 ? 2 : -1;
  else
    t = r2 >= 625.0 && kR2 <= 0.04 ? 4 : r2 >= 64.0 && kR2 <= 0.25 ? 3 : r2 >= 25.0 ? 2 : r2 >= 12.25 ? 1 : r2 >= 9.0 ? 0 : -1;
  if (t < 0) return -1;
  // |z(zeta, eta) - c0z| <= |c1z| + |c2z| + |c3z| over the element
  const double zr = fabs(el.cr[2][1]) + fabs(el.cr[2][2]) + fabs(el.cr[2][3]);
  if (fabs(el.cr[2][0] - rt[2]) - zr > 2.0 * BEM_FAR_PLANE_TOL) return t;
  const int n = BEM_TIER_N0 - t;
  for (int ij = 0; ij < n * n; ++ij) {
    double z, e, r[3], w[3];
    tier_point(t, tri, ij / n, ij % n, z, e);
    bem_rw(el, z, e, r, w);
    if (fabs(r[2] - rt[2]) < BEM_FAR_PLANE_TOL) return -1;
  }
  return t;
}

// Compacted pair lists: k_classify counts the regular pairs (list 0, flag 0)
// and each tier's pairs (list 1 + t, flag 3 + t) into n[0 .. BEM_NTIER];
// k_plist_fill writes them, as p * ne + s, list after list into one buffer.  A
// kernel given a list runs a fixed grid over it; given none, it covers the
// pair range [pair0, pair0 + npairs) one block per unit group and checks flags.
#define BEM_NLIST (1 + BEM_NTIER)
struct bem_plist {
  const unsigned *e;  // all lists (null: pair-range mode)
  const unsigned *n;  // list lengths n[0 .. BEM_NLIST - 1], then BEM_NLIST fill counters
  int type;           // this kernel's list
};
__device__ __forceinline__ long long plist_units(const bem_plist &L, long long npairs) {
  return L.e ? (long long)L.n[L.type] : npairs;
}
__device__ __forceinline__ unsigned long long plist_base(const bem_plist &L) {
  unsigned long long b = 0;
  if (L.e)
    for (int t = 0; t < L.type; ++t) b += L.n[t];
  return b;
}
__device__ __forceinline__ long long plist_pair(const bem_plist &L, unsigned long long base, long long pair0, long long u) {
  return L.e ? (long long)L.e[base + u] : pair0 + u;
}
__device__ __forceinline__ int plist_of_flag(uint8_t fl) { return fl == 0 ? 0 : fl >= 3 ? fl - 2 : -1; }

__global__ void __launch_bounds__(128) k_classify(bem_dom_dev D, bem_far fr, double *__restrict__ rowF,
                                                   int *__restrict__ near_s, int *__restrict__ near_n,
                                                   uint8_t *__restrict__ flag, unsigned *status,
                                                   unsigned *__restrict__ lcnt) {
  const int p = blockIdx.x;
  if (bem_pad_row(D, p)) {
    for (int s = threadIdx.x; s < D.ne; s += blockDim.x) flag[(size_t)p * D.ne + s] = 0;
    if (threadIdx.x == 0) {
      near_n[p] = 0;
      rowF[3 * p] = rowF[3 * p + 1] = rowF[3 * p + 2] = 0.0;
    }
    return;
  }
  bem_node nd;
  int t, te;
  bem_load_node(D, p, nd, t, te);
  __shared__ int cnt;
  __shared__ int list[BEM_MAXNEAR];
  __shared__ double red[3][128];
  if (threadIdx.x == 0) cnt = 0;
  __syncthreads();
  double sF = 0, sFz = 0, sFe = 0;
  for (int s = threadIdx.x; s < D.ne; s += blockDim.x) {
    const int se = abs(D.sid[s]) - 1;
    uint8_t fl = 0;
    if (se == te) {
      fl = 2;  // self pair
    } else {
      bem_el el;
      bem_load_el(D.cr, D.cw, se, el);
      const bool tri = bem_is_tri(D, se);
      double F = 0, Fz = 0, Fe = 0, rzmin = 1e300;
      for (int part = 0; part < (tri ? 3 : 1); ++part)
        for (int i = 0; i < BEM_GLN; ++i) {
          double f = 0, fz = 0, fe = 0;
          for (int j = 0; j < BEM_GLN; ++j) {
            double z = c_q.xl[i], e = c_q.xl[j], wf = 1.0;
            if (tri) {
              bem_tri_point(part, z, e, z, e);
              wf = bem_tri_wfac(c_q.xl[i], c_q.xl[j]);
            }
            double vR[3], vW[3];
            bem_rw(el, z, e, vR, vW);
            for (int d = 0; d < 3; ++d) vR[d] -= nd.rt[d];
            rzmin = fmin(rzmin, fabs(vR[2]));
            double a, b, c;
            geomF(vR, vW, nd, a, b, c);
            f += c_q.wl[j] * wf * a;
            fz += c_q.wl[j] * wf * b;
            fe += c_q.wl[j] * wf * c;
          }
          F += c_q.wl[i] * f;
          Fz += c_q.wl[i] * fz;
          Fe += c_q.wl[i] * fe;
        }
      F *= BEM_I_FP; Fz *= BEM_I_FP; Fe *= BEM_I_FP;
      if (D.sid[s] < 0) { F = -F; Fz = -Fz; Fe = -Fe; }  // bil_convert_CC / _dCC
      if (fabs(Fz) > BEM_CBD_SDF || fabs(Fe) > BEM_CBD_SDF) {
        fl = 1;
        const int k = atomicAdd(&cnt, 1);
        if (k < D.near_cap) list[k] = s;
      } else {
        sF += F; sFz += Fz; sFe += Fe;
        if (fr.on && rzmin >= BEM_FAR_PLANE_TOL) {
          const int tier = far_tier(fr, el, nd.rt, tri);
          if (tier >= 0) fl = (uint8_t)(3 + tier);
        }
      }
    }
    flag[(size_t)p * D.ne + s] = fl;
  }
  red[0][threadIdx.x] = sF;
  red[1][threadIdx.x] = sFz;
  red[2][threadIdx.x] = sFe;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      for (int c = 0; c < 3; ++c) red[c][threadIdx.x] += red[c][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    int n = cnt;
    if (n > D.near_cap) { set_status(status, BEM_ST_NEAR_OVERFLOW); n = D.near_cap; }
    // deterministic order: sort the row's near-singular sources by index
    for (int a = 1; a < n; ++a) {
      const int v = list[a];
      int b = a - 1;
      while (b >= 0 && list[b] > v) { list[b + 1] = list[b]; --b; }
      list[b + 1] = v;
    }
    for (int a = 0; a < n; ++a) near_s[(size_t)p * D.near_cap + a] = list[a];
    near_n[p] = n;
    rowF[3 * p + 0] = red[0][0];
    rowF[3 * p + 1] = red[1][0];
    rowF[3 * p + 2] = red[2][0];
  }
  if (!lcnt) return;
  // this row's pairs counted into the list lengths (flags written above by this block)
  __shared__ unsigned nl[BEM_NLIST];
  if (threadIdx.x < BEM_NLIST) nl[threadIdx.x] = 0;
  __syncthreads();
  for (int s = threadIdx.x; s < D.ne; s += blockDim.x) {
    const int l = plist_of_flag(flag[(size_t)p * D.ne + s]);
    if (l >= 0) atomicAdd(&nl[l], 1u);
  }
  __syncthreads();
  if (threadIdx.x < BEM_NLIST && nl[threadIdx.x]) atomicAdd(lcnt + threadIdx.x, nl[threadIdx.x]);
}

// One block per row p: the row's pairs into the lists whose lengths k_classify
// counted (lcnt[0 .. BEM_NLIST - 1]); lcnt[BEM_NLIST + l] hands out the places
// of list l.  Order within a list is immaterial: each pair writes its own entries.
__global__ void __launch_bounds__(128) k_plist_fill(bem_dom_dev D, const uint8_t *__restrict__ flag,
                                                    unsigned *__restrict__ lst, unsigned *__restrict__ lcnt,
                                                    unsigned long long lcap) {
  const int p = blockIdx.x;
  if (bem_pad_row(D, p)) return;  // k_classify counts no pair of a padding row
  __shared__ unsigned nl[BEM_NLIST];
  __shared__ unsigned long long at[BEM_NLIST];
  if (threadIdx.x < BEM_NLIST) nl[threadIdx.x] = 0;
  __syncthreads();
  for (int s = threadIdx.x; s < D.ne; s += blockDim.x) {
    const int l = plist_of_flag(flag[(size_t)p * D.ne + s]);
    if (l >= 0) atomicAdd(&nl[l], 1u);
  }
  __syncthreads();
  if (threadIdx.x < BEM_NLIST) {
    const int l = threadIdx.x;
    unsigned long long base = 0;
    for (int m = 0; m < l; ++m) base += lcnt[m];
    at[l] = base + (nl[l] ? atomicAdd(lcnt + BEM_NLIST + l, nl[l]) : 0u);
    nl[l] = 0;
  }
  __syncthreads();
  for (int s = threadIdx.x; s < D.ne; s += blockDim.x) {
    const int l = plist_of_flag(flag[(size_t)p * D.ne + s]);
    if (l < 0) continue;
    const unsigned long long u = at[l] + atomicAdd(&nl[l], 1u);
    if (u < lcap) lst[u] = (unsigned)((size_t)p * D.ne + s);
  }
}

// ------------------------------------------------------------------ batches of Bloch vectors
// A batch: nb problems on one body, media, lattice and frequency that differ
// only in the in-plane Bloch wave vector (and incident field).  Their pair
// flags, pair lists, near lists and real-space term table are the same; each
// has its own Ewald parameters (bem_qp: Bloch phases, spectral table) and its
// own G and H.  The batched kernels (BA = bem_bat) read instance b's
// parameters from the argument block (qp[b], like a single problem's q0) and
// write G[b], H[b].
#ifndef BEM_BAT_MAX
// instances per launch: the parameters travel in the kernel's argument block,
// and the regular-pair kernels unroll their instance loop, so that each copy
// reads its instance's parameters at fixed offsets (as constant-bank operands)
#define BEM_BAT_MAX 8
#endif
struct bem_bat {
  int nb;
  bem_qp qp[BEM_BAT_MAX];
  double *G[BEM_BAT_MAX];
  double *H[BEM_BAT_MAX];
};
struct bat_none {};  // a single problem: the kernel's own q0, G0, H0
__device__ __forceinline__ int bat_n(const bat_none &) { return 1; }
__device__ __forceinline__ int bat_n(const bem_bat &B) { return B.nb; }
__device__ __forceinline__ const bem_qp &bat_q(const bat_none &, int, const bem_qp &q0) { return q0; }
__device__ __forceinline__ const bem_qp &bat_q(const bem_bat &B, int b, const bem_qp &) { return B.qp[b]; }
__device__ __forceinline__ double *bat_G(const bat_none &, int, double *G0) { return G0; }
__device__ __forceinline__ double *bat_G(const bem_bat &B, int b, double *) { return B.G[b]; }
__device__ __forceinline__ double *bat_H(const bat_none &, int, double *H0) { return H0; }
__device__ __forceinline__ double *bat_H(const bem_bat &B, int b, double *) { return B.H[b]; }
template <class BA> struct bat_is { static constexpr bool on = false; };
template <> struct bat_is<bem_bat> { static constexpr bool on = true; };
// trip count of a kernel's instance loop (unrolled)
template <class BA> struct bat_max { static constexpr int n = bat_is<BA>::on ? BEM_BAT_MAX : 1; };

// ------------------------------------------------------------------ periodic regular pairs
// 2 pairs x 144 points per block; one quasi-periodic Green's function per thread
// (q0_bil_dcoef_v2_cc_GL, q0_bil_dcoef_v2_cc.c:129-204, evaluated once per
// point and shared by the four interpolation functions).
#define RP_THREADS 288
#ifndef RP_MINB
#define RP_MINB 2  // two blocks (18 warps) per SM: caps registers at 113
#endif
template <class BA>
__global__ void __launch_bounds__(RP_THREADS, RP_MINB) k_q0_regular(bem_dom_dev D, const __grid_constant__ bem_qp q0, const uint8_t *__restrict__ flag,
                                                           double *G0, double *H0,
                                                           unsigned *status, unsigned long long *terms, long long pair0,
                                                           long long npairs, bem_plist L, const __grid_constant__ BA B) {
  __shared__ double acc[16][RP_THREADS + 1];
  extern __shared__ double2 wts_s[];  // BEM_WT_SMEM bytes of dynamic shared memory
  const double2 *wts = bem_wtab_stage(q0, wts_s);  // one table for every instance of a batch
  __syncthreads();
  const int lp = threadIdx.x / 144, pt = threadIdx.x % 144;
  const long long nu = plist_units(L, npairs);
  const unsigned long long lb = plist_base(L);
  unsigned long long nterm = 0, npt = 0;
#pragma unroll
  for (int b = 0; b < bat_max<BA>::n; ++b) {
  if (b >= bat_n(B)) break;
  double *__restrict__ G = bat_G(B, b, G0), *__restrict__ H = bat_H(B, b, H0);
  const bem_qp &q = bat_q(B, b, q0);
  for (long long u0 = 2LL * blockIdx.x; u0 < nu; u0 += 2LL * gridDim.x) {
    const bool valid = u0 + lp < nu;
    const long long pair = valid ? plist_pair(L, lb, pair0, u0 + lp) : 0;
    const int p = (int)(pair / D.ne);
    const int s = (int)(pair % D.ne);
    // triangle sources are k_q0_regular_tri's; padded rows keep their zeros
    const bool work = valid && flag[(size_t)p * D.ne + s] == 0 && !bem_is_tri(D, abs(D.sid[s]) - 1) && !bem_pad_row(D, p);
    double v[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) v[c] = 0.0;
    if (work) {
      bem_node nd;
      int t, te;
      bem_load_node(D, p, nd, t, te);
      bem_el el;
      bem_load_el(D.cr, D.cw, abs(D.sid[s]) - 1, el);
      const int i = pt / BEM_GLN, j = pt % BEM_GLN;
      const double z = c_q.xl[i], e = c_q.xl[j];
      double vR[3], vW[3];
      bem_rw(el, z, e, vR, vW);
      for (int d = 0; d < 3; ++d) vR[d] -= nd.rt[d];
      bem_gval gv;
      const int rc = bem_qpgf(q, vR[0], vR[1], vR[2], gv, wts);
      if (rc < 0) set_status(status, rc == -12 || rc == -23 ? BEM_ST_RAYLEIGH : BEM_ST_QPGF_LIMIT);
      nterm += rc > 0 ? (unsigned long long)rc : 0ULL;
      ++npt;
      const double aW = sqrt(vW[0] * vW[0] + vW[1] * vW[1] + vW[2] * vW[2]);
      const double wt = c_q.wl[i] * c_q.wl[j];
      const cplx g = cscale(gv.g, aW * wt);
      const cplx h = cscale(cadd(cadd(cscale(gv.gx, vW[0]), cscale(gv.gy, vW[1])), cscale(gv.gz, vW[2])), wt);
      double N[4];
      bem_Nn4(z, e, N);
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        v[2 * a] = g.re * N[a];
        v[2 * a + 1] = g.im * N[a];
        v[8 + 2 * a] = h.re * N[a];
        v[8 + 2 * a + 1] = h.im * N[a];
      }
    }
#pragma unroll
    for (int c = 0; c < 16; ++c) acc[c][threadIdx.x] = v[c];
    __syncthreads();
    if (threadIdx.x < 32) {
      const int q2 = threadIdx.x >> 4, c = threadIdx.x & 15;
      if (u0 + q2 < nu) {
        const long long pr = plist_pair(L, lb, pair0, u0 + q2);
        const int pp = (int)(pr / D.ne), ss = (int)(pr % D.ne);
        if (flag[(size_t)pp * D.ne + ss] == 0 && !bem_is_tri(D, abs(D.sid[ss]) - 1) && !bem_pad_row(D, pp)) {
          double sum = 0.0;
          for (int k = 0; k < 144; ++k) sum += acc[c][q2 * 144 + k];
          const size_t N = (size_t)D.ne * 4;
          double *dst = c < 8 ? G : H;
          const int a = (c & 7) >> 1, part = c & 1;
          dst[2 * ((size_t)pp * N + 4 * ss + a) + part] = sum;
        }
      }
    }
    __syncthreads();  // acc is rewritten by the next unit group
  }
  }
  count_work(terms + 0, nterm, npt);
}

// Triangle sources (q0_lit_dcoef_v2_cc_GL, q0_lit_dcoef_v2_cc.c:156-237 with
// q0_lit_sdqGHF_v2_cc_zeta_eta, :345-381): 3 parts x 12 x 12 points; a thread
// takes the 3 parts of one (a, b) point, 2 pairs per 288-thread block.
__global__ void __launch_bounds__(RP_THREADS, RP_MINB) k_q0_regular_tri(bem_dom_dev D, const __grid_constant__ bem_qp q,
                                                               const uint8_t *__restrict__ flag, double *__restrict__ G,
                                                               double *__restrict__ H, unsigned *status,
                                                               unsigned long long *terms, long long pair0,
                                                               long long npairs, bem_plist L) {
  __shared__ double acc[16][RP_THREADS + 1];
  extern __shared__ double2 wts_s[];  // BEM_WT_SMEM bytes of dynamic shared memory
  const double2 *wts = bem_wtab_stage(q, wts_s);
  __syncthreads();
  const int lp = threadIdx.x / 144, pt = threadIdx.x % 144;
  const long long nu = plist_units(L, npairs);
  const unsigned long long lb = plist_base(L);
  unsigned long long nterm = 0, npt = 0;
  for (long long u0 = 2LL * blockIdx.x; u0 < nu; u0 += 2LL * gridDim.x) {
    const bool valid = u0 + lp < nu;
    const long long pair = valid ? plist_pair(L, lb, pair0, u0 + lp) : 0;
    const int p = (int)(pair / D.ne);
    const int s = (int)(pair % D.ne);
    const bool work = valid && flag[(size_t)p * D.ne + s] == 0 && bem_is_tri(D, abs(D.sid[s]) - 1) && !bem_pad_row(D, p);
    // the 3 parts accumulate in this thread's shared-memory column, so that no
    // accumulator stays live in registers across the Green's-function calls
#pragma unroll
    for (int c = 0; c < 16; ++c) acc[c][threadIdx.x] = 0.0;
    if (work) {
      const int i = pt / BEM_GLN, j = pt % BEM_GLN;
      const int se = abs(D.sid[s]) - 1, te = abs(D.sid[p >> 2]) - 1;
      unsigned st = 0;
      for (int part = 0; part < 3; ++part) {
        // geometry is re-read (L1) per part rather than kept in registers
        // across the Green's-function calls
        double z, e, vR[3], vW[3];
        {
          const double a = c_q.xl[i], b = c_q.xl[j];
          bem_el el;
          bem_load_el(D.cr, D.cw, se, el);
          bem_tri_point_ref(part, a, b, z, e);
          bem_rw_ref(el, z, e, vR, vW);
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) vR[d] = __dsub_rn(vR[d], __ldg(D.ren + (size_t)te * 12 + (p & 3) * 3 + d));
        bem_gval gv;
        const int rc = bem_qpgf(q, vR[0], vR[1], vR[2], gv, wts);
        if (rc < 0) st |= rc == -12 || rc == -23 ? BEM_ST_RAYLEIGH : BEM_ST_QPGF_LIMIT;
        nterm += rc > 0 ? (unsigned long long)rc : 0ULL;
        ++npt;
        // a triangle's W is the constant cw[.][0]
#pragma unroll
        for (int d = 0; d < 3; ++d) vW[d] = __ldg(D.cw + (size_t)se * 9 + d * 3);
        const double a2 = c_q.xl[i], b2 = c_q.xl[j];
        bem_tri_point_ref(part, a2, b2, z, e);  // recomputed: not kept across the call
        const double wt = c_q.wl[i] * c_q.wl[j] * bem_tri_wfac(a2, b2);
        const double aW = sqrt(vW[0] * vW[0] + vW[1] * vW[1] + vW[2] * vW[2]);
        const cplx g = cscale(gv.g, aW * wt);
        const cplx h = cscale(cadd(cadd(cscale(gv.gx, vW[0]), cscale(gv.gy, vW[1])), cscale(gv.gz, vW[2])), wt);
        double N[4];
        bem_Nn3(z, e, N);
#pragma unroll
        for (int n = 0; n < 4; ++n) {
          acc[2 * n][threadIdx.x] += g.re * N[n];
          acc[2 * n + 1][threadIdx.x] += g.im * N[n];
          acc[8 + 2 * n][threadIdx.x] += h.re * N[n];
          acc[8 + 2 * n + 1][threadIdx.x] += h.im * N[n];
        }
      }
      set_status(status, st);
    }
    __syncthreads();
    if (threadIdx.x < 32) {
      const int q2 = threadIdx.x >> 4, c = threadIdx.x & 15;
      if (u0 + q2 < nu) {
        const long long pr = plist_pair(L, lb, pair0, u0 + q2);
        const int pp = (int)(pr / D.ne), ss = (int)(pr % D.ne);
        if (flag[(size_t)pp * D.ne + ss] == 0 && bem_is_tri(D, abs(D.sid[ss]) - 1) && !bem_pad_row(D, pp)) {
          double sum = 0.0;
          for (int k = 0; k < 144; ++k) sum += acc[c][q2 * 144 + k];
          const size_t N = (size_t)D.ne * 4;
          double *dst = c < 8 ? G : H;
          const int a = (c & 7) >> 1, part = c & 1;
          dst[2 * ((size_t)pp * N + 4 * ss + a) + part] = sum;
        }
      }
    }
    __syncthreads();  // acc is rewritten by the next unit group
  }
  count_work(terms + 0, nterm, npt);
}

// Regular pairs on tier t's shorter rule (flag 3 + t, far_tier): NF x NF
// points (NF = BEM_TIER_N0 - t), Gauss on a quad, collapsed over a triangle
// (tier_point; the weights u w_u w_v total 1/2, as the 3-part rule's do).  One
// thread per point, PB = FP_THREADS / NF^2 pairs per block, contributions
// accumulated in the thread's shared-memory column; otherwise as k_q0_regular /
// k_q0_regular_tri.
#define FP_THREADS 256
#ifndef FP_MINB
#define FP_MINB 2  // two blocks (16 warps) per SM: caps registers at 128
#endif
template <int NF>
struct far_shape {
  // TH threads hold points; the block has TB (whole warps), the rest idle
  static constexpr int NP = NF * NF, PB = FP_THREADS / NP, TH = PB * NP, TB = (TH + 31) / 32 * 32,
                       T = BEM_TIER_N0 - NF;
};
template <int NF, class BA>
__global__ void __launch_bounds__(FP_THREADS, FP_MINB) k_q0_far(bem_dom_dev D, const __grid_constant__ bem_qp q0,
                                                        const uint8_t *__restrict__ flag, double *G0,
                                                        double *H0, unsigned *status,
                                                        unsigned long long *terms, long long pair0, long long npairs,
                                                        bem_plist L, const __grid_constant__ BA B) {
  using F = far_shape<NF>;
  constexpr uint8_t FL = (uint8_t)(3 + F::T);
  __shared__ double acc[16][F::TB + 1];
  extern __shared__ double2 wts_s[];  // BEM_WT_SMEM bytes of dynamic shared memory
  const long long nu = plist_units(L, npairs);
  const unsigned long long lb = plist_base(L);
  if (!L.e) {
    // pair-range mode: a block none of whose pairs is on this tier stops
    // before staging the table
    bool mine = false;
    for (long long u0 = (long long)F::PB * blockIdx.x; u0 < nu; u0 += (long long)F::PB * gridDim.x)
      if (threadIdx.x < F::PB && u0 + threadIdx.x < nu) mine |= flag[pair0 + u0 + threadIdx.x] == FL;
    if (!__syncthreads_or(mine)) return;
  }
  const double2 *wts = bem_wtab_stage(q0, wts_s);  // one table for every instance of a batch
  __syncthreads();
  const int lp = threadIdx.x / F::NP, pt = threadIdx.x % F::NP;
  unsigned long long nterm = 0, npt = 0;
#pragma unroll
  for (int b = 0; b < bat_max<BA>::n; ++b) {
  if (b >= bat_n(B)) break;
  double *__restrict__ G = bat_G(B, b, G0), *__restrict__ H = bat_H(B, b, H0);
  const bem_qp &q = bat_q(B, b, q0);
  for (long long u0 = (long long)F::PB * blockIdx.x; u0 < nu; u0 += (long long)F::PB * gridDim.x) {
    const bool valid = threadIdx.x < F::TH && u0 + lp < nu;
    const long long pair = valid ? plist_pair(L, lb, pair0, u0 + lp) : 0;
    const int p = (int)(pair / D.ne);
    const int s = (int)(pair % D.ne);
    const bool work = valid && flag[(size_t)p * D.ne + s] == FL;
#pragma unroll
    for (int c = 0; c < 16; ++c) acc[c][threadIdx.x] = 0.0;
    if (work) {
      const int se = abs(D.sid[s]) - 1, te = abs(D.sid[p >> 2]) - 1;
      const bool tri = bem_is_tri(D, se);
      const int i = pt / NF, j = pt % NF;
      unsigned st = 0;
      {
        double z, e, vR[3], vW[3];
        {
          bem_el el;
          bem_load_el(D.cr, D.cw, se, el);
          tier_point(F::T, tri, i, j, z, e);
          bem_rw(el, z, e, vR, vW);
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) vR[d] -= __ldg(D.ren + (size_t)te * 12 + (p & 3) * 3 + d);
        bem_gval gv;
        const int rc = bem_qpgf(q, vR[0], vR[1], vR[2], gv, wts);
        if (rc < 0) st |= rc == -12 || rc == -23 ? BEM_ST_RAYLEIGH : BEM_ST_QPGF_LIMIT;
        nterm += rc > 0 ? (unsigned long long)rc : 0ULL;
        ++npt;
        // re-derived after the call rather than kept live across it
        double wt = c_q.wt[F::T][i] * c_q.wt[F::T][j];
        tier_point(F::T, tri, i, j, z, e);
        if (tri) {
#pragma unroll
          for (int d = 0; d < 3; ++d) vW[d] = __ldg(D.cw + (size_t)se * 9 + d * 3);
          wt *= 0.125 * (c_q.xt[F::T][i] + 1.0);  // u w_u w_v with u = (x + 1) / 2, w_u = w / 2
        } else {
          bem_el el;
          bem_load_el(D.cr, D.cw, se, el);
          double r[3];
          bem_rw(el, z, e, r, vW);
        }
        const double aW = sqrt(vW[0] * vW[0] + vW[1] * vW[1] + vW[2] * vW[2]);
        const cplx g = cscale(gv.g, aW * wt);
        const cplx h = cscale(cadd(cadd(cscale(gv.gx, vW[0]), cscale(gv.gy, vW[1])), cscale(gv.gz, vW[2])), wt);
        double N[4];
        if (tri) bem_Nn3(z, e, N);
        else bem_Nn4(z, e, N);
#pragma unroll
        for (int n = 0; n < 4; ++n) {
          acc[2 * n][threadIdx.x] += g.re * N[n];
          acc[2 * n + 1][threadIdx.x] += g.im * N[n];
          acc[8 + 2 * n][threadIdx.x] += h.re * N[n];
          acc[8 + 2 * n + 1][threadIdx.x] += h.im * N[n];
        }
      }
      set_status(status, st);
    }
    __syncthreads();
    if (threadIdx.x < 16 * F::PB) {
      const int qq = threadIdx.x >> 4, c = threadIdx.x & 15;
      if (u0 + qq < nu) {
        const long long pr = plist_pair(L, lb, pair0, u0 + qq);
        const int pp = (int)(pr / D.ne), ss = (int)(pr % D.ne);
        if (flag[(size_t)pp * D.ne + ss] == FL) {
          double sum = 0.0;
          for (int k = 0; k < F::NP; ++k) sum += acc[c][qq * F::NP + k];
          const size_t N = (size_t)D.ne * 4;
          double *dst = c < 8 ? G : H;
          const int a = (c & 7) >> 1, part = c & 1;
          dst[2 * ((size_t)pp * N + 4 * ss + a) + part] = sum;
        }
      }
    }
    __syncthreads();  // acc is rewritten by the next unit group
  }
  }
  count_work(terms + 0, nterm, npt);
}

// ------------------------------------------------------------------ periodic near-singular pairs
// 64x64 points (q0_bil_dcoef_v2_cc_GH, q0_bil_dcoef_v2_cc.c:206-281).
#define NP_THREADS 256
// The home-cell image of the quasi-periodic Green's function: the free-space
// e^{ikR} / (4 pi R) and its gradient at r, in bem_qpgf's conventions.  The
// near-singular and self integrals split G_qp = G0 + (G_qp - G0): G0 carries
// the whole singularity and costs a sincos, so it is integrated on the
// reference's own points (64 x 64 Gauss, the polar rule); the rest is smooth
// over the element (its nearest singularities are the other lattice images)
// and is integrated on the 12 x 12 Gauss rule of regular pairs, a lattice sum
// at 144 points instead of 4096 or 6144.
__device__ __forceinline__ void bem_g0(double k, const double vR[3], bem_gval &o) {
  const double R2 = vR[0] * vR[0] + vR[1] * vR[1] + vR[2] * vR[2];
  const double R = sqrt(R2), iR = 1.0 / R;
  const cplx ce = cexpi(k * R);
  const double c4 = 0.07957747154594766788 * iR;  // 1 / (4 pi R)
  o.g = cscale(ce, c4);
  // (i k R - 1) e^{ikR} / (4 pi R^3) times r
  const cplx f = cscale(cmul(cmk(-1.0, k * R), ce), c4 * iR * iR);
  o.gx = cscale(f, vR[0]);
  o.gy = cscale(f, vR[1]);
  o.gz = cscale(f, vR[2]);
}
// accumulate a point's G and H contributions: g = gv.g |W| wg, h = (grad gv . W) wh
__device__ __forceinline__ void acc_gh(double (&v)[19], const bem_gval &gv, const double vW[3], double wg, double wh,
                                       const double N[4]) {
  const cplx g = cscale(gv.g, wg);
  const cplx h = cscale(cadd(cadd(cscale(gv.gx, vW[0]), cscale(gv.gy, vW[1])), cscale(gv.gz, vW[2])), wh);
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    v[2 * a] += g.re * N[a];
    v[2 * a + 1] += g.im * N[a];
    v[8 + 2 * a] += h.re * N[a];
    v[8 + 2 * a + 1] += h.im * N[a];
  }
}
// gv -= g0
__device__ __forceinline__ void gval_sub(bem_gval &gv, const bem_gval &g0) {
  gv.g = csub(gv.g, g0.g);
  gv.gx = csub(gv.gx, g0.gx);
  gv.gy = csub(gv.gy, g0.gy);
  gv.gz = csub(gv.gz, g0.gz);
}

// point pt of the reference's near-singular rule (64 x 64, 3 parts of 64 x 64
// on a triangle, with the reference's rounding there): (z, e), weight, R from
// the node, W
__device__ __forceinline__ void near_point(const bem_dom_dev &D, const bem_el &el, const bem_node &nd, bool tri, int pt,
                                           double &z, double &e, double &wt, double vR[3], double vW[3]) {
  const int part = pt / (BEM_GHN * BEM_GHN), ij = pt % (BEM_GHN * BEM_GHN);
  const int i = ij / BEM_GHN, j = ij % BEM_GHN;
  z = c_q.xh[i];
  e = c_q.xh[j];
  wt = c_q.wh[i] * c_q.wh[j];
  if (tri) {
    bem_tri_point_ref(part, c_q.xh[i], c_q.xh[j], z, e);
    wt *= bem_tri_wfac(c_q.xh[i], c_q.xh[j]);
    bem_rw_ref(el, z, e, vR, vW);
    for (int d = 0; d < 3; ++d) vR[d] = __dsub_rn(vR[d], nd.rt[d]);
  } else {
    bem_rw(el, z, e, vR, vW);
    for (int d = 0; d < 3; ++d) vR[d] -= nd.rt[d];
  }
}
// point pt of the regular-pair rule (12 x 12, 3 parts of 12 x 12 on a triangle)
__device__ __forceinline__ void reg_point(const bem_el &el, const bem_node &nd, bool tri, int pt, double &z, double &e,
                                          double &wt, double vR[3], double vW[3]) {
  const int part = pt / (BEM_GLN * BEM_GLN), ij = pt % (BEM_GLN * BEM_GLN);
  const int i = ij / BEM_GLN, j = ij % BEM_GLN;
  z = c_q.xl[i];
  e = c_q.xl[j];
  wt = c_q.wl[i] * c_q.wl[j];
  if (tri) {
    bem_tri_point(part, c_q.xl[i], c_q.xl[j], z, e);
    wt *= bem_tri_wfac(c_q.xl[i], c_q.xl[j]);
  }
  bem_rw(el, z, e, vR, vW);
  for (int d = 0; d < 3; ++d) vR[d] -= nd.rt[d];
}

// register cap of the periodic near-singular and self kernels (0: compiler's choice)
#ifndef NP_MAXREG
#define NP_MAXREG 0
#endif
#if NP_MAXREG > 0
#define NP_BOUNDS __maxnreg__(NP_MAXREG)
#else
#define NP_BOUNDS __launch_bounds__(NP_THREADS, 2)  // two blocks (16 warps) per SM: at most 128 registers
#endif
template <int NV>
__device__ __forceinline__ void block_reduce(double (&v)[NV], double *sm /* NV*NP_THREADS */) {
#pragma unroll
  for (int c = 0; c < NV; ++c) {
    double x = v[c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0) sm[c * (NP_THREADS / 32) + (threadIdx.x >> 5)] = x;
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    double x = 0.0;
    for (int w = 0; w < NP_THREADS / 32; ++w) x += sm[threadIdx.x * (NP_THREADS / 32) + w];
    sm[NV * (NP_THREADS / 32) + threadIdx.x] = x;
  }
  __syncthreads();
#pragma unroll
  for (int c = 0; c < NV; ++c) v[c] = sm[NV * (NP_THREADS / 32) + c];
  __syncthreads();
}

template <class BA>
__global__ void NP_BOUNDS k_q0_near(bem_dom_dev D, const __grid_constant__ bem_qp q0, const int *__restrict__ near_s,
                                                        const int *__restrict__ near_n, double *G0,
                                                        double *H0, double *__restrict__ nearF, unsigned *status,
                                                        unsigned long long *terms, const __grid_constant__ BA B) {
  // blocks (p, y) take the node's near pairs y, y + gridDim.y, ...; a batch:
  // block (p, y, b) those of instance b, and instance 0 alone writes the geometric sums
  const int p = blockIdx.x, nn = near_n[p];
  if ((int)blockIdx.y >= nn) return;
  const int bz = bat_is<BA>::on ? (int)blockIdx.z : 0;
  double *__restrict__ G = bat_G(B, bz, G0), *__restrict__ H = bat_H(B, bz, H0);
  if (bz) nearF = nullptr;
  const bem_qp &q = bat_q(B, bz, q0);
  extern __shared__ double2 wts_s[];  // BEM_WT_SMEM bytes of dynamic shared memory
  const double2 *wts = bem_wtab_stage(q, wts_s);
  __syncthreads();
  __shared__ double sm[19 * (NP_THREADS / 32) + 19];
  for (int k = blockIdx.y; k < nn; k += gridDim.y) {
    const int s = near_s[(size_t)p * D.near_cap + k];
    bem_node nd;
    int t, te;
    bem_load_node(D, p, nd, t, te);
    bem_el el;
    const int se = abs(D.sid[s]) - 1;
    bem_load_el(D.cr, D.cw, se, el);
    const bool tri = bem_is_tri(D, se);  // q0_lit_dcoef_v2_cc_GH: 3 parts x 64 x 64
    double v[19];
#pragma unroll
    for (int c = 0; c < 19; ++c) v[c] = 0.0;
    unsigned st = 0;
    unsigned long long nterm = 0, npt = 0;
    const int npts = (tri ? 3 : 1) * BEM_GHN * BEM_GHN;
    // the reference's points (q0_lit_dcoef_v2_cc_GH / q0_bil_dcoef_v2_cc_GH):
    // the geometric F, and G0 unless a point lies on the lattice plane
    bool on_plane = false;
    for (int pt = threadIdx.x; pt < npts; pt += NP_THREADS) {
      double z, e, wt, vR[3], vW[3], N[4];
      near_point(D, el, nd, tri, pt, z, e, wt, vR, vW);
      on_plane |= fabs(vR[2]) < BEM_FAR_PLANE_TOL;
      bem_gval g0;
      bem_g0(q.k, vR, g0);
      bem_Nn(tri, z, e, N);
      acc_gh(v, g0, vW, sqrt(vW[0] * vW[0] + vW[1] * vW[1] + vW[2] * vW[2]) * wt, wt, N);
      double f, fz, fe;
      geomF(vR, vW, nd, f, fz, fe);
      v[16] += wt * f;
      v[17] += wt * fz;
      v[18] += wt * fe;
    }
    // G_qp - G0 on the regular-pair rule (12 x 12 on a quad, 3 parts of 12 x
    // 12 on a triangle), whose points must stay off the lattice plane too
    const int nreg = (tri ? 3 : 1) * BEM_GLN * BEM_GLN;
    for (int pt = threadIdx.x; pt < nreg; pt += NP_THREADS) {
      double z, e, wt, vR[3], vW[3];
      reg_point(el, nd, tri, pt, z, e, wt, vR, vW);
      on_plane |= fabs(vR[2]) < BEM_FAR_PLANE_TOL;
    }
    if (!__syncthreads_or(on_plane)) {
      for (int pt = threadIdx.x; pt < nreg; pt += NP_THREADS) {
        double z, e, wt, vR[3], vW[3], N[4];
        reg_point(el, nd, tri, pt, z, e, wt, vR, vW);
        bem_gval gv, g0;
        const int rc = bem_qpgf(q, vR[0], vR[1], vR[2], gv, wts);
        if (rc < 0) st |= (rc == -12 || rc == -23) ? BEM_ST_RAYLEIGH : BEM_ST_QPGF_LIMIT;
        nterm += rc > 0 ? (unsigned long long)rc : 0ULL;
        ++npt;
        bem_g0(q.k, vR, g0);
        gval_sub(gv, g0);
        bem_Nn(tri, z, e, N);
        acc_gh(v, gv, vW, sqrt(vW[0] * vW[0] + vW[1] * vW[1] + vW[2] * vW[2]) * wt, wt, N);
      }
    } else {
      // a point on the lattice plane: the reference's rule on the full
      // quasi-periodic Green's function (its sums stop on rounding-decided
      // zeros there, which only its own points reproduce)
#pragma unroll
      for (int c = 0; c < 16; ++c) v[c] = 0.0;
      for (int pt = threadIdx.x; pt < npts; pt += NP_THREADS) {
        double z, e, wt, vR[3], vW[3], N[4];
        near_point(D, el, nd, tri, pt, z, e, wt, vR, vW);
        bem_gval gv;
        const int rc = bem_qpgf(q, vR[0], vR[1], vR[2], gv, wts);
        if (rc < 0) st |= (rc == -12 || rc == -23) ? BEM_ST_RAYLEIGH : BEM_ST_QPGF_LIMIT;
        nterm += rc > 0 ? (unsigned long long)rc : 0ULL;
        ++npt;
        bem_Nn(tri, z, e, N);
        acc_gh(v, gv, vW, sqrt(vW[0] * vW[0] + vW[1] * vW[1] + vW[2] * vW[2]) * wt, wt, N);
      }
    }
    count_work(terms + 1, nterm, npt);
    set_status(status, st);
    block_reduce<19>(v, sm);
    if (threadIdx.x < 16) {
      const size_t N = (size_t)D.ne * 4;
      const int c = threadIdx.x;
      double *dst = c < 8 ? G : H;
      const int a = (c & 7) >> 1, part = c & 1;
      dst[2 * ((size_t)p * N + 4 * s + a) + part] = v[c];
    } else if (threadIdx.x < 19 && nearF) {
      nearF[((size_t)p * D.near_cap + k) * 3 + (threadIdx.x - 16)] = v[threadIdx.x] * BEM_I_FP;
    }
    __syncthreads();  // sm is reused by the next pair
  }
}

// ------------------------------------------------------------------ singular (self) integrals
// Polar quadrature around the collocation point (zt,et) of the element itself:
// 4 sub-triangles x (2 x 64) angles x 12 radii (q0_bil_coef_bd, q0_bil_coef.c:246-338,
// and bil_coef_bd, bil_coef.c:244-342).  The angular rule of the reference
// splits each sub-triangle's angle range in two halves with 64 points each.
struct polar_pt { double th, wth; int j; };
__device__ __forceinline__ polar_pt polar_theta(const double th[5], int idx /* 0..511 */) {
  const int j = idx >> 7, h = (idx >> 6) & 1, m = idx & 63;
  const double t0 = th[j], t1 = th[j + 1];
  polar_pt r;
  r.th = h == 0 ? 0.25 * (t1 - t0) * c_q.xh[m] + 0.25 * (t1 + 3.0 * t0) : 0.25 * (t1 - t0) * c_q.xh[m] + 0.25 * (3.0 * t1 + t0);
  r.wth = c_q.wh[m] * 0.25 * (t1 - t0);
  r.j = j;
  return r;
}

// geometric F of the element at parameter point (zt,et) by the polar rule (q0_bil_coef_bd_F,
// q0_bil_dcoef_v2_cc.c:401-454 / bil_sF_theta): returns the un-normalised sum (times bdC/4pi later)
__device__ double polar_F_partial(const bem_el &el, double zt, double et, unsigned &st) {
  double r[5], th[5];
  bem_node_r_th(zt, et, r, th);
  double acc = 0.0;
  for (int idx = threadIdx.x; idx < 512; idx += blockDim.x) {
    const polar_pt tp = polar_theta(th, idx);
    const double rm = bem_rmax(r[tp.j], r[tp.j + 1], th[tp.j], th[tp.j + 1], tp.th);
    if (rm < 0.0) st |= BEM_ST_GEOMETRY;
    double sth, cth;
    sincos(tp.th, &sth, &cth);
    double inner = 0.0;
    for (int ir = 0; ir < BEM_GLN; ++ir) {
      const double rr = 0.5 * rm * (c_q.xl[ir] + 1.0);
      double K[3];
      bem_K(el, rr, cth, sth, zt, et, K);
      const double aK = sqrt(K[0] * K[0] + K[1] * K[1] + K[2] * K[2]);
      inner += c_q.wl[ir] / (aK * aK * aK) * cth * sth;
    }
    acc += tp.wth * 0.5 * rm * inner;
  }
  return acc;
}

__device__ __forceinline__ double bem_bdC(const bem_el &el) {
  return el.cr[0][1] * el.cw[0][2] + el.cr[1][1] * el.cw[1][2] + el.cr[2][1] * el.cw[2][2];
}

// periodic self pair: one block per collocation node p
// point pt of the polar rule around the node (zt, et) on its own quad: (z, e),
// the weight with the polar Jacobian, R = rr K from the node, W; false when
// the rule's radius comes out negative (bad geometry)
__device__ __forceinline__ bool self_point(const bem_el &el, const double th[5], const double r[5], double zt, double et,
                                           int pt, double &z, double &e, double &wr, double vR[3], double vW[3]) {
  const int idx = pt / BEM_GLN, ir = pt % BEM_GLN;
  const polar_pt tp = polar_theta(th, idx);
  const double rm = bem_rmax(r[tp.j], r[tp.j + 1], th[tp.j], th[tp.j + 1], tp.th);
  double sth, cth;
  sincos(tp.th, &sth, &cth);
  const double rr = 0.5 * rm * (c_q.xl[ir] + 1.0);
  wr = tp.wth * 0.5 * rm * c_q.wl[ir] * rr;
  z = rr * cth + zt;
  e = rr * sth + et;
  double K[3];
  bem_K(el, rr, cth, sth, zt, et, K);
  for (int d = 0; d < 3; ++d) {
    vR[d] = rr * K[d];
    vW[d] = el.cw[d][0] + el.cw[d][1] * z + el.cw[d][2] * e;
  }
  return rm >= 0.0;
}

template <class BA>
__global__ void NP_BOUNDS k_q0_self(bem_dom_dev D, const __grid_constant__ bem_qp q0, double *G0,
                                                        double *H0, double *__restrict__ selfF,
                                                        unsigned *status, unsigned long long *terms,
                                                        const __grid_constant__ BA B) {
  const int p = blockIdx.x;
  const int t = p >> 2, tn = p & 3;
  const int te = abs(D.sid[t]) - 1;
  if (bem_is_tri(D, te)) return;  // k_q0_self_tri
  // a batch: block (p, 0, b) integrates instance b; instance 0 alone writes selfF
  const int bz = bat_is<BA>::on ? (int)blockIdx.z : 0;
  double *__restrict__ G = bat_G(B, bz, G0), *__restrict__ H = bat_H(B, bz, H0);
  if (bz) selfF = nullptr;
  const bem_qp &q = bat_q(B, bz, q0);
  extern __shared__ double2 wts_s[];  // BEM_WT_SMEM bytes of dynamic shared memory
  const double2 *wts = bem_wtab_stage(q, wts_s);
  __syncthreads();
  bem_el el;
  bem_load_el(D.cr, D.cw, te, el);
  const double zt = c_q.zt[tn], et = c_q.et[tn];
  double r[5], th[5];
  bem_node_r_th(zt, et, r, th);
  unsigned long long nterm = 0, npt = 0;
  double v[19];
#pragma unroll
  for (int c = 0; c < 19; ++c) v[c] = 0.0;
  unsigned st = 0;
  // the node on its own element
  bem_node nd;
  {
    double w0[3];
    bem_rw(el, zt, et, nd.rt, w0);
  }
  // the polar rule around the node (q0_bil_coef_bd, q0_bil_coef.c:246-338):
  // G0 at every point, unless a point lies on the lattice plane
  bool on_plane = false;
  for (int pt = threadIdx.x; pt < 512 * BEM_GLN; pt += NP_THREADS) {
    double z, e, wr, vR[3], vW[3], N[4];
    if (!self_point(el, th, r, zt, et, pt, z, e, wr, vR, vW)) st |= BEM_ST_GEOMETRY;
    on_plane |= fabs(vR[2]) < BEM_FAR_PLANE_TOL;
    bem_gval g0;
    bem_g0(q.k, vR, g0);
    bem_Nn4(z, e, N);
    acc_gh(v, g0, vW, sqrt(vW[0] * vW[0] + vW[1] * vW[1] + vW[2] * vW[2]) * wr, wr, N);
  }
  // G_qp - G0 on the 12 x 12 Gauss rule over the element
  for (int pt = threadIdx.x; pt < BEM_GLN * BEM_GLN; pt += NP_THREADS) {
    double z, e, wt, vR[3], vW[3];
    reg_point(el, nd, false, pt, z, e, wt, vR, vW);
    on_plane |= fabs(vR[2]) < BEM_FAR_PLANE_TOL;
  }
  if (!__syncthreads_or(on_plane)) {
    for (int pt = threadIdx.x; pt < BEM_GLN * BEM_GLN; pt += NP_THREADS) {
      double z, e, wt, vR[3], vW[3], N[4];
      reg_point(el, nd, false, pt, z, e, wt, vR, vW);
      bem_gval gv, g0;
      const int rc = bem_qpgf(q, vR[0], vR[1], vR[2], gv, wts);
      if (rc < 0) st |= (rc == -12 || rc == -23) ? BEM_ST_RAYLEIGH : BEM_ST_QPGF_LIMIT;
      nterm += rc > 0 ? (unsigned long long)rc : 0ULL;
      ++npt;
      bem_g0(q.k, vR, g0);
      gval_sub(gv, g0);
      bem_Nn4(z, e, N);
      acc_gh(v, gv, vW, sqrt(vW[0] * vW[0] + vW[1] * vW[1] + vW[2] * vW[2]) * wt, wt, N);
    }
  } else {
    // a point on the lattice plane (a plane element, or a curved one whose
    // points meet the node's height): the reference's polar rule on the full
    // quasi-periodic Green's function
#pragma unroll
    for (int c = 0; c < 16; ++c) v[c] = 0.0;
    for (int pt = threadIdx.x; pt < 512 * BEM_GLN; pt += NP_THREADS) {
      double z, e, wr, vR[3], vW[3], N[4];
      self_point(el, th, r, zt, et, pt, z, e, wr, vR, vW);
      bem_gval gv;
      const int rc = bem_qpgf(q, vR[0], vR[1], vR[2], gv, wts);
      if (rc < 0) st |= (rc == -12 || rc == -23) ? BEM_ST_RAYLEIGH : BEM_ST_QPGF_LIMIT;
      nterm += rc > 0 ? (unsigned long long)rc : 0ULL;
      ++npt;
      bem_Nn4(z, e, N);
      acc_gh(v, gv, vW, sqrt(vW[0] * vW[0] + vW[1] * vW[1] + vW[2] * vW[2]) * wr, wr, N);
    }
  }
  count_work(terms + 2, nterm, npt);
  // F at the node and at (zt+-h, et), (zt, et+-h) for the central differences
  // (q0_bil_dcoef_bd_tz0_cc_DV / _te0_, q0_bil_dcoef_v2_cc.c:336-399)
  const bool plane = D.plane[te] != 0;
  double f[5] = {0, 0, 0, 0, 0};
  if (!plane) {
    f[0] = polar_F_partial(el, zt, et, st);
    f[1] = polar_F_partial(el, zt + BEM_CDFH, et, st);
    f[2] = polar_F_partial(el, zt - BEM_CDFH, et, st);
    f[3] = polar_F_partial(el, zt, et + BEM_CDFH, st);
    f[4] = polar_F_partial(el, zt, et - BEM_CDFH, st);
  }
  set_status(status, st);
  __shared__ double sm[21 * (NP_THREADS / 32) + 21];
  double all[21];
#pragma unroll
  for (int c = 0; c < 16; ++c) all[c] = v[c];
#pragma unroll
  for (int c = 0; c < 5; ++c) all[16 + c] = f[c];
  block_reduce<21>(all, sm);
  if (threadIdx.x < 16) {
    const size_t N = (size_t)D.ne * 4;
    const int c = threadIdx.x;
    double *dst = c < 8 ? G : H;
    const int a = (c & 7) >> 1, part = c & 1;
    dst[2 * ((size_t)p * N + 4 * t + a) + part] = all[c];
  } else if (threadIdx.x == 16) {
    const double bdC = bem_bdC(el);
    const double F0 = plane ? 0.0 : all[16] * BEM_I_FP * bdC;
    const double Fzp = all[17] * BEM_I_FP * bdC, Fzm = all[18] * BEM_I_FP * bdC;
    const double Fep = all[19] * BEM_I_FP * bdC, Fem = all[20] * BEM_I_FP * bdC;
    double Tz[3], Te[3];
    for (int d = 0; d < 3; ++d) {
      Tz[d] = el.cr[d][1] + el.cr[d][3] * et;
      Te[d] = el.cr[d][2] + el.cr[d][3] * zt;
    }
    const double iTz = 1.0 / sqrt(dot3(Tz, Tz)), iTe = 1.0 / sqrt(dot3(Te, Te));
    if (selfF) {
      selfF[3 * p + 0] = F0;
      selfF[3 * p + 1] = plane ? 0.0 : iTz * (Fzp - Fzm) / (2.0 * BEM_CDFH);
      selfF[3 * p + 2] = plane ? 0.0 : iTe * (Fep - Fem) / (2.0 * BEM_CDFH);
    }
  }
}

// ------------------------------------------------------------------ free-space (interior) pairs
// Integrand of bil_dcoef_v2_GL / _GH (bil_dcoef_v2.c:141-325) at one point,
// accumulated into 24 complex sums + 3 geometric ones.
struct fs_acc { double g[8], h[8], gz[8], ge[8], hz[8], he[8], f, fz, fe; };

__device__ __forceinline__ void fs_zero(fs_acc &a) {
#pragma unroll
  for (int c = 0; c < 8; ++c) { a.g[c] = a.h[c] = a.gz[c] = a.ge[c] = a.hz[c] = a.he[c] = 0.0; }
  a.f = a.fz = a.fe = 0.0;
}

__device__ __forceinline__ void fs_point(const bem_el &el, const bem_node &nd, double k, double z, double e, double wt, fs_acc &a,
                                         bool tri = false) {
  double vR[3], vW[3];
  bem_rw(el, z, e, vR, vW);
  for (int d = 0; d < 3; ++d) vR[d] -= nd.rt[d];
  const double aR = sqrt(vR[0] * vR[0] + vR[1] * vR[1] + vR[2] * vR[2]);
  const double iR = 1.0 / aR;
  const double aW = sqrt(vW[0] * vW[0] + vW[1] * vW[1] + vW[2] * vW[2]);
  const cplx ce = cexpi(k * aR);
  const cplx cb = cmk(-1.0, k * aR);  // i k R - 1
  const double rdW = dot3(vR, vW) * iR;
  const double tD = rdW * iR * iR;
  const double rdz = dot3(vR, nd.vz) * iR, rde = dot3(vR, nd.vt) * iR;
  const double Wdz = dot3(vW, nd.vz), Wde = dot3(vW, nd.vt);
  const double i3 = iR * iR * iR;
  double N[4];
  bem_Nn(tri, z, e, N);
  const cplx cbce = cmul(cb, ce);
  const cplx g = cscale(ce, iR * aW * wt);                       // e^{ikR}/R |W|
  const cplx h = cscale(cbce, tD * wt);                          // (ikR-1) e^{ikR} (R.W)/R^3
  const cplx gz = cscale(cbce, iR * iR * rdz * aW * wt);         // dG/dv before the -1/4pi
  const cplx ge = cscale(cbce, iR * iR * rde * aW * wt);
  const cplx kk3 = cmk(k * k * aR * aR + 3.0 * cb.re, 3.0 * cb.im);  // k^2 R^2 + 3 (ikR-1)
  const cplx hz = cscale(cmul(ce, csub(cscale(kk3, rdz * rdW), cscale(cb, Wdz))), i3 * wt);
  const cplx he = cscale(cmul(ce, csub(cscale(kk3, rde * rdW), cscale(cb, Wde))), i3 * wt);
#pragma unroll
  for (int n = 0; n < 4; ++n) {
    a.g[2 * n] += g.re * N[n];  a.g[2 * n + 1] += g.im * N[n];
    a.h[2 * n] += h.re * N[n];  a.h[2 * n + 1] += h.im * N[n];
    a.gz[2 * n] += gz.re * N[n]; a.gz[2 * n + 1] += gz.im * N[n];
    a.ge[2 * n] += ge.re * N[n]; a.ge[2 * n + 1] += ge.im * N[n];
    a.hz[2 * n] += hz.re * N[n]; a.hz[2 * n + 1] += hz.im * N[n];
    a.he[2 * n] += he.re * N[n]; a.he[2 * n + 1] += he.im * N[n];
  }
  a.f += wt * tD;
  a.fz += wt * i3 * (3.0 * rdz * rdW - Wdz);
  a.fe += wt * i3 * (3.0 * rde * rdW - Wde);
}

// write one pair's 24 complex coefficients with the reference's scale factors
// (1/4pi, -1/4pi for dG) and the sign flip for negative element ids.  G, H
// (and dG, dH) may be null: a pass that only recomputes the derivative rows
// writes dG, dH alone, row 2 (p - p0) of a block of rows starting at p0.
__device__ __forceinline__ void fs_store(const bem_dom_dev &D, int p, int s, const fs_acc &a, double *G, double *H,
                                         double *dG, double *dH, int p0) {
  const size_t N = (size_t)D.ne * 4;
  const double sg = D.sid[s] < 0 ? -1.0 : 1.0;
  const double c = BEM_I_FP;
  if (G) {
    double2 *g2 = reinterpret_cast<double2 *>(G + 2 * ((size_t)p * N + 4 * s));
    double2 *h2 = reinterpret_cast<double2 *>(H + 2 * ((size_t)p * N + 4 * s));
#pragma unroll
    for (int n = 0; n < 4; ++n) {
      g2[n] = make_double2(a.g[2 * n] * c, a.g[2 * n + 1] * c);
      h2[n] = make_double2(sg * a.h[2 * n] * c, sg * a.h[2 * n + 1] * c);
    }
  }
  if (dG) {
    const size_t r = 2 * (size_t)(p - p0);
    double2 *gz = reinterpret_cast<double2 *>(dG + 2 * (r * N + 4 * s));
    double2 *ge = reinterpret_cast<double2 *>(dG + 2 * ((r + 1) * N + 4 * s));
    double2 *hz = reinterpret_cast<double2 *>(dH + 2 * (r * N + 4 * s));
    double2 *he = reinterpret_cast<double2 *>(dH + 2 * ((r + 1) * N + 4 * s));
#pragma unroll
    for (int n = 0; n < 4; ++n) {
      gz[n] = make_double2(-a.gz[2 * n] * c, -a.gz[2 * n + 1] * c);
      ge[n] = make_double2(-a.ge[2 * n] * c, -a.ge[2 * n + 1] * c);
      hz[n] = make_double2(sg * a.hz[2 * n] * c, sg * a.hz[2 * n + 1] * c);
      he[n] = make_double2(sg * a.he[2 * n] * c, sg * a.he[2 * n + 1] * c);
    }
  }
}

// one thread per (p, s) pair, 12x12 points; rows p0 .. p0 + np - 1
__global__ void __launch_bounds__(128) k_fs_regular(bem_dom_dev D, double k, const uint8_t *__restrict__ flag,
                                                    double *__restrict__ G, double *__restrict__ H,
                                                    double *__restrict__ dG, double *__restrict__ dH, int p0, int np) {
  const long long pair = (long long)p0 * D.ne + (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long total = (long long)(p0 + np) * D.ne;
  if (pair >= total) return;
  const int p = (int)(pair / D.ne), s = (int)(pair % D.ne);
  if (flag[pair] != 0 || bem_pad_row(D, p)) return;
  bem_node nd;
  int t, te;
  bem_load_node(D, p, nd, t, te);
  bem_el el;
  const int se = abs(D.sid[s]) - 1;
  bem_load_el(D.cr, D.cw, se, el);
  fs_acc a;
  fs_zero(a);
  if (bem_is_tri(D, se)) {
    // lit_dcoef_v2_GL (lit_dcoef_v2.c:185-270): 3 parts x 12 x 12
    for (int part = 0; part < 3; ++part)
      for (int i = 0; i < BEM_GLN; ++i)
        for (int j = 0; j < BEM_GLN; ++j) {
          double z, e;
          bem_tri_point(part, c_q.xl[i], c_q.xl[j], z, e);
          fs_point(el, nd, k, z, e, c_q.wl[i] * c_q.wl[j] * bem_tri_wfac(c_q.xl[i], c_q.xl[j]), a, true);
        }
  } else {
    for (int i = 0; i < BEM_GLN; ++i)
      for (int j = 0; j < BEM_GLN; ++j) fs_point(el, nd, k, c_q.xl[i], c_q.xl[j], c_q.wl[i] * c_q.wl[j], a);
  }
  fs_store(D, p, s, a, G, H, dG, dH, p0);
}

// one block per flagged pair, 64x64 points
__global__ void __launch_bounds__(NP_THREADS) k_fs_near(bem_dom_dev D, double k, const int *__restrict__ near_s,
                                                        const int *__restrict__ near_n, double *__restrict__ G,
                                                        double *__restrict__ H, double *__restrict__ dG,
                                                        double *__restrict__ dH, double *__restrict__ nearF, int p0) {
  // blocks (p, y) take the node's near pairs y, y + gridDim.y, ...
  const int p = p0 + blockIdx.x, nn = near_n[p];
  __shared__ double sm[51 * (NP_THREADS / 32) + 51];
  for (int kk = blockIdx.y; kk < nn; kk += gridDim.y) {
    const int s = near_s[(size_t)p * D.near_cap + kk];
    bem_node nd;
    int t, te;
    bem_load_node(D, p, nd, t, te);
    bem_el el;
    const int se = abs(D.sid[s]) - 1;
    bem_load_el(D.cr, D.cw, se, el);
    const bool tri = bem_is_tri(D, se);  // lit_dcoef_v2_GH: 3 parts x 64 x 64
    fs_acc a;
    fs_zero(a);
    for (int pt = threadIdx.x; pt < (tri ? 3 : 1) * BEM_GHN * BEM_GHN; pt += NP_THREADS) {
      const int part = pt / (BEM_GHN * BEM_GHN), ij = pt % (BEM_GHN * BEM_GHN);
      const int i = ij / BEM_GHN, j = ij % BEM_GHN;
      if (tri) {
        double z, e;
        bem_tri_point(part, c_q.xh[i], c_q.xh[j], z, e);
        fs_point(el, nd, k, z, e, c_q.wh[i] * c_q.wh[j] * bem_tri_wfac(c_q.xh[i], c_q.xh[j]), a, true);
      } else {
        fs_point(el, nd, k, c_q.xh[i], c_q.xh[j], c_q.wh[i] * c_q.wh[j], a);
      }
    }
    double *av = reinterpret_cast<double *>(&a);
    double v[51];
#pragma unroll
    for (int c = 0; c < 51; ++c) v[c] = av[c];
    block_reduce<51>(v, sm);
    if (threadIdx.x == 0) {
#pragma unroll
      for (int c = 0; c < 51; ++c) av[c] = v[c];
      fs_store(D, p, s, a, G, H, dG, dH, p0);
      if (G) {
        const double sg = D.sid[s] < 0 ? -1.0 : 1.0;
        double *nf = nearF + ((size_t)p * D.near_cap + kk) * 3;
        nf[0] = sg * a.f * BEM_I_FP;
        nf[1] = sg * a.fz * BEM_I_FP;
        nf[2] = sg * a.fe * BEM_I_FP;
      }
    }
    __syncthreads();  // sm is reused by the next pair
  }
}

// free-space self pair with the principal-value derivative integrals
// (bil_dcoef_bd_vt2_PV -> bil_coef_bd, bil_dcoef_bd_tz0_PV, bil_dcoef_bd_te0_PV;
//  bil_coef.c:244-342, bil_dcoef.c:369-740, integrands bil_dcoef.c:916-1630).
// Accumulators (complex unless noted), per interpolation function n:
//   G, H, and F (real)                       over the 12-radius polar rule
//   dG (shared rule, vt differs), dHz, dHe   over D-bar-eps (64 radii from DEPS to rm),
//   D-eps (4 x 64 angles, 12 radii) and the PV pair (2 x 64 angles, 12 radii)
//   dFz, dFe (real)                           over D-bar-eps and the PV pair
struct self_acc {
  double g[8], h[8];
  double dgz[8], dge[8], dhz[8], dhe[8];
  double f, fz, fe;
};

#ifndef FS_SELF_MINB
// two blocks (16 warps) per SM: 128 registers with 520 B of spills, 1.1 % faster
// per 216-quad solve than one block at 244 registers (it shares the SMs with
// the periodic domain's kernels)
#define FS_SELF_MINB 2
#endif
__global__ void __launch_bounds__(NP_THREADS, FS_SELF_MINB) k_fs_self(bem_dom_dev D, double k, double *__restrict__ G,
                                                        double *__restrict__ H, double *__restrict__ dG,
                                                        double *__restrict__ dH, double *__restrict__ selfF,
                                                        unsigned *status, int p0) {
  const int p = p0 + blockIdx.x;
  const int t = p >> 2, tn = p & 3;
  const int te = abs(D.sid[t]) - 1;
  if (bem_is_tri(D, te)) return;  // k_fs_self_tri
  bem_el el;
  bem_load_el(D.cr, D.cw, te, el);
  const double zt = c_q.zt[tn], et = c_q.et[tn];
  double r[5], th[5];
  bem_node_r_th(zt, et, r, th);
  double vz[3], ve[3];  // T_zeta, T_eta at (zt,et) (not normalised), bil_t_zeta / bil_t_eta
  for (int d = 0; d < 3; ++d) {
    vz[d] = el.cr[d][1] + el.cr[d][3] * et;
    ve[d] = el.cr[d][2] + el.cr[d][3] * zt;
  }
  self_acc A;
  double *Av = reinterpret_cast<double *>(&A);
#pragma unroll
  for (int c = 0; c < 51; ++c) Av[c] = 0.0;
  unsigned st = 0;
  // (1) G, H, F over the polar rule with 12 radii from 0 to rm
  for (int pt = threadIdx.x; pt < 512 * BEM_GLN; pt += NP_THREADS) {
    const int idx = pt / BEM_GLN, ir = pt % BEM_GLN;
    const polar_pt tp = polar_theta(th, idx);
    const double rm = bem_rmax(r[tp.j], r[tp.j + 1], th[tp.j], th[tp.j + 1], tp.th);
    if (rm < 0.0) st |= BEM_ST_GEOMETRY;
    double sth, cth;
    sincos(tp.th, &sth, &cth);
    const double rr = 0.5 * rm * (c_q.xl[ir] + 1.0);
    const double w = tp.wth * 0.5 * rm * c_q.wl[ir];
    const double z = rr * cth + zt, e = rr * sth + et;
    double K[3], W[3];
    bem_K(el, rr, cth, sth, zt, et, K);
    for (int d = 0; d < 3; ++d) W[d] = el.cw[d][0] + el.cw[d][1] * z + el.cw[d][2] * e;
    const double aK = sqrt(dot3(K, K)), aW = sqrt(dot3(W, W));
    const double kR = k * aK * rr;
    const cplx ce = cexpi(kR);
    const cplx g = cscale(ce, w * aW / aK);                                          // bil_sG_r
    const cplx h = cscale(cmul(cmk(-1.0, kR), ce), w * cth * sth / (aK * aK * aK));  // bil_sH_r
    double N[4];
    bem_Nn4(z, e, N);
#pragma unroll
    for (int n = 0; n < 4; ++n) {
      A.g[2 * n] += g.re * N[n]; A.g[2 * n + 1] += g.im * N[n];
      A.h[2 * n] += h.re * N[n]; A.h[2 * n + 1] += h.im * N[n];
    }
    A.f += w * cth * sth / (aK * aK * aK);                                           // bil_sF_r
  }
  // (2) D-bar-eps: 512 angles x 64 radii from DEPS to rm
  for (int pt = threadIdx.x; pt < 512 * BEM_GHN; pt += NP_THREADS) {
    const int idx = pt / BEM_GHN, ir = pt % BEM_GHN;
    const polar_pt tp = polar_theta(th, idx);
    const double rm = bem_rmax(r[tp.j], r[tp.j + 1], th[tp.j], th[tp.j + 1], tp.th);
    if (rm < 0.0) st |= BEM_ST_GEOMETRY;
    double sth, cth;
    sincos(tp.th, &sth, &cth);
    const double rr = 0.5 * (rm - BEM_DEPS) * c_q.xh[ir] + 0.5 * (rm + BEM_DEPS);
    const double w = tp.wth * 0.5 * (rm - BEM_DEPS) * c_q.wh[ir];
    const double z = rr * cth + zt, e = rr * sth + et;
    double K[3], W[3];
    bem_K(el, rr, cth, sth, zt, et, K);
    for (int d = 0; d < 3; ++d) W[d] = el.cw[d][0] + el.cw[d][1] * z + el.cw[d][2] * e;
    const double aK = sqrt(dot3(K, K)), aW = sqrt(dot3(W, W));
    const double iK = 1.0 / aK;
    const double kR = k * aK * rr;
    const cplx ce = cexpi(kR);
    const cplx cb = cmk(-1.0, kR);
    const cplx cbce = cmul(cb, ce);
    const double KTz = dot3(K, vz), KTe = dot3(K, ve);
    // bil_sdG_Db_r: cb ce / aK^2 / r * (K.vt/aK) * N * aW
    const double gfac = w * iK * iK / rr * aW * iK;
    const cplx dgz = cscale(cbce, gfac * KTz), dge = cscale(cbce, gfac * KTe);
    // bil_sdHz_Db_r: ce/(r aK^5) ((kR^2 + 3cb) K.vt cth - cb aK^2), then * sth (outer)
    // bil_sdHe_Db_r: same with sth inside and cth outer
    const double i5 = 1.0 / (rr * aK * aK * aK * aK * aK);
    const cplx kk3 = cmk(kR * kR + 3.0 * cb.re, 3.0 * cb.im);
    const cplx hz = cscale(cmul(ce, csub(cscale(kk3, KTz * cth), cscale(cb, aK * aK))), w * i5 * sth);
    const cplx he = cscale(cmul(ce, csub(cscale(kk3, KTe * sth), cscale(cb, aK * aK))), w * i5 * cth);
    double N[4];
    bem_Nn4(z, e, N);
#pragma unroll
    for (int n = 0; n < 4; ++n) {
      A.dgz[2 * n] += dgz.re * N[n]; A.dgz[2 * n + 1] += dgz.im * N[n];
      A.dge[2 * n] += dge.re * N[n]; A.dge[2 * n + 1] += dge.im * N[n];
      A.dhz[2 * n] += hz.re * N[n];  A.dhz[2 * n + 1] += hz.im * N[n];
      A.dhe[2 * n] += he.re * N[n];  A.dhe[2 * n + 1] += he.im * N[n];
    }
    A.fz += w * i5 * (3.0 * KTz * cth - aK * aK) * sth;   // bil_sdFz_Db_r
    A.fe += w * i5 * (3.0 * KTe * sth - aK * aK) * cth;   // bil_sdFe_Db_r
  }
  // (3) D-eps: 4 x 64 angles over [0, 2 pi), 12 radii from 0 to DEPS
  for (int pt = threadIdx.x; pt < 256 * BEM_GLN; pt += NP_THREADS) {
    const int idx = pt / BEM_GLN, ir = pt % BEM_GLN;
    const int qd = idx >> 6, m = idx & 63;
    const double tht = 0.25 * CUDART_PI * c_q.xh[m] + (-0.75 + 0.5 * qd) * CUDART_PI;
    const double wth = 0.25 * CUDART_PI * c_q.wh[m];
    double sth, cth;
    sincos(tht, &sth, &cth);
    const double rr = 0.5 * BEM_DEPS * (c_q.xl[ir] + 1.0);
    const double w = wth * 0.5 * BEM_DEPS * c_q.wl[ir];
    const double z = rr * cth + zt, e = rr * sth + et;
    double K[3], W[3];
    bem_K(el, rr, cth, sth, zt, et, K);
    for (int d = 0; d < 3; ++d) W[d] = el.cw[d][0] + el.cw[d][1] * z + el.cw[d][2] * e;
    const double aK = sqrt(dot3(K, K)), aW = sqrt(dot3(W, W));
    const double iK = 1.0 / aK;
    const double kR = k * aK * rr;
    double skr, ckr;
    sincos(kR, &skr, &ckr);
    const cplx ce = cmk(ckr, skr);
    const double KTz = dot3(K, vz), KTe = dot3(K, ve);
    // bil_sdG_De_r: (cb sin kR + kR cos kR)/aK^2/r * (K.vt/aK) aW N, times i (outer)
    const cplx cbsk = cmk(-skr + kR * ckr, kR * skr);
    const double gfac = w * iK * iK / rr * aW * iK;
    const cplx dgz = cmul(cmk(0.0, 1.0), cscale(cbsk, gfac * KTz));
    const cplx dge = cmul(cmk(0.0, 1.0), cscale(cbsk, gfac * KTe));
    // bil_sdHz_De0_r: ce/aK^4 ((k kR + 3 i k) K.vt cth - i k aK^2);  _De1_r: sin(kR)/(aK^5 r)(3 K.vt cth - aK^2)
    // theta function: sth * (De0 - i De1)
    const double i4 = 1.0 / (aK * aK * aK * aK);
    const double i5 = i4 / (aK * rr);
    const cplx h0z = cmul(ce, cmk(k * kR * KTz * cth, 3.0 * k * KTz * cth - k * aK * aK));
    const cplx h0e = cmul(ce, cmk(k * kR * KTe * sth, 3.0 * k * KTe * sth - k * aK * aK));
    const double h1z = skr * i5 * (3.0 * KTz * cth - aK * aK);
    const double h1e = skr * i5 * (3.0 * KTe * sth - aK * aK);
    const cplx hz = cscale(cmk(h0z.re * i4, h0z.im * i4 - h1z), w * sth);
    const cplx he = cscale(cmk(h0e.re * i4, h0e.im * i4 - h1e), w * cth);
    double N[4];
    bem_Nn4(z, e, N);
#pragma unroll
    for (int n = 0; n < 4; ++n) {
      A.dgz[2 * n] += dgz.re * N[n]; A.dgz[2 * n + 1] += dgz.im * N[n];
      A.dge[2 * n] += dge.re * N[n]; A.dge[2 * n + 1] += dge.im * N[n];
      A.dhz[2 * n] += hz.re * N[n];  A.dhz[2 * n + 1] += hz.im * N[n];
      A.dhe[2 * n] += he.re * N[n];  A.dhe[2 * n + 1] += he.im * N[n];
    }
  }
  // (4) PV pair: 2 x 64 angles over [0, pi), 12 radii, symmetric points +-r (subtracted)
  for (int pt = threadIdx.x; pt < 128 * BEM_GLN; pt += NP_THREADS) {
    const int idx = pt / BEM_GLN, ir = pt % BEM_GLN;
    const int hh = idx >> 6, m = idx & 63;
    const double tht = 0.25 * CUDART_PI * c_q.xh[m] + (0.25 + 0.5 * hh) * CUDART_PI;
    const double wth = 0.25 * CUDART_PI * c_q.wh[m];
    double sth, cth;
    sincos(tht, &sth, &cth);
    const double rr = 0.5 * BEM_DEPS * (c_q.xl[ir] + 1.0);
    const double w = wth * 0.5 * BEM_DEPS * c_q.wl[ir] / rr;
    double Np[4], Nm[4], Kp[3], Km[3], Wp[3], Wm[3];
    const double zp = rr * cth + zt, ep = rr * sth + et, zm = -rr * cth + zt, em = -rr * sth + et;
    bem_K(el, rr, cth, sth, zt, et, Kp);
    bem_K(el, -rr, cth, sth, zt, et, Km);
    for (int d = 0; d < 3; ++d) {
      Wp[d] = el.cw[d][0] + el.cw[d][1] * zp + el.cw[d][2] * ep;
      Wm[d] = el.cw[d][0] + el.cw[d][1] * zm + el.cw[d][2] * em;
    }
    bem_Nn4(zp, ep, Np);
    bem_Nn4(zm, em, Nm);
    const double aKp = sqrt(dot3(Kp, Kp)), aKm = sqrt(dot3(Km, Km));
    const double aWp = sqrt(dot3(Wp, Wp)), aWm = sqrt(dot3(Wm, Wm));
    const double ccp = cos(k * aKp * rr), ccm = cos(-k * aKm * rr);
    const double KpTz = dot3(Kp, vz), KmTz = dot3(Km, vz), KpTe = dot3(Kp, ve), KmTe = dot3(Km, ve);
    // bil_sdG_DP_r: ccp/aKp^2 (Kp.vt/aKp) N(p) aWp - (same with m)
    const double gzp = ccp / (aKp * aKp) * (KpTz / aKp) * aWp, gzm = ccm / (aKm * aKm) * (KmTz / aKm) * aWm;
    const double gep = ccp / (aKp * aKp) * (KpTe / aKp) * aWp, gem = ccm / (aKm * aKm) * (KmTe / aKm) * aWm;
    // bil_sdHz_DP_r: ccp/aKp^5 (3 Kp.vt cth - aKp^2) N(p) - (m); outer sth
    const double ip5 = 1.0 / (aKp * aKp * aKp * aKp * aKp), im5 = 1.0 / (aKm * aKm * aKm * aKm * aKm);
    const double hzp = ccp * ip5 * (3.0 * KpTz * cth - aKp * aKp), hzm = ccm * im5 * (3.0 * KmTz * cth - aKm * aKm);
    const double hep = ccp * ip5 * (3.0 * KpTe * sth - aKp * aKp), hem = ccm * im5 * (3.0 * KmTe * sth - aKm * aKm);
#pragma unroll
    for (int n = 0; n < 4; ++n) {
      // subtracted from dG and dH (the reference's "dCC[i] -= tC"), real-valued
      A.dgz[2 * n] -= w * (gzp * Np[n] - gzm * Nm[n]);
      A.dge[2 * n] -= w * (gep * Np[n] - gem * Nm[n]);
      A.dhz[2 * n] -= w * sth * (hzp * Np[n] - hzm * Nm[n]);
      A.dhe[2 * n] -= w * cth * (hep * Np[n] - hem * Nm[n]);
    }
    // bil_sdFz_DP_r / _Fe_: added
    A.fz += w * sth * (ip5 * (3.0 * KpTz * cth - aKp * aKp) - im5 * (3.0 * KmTz * cth - aKm * aKm));
    A.fe += w * cth * (ip5 * (3.0 * KpTe * sth - aKp * aKp) - im5 * (3.0 * KmTe * sth - aKm * aKm));
  }
  set_status(status, st);
  __shared__ double sm[51 * (NP_THREADS / 32) + 51];
  double v[51];
#pragma unroll
  for (int c = 0; c < 51; ++c) v[c] = Av[c];
  block_reduce<51>(v, sm);
  if (threadIdx.x == 0) {
    const size_t N = (size_t)D.ne * 4;
    const double sg = D.sid[t] < 0 ? -1.0 : 1.0;
    const bool plane = D.plane[te] != 0;
    const double bdC = bem_bdC(el);
    const double iTz = 1.0 / sqrt(dot3(vz, vz)), iTe = 1.0 / sqrt(dot3(ve, ve));
    const double c = BEM_I_FP;
    if (G) {
      double2 *g2 = reinterpret_cast<double2 *>(G + 2 * ((size_t)p * N + 4 * t));
      double2 *h2 = reinterpret_cast<double2 *>(H + 2 * ((size_t)p * N + 4 * t));
      for (int n = 0; n < 4; ++n) {
        g2[n] = make_double2(v[2 * n] * c, v[2 * n + 1] * c);
        const double hs = plane ? 0.0 : sg * bdC * c;
        h2[n] = make_double2(v[8 + 2 * n] * hs, v[8 + 2 * n + 1] * hs);
      }
      selfF[3 * p + 0] = plane ? 0.0 : sg * v[48] * bdC * c;
      selfF[3 * p + 1] = plane ? 0.0 : sg * v[49] * bdC * c * iTz;
      selfF[3 * p + 2] = plane ? 0.0 : sg * v[50] * bdC * c * iTe;
    }
    if (dG) {
      const size_t r = 2 * (size_t)(p - p0);
      double2 *gz = reinterpret_cast<double2 *>(dG + 2 * (r * N + 4 * t));
      double2 *ge = reinterpret_cast<double2 *>(dG + 2 * ((r + 1) * N + 4 * t));
      double2 *hz = reinterpret_cast<double2 *>(dH + 2 * (r * N + 4 * t));
      double2 *he = reinterpret_cast<double2 *>(dH + 2 * ((r + 1) * N + 4 * t));
      for (int n = 0; n < 4; ++n) {
        // dG: times -1/4pi/|T|; not affected by the element orientation
        gz[n] = make_double2(-c * iTz * v[16 + 2 * n], -c * iTz * v[16 + 2 * n + 1]);
        ge[n] = make_double2(-c * iTe * v[24 + 2 * n], -c * iTe * v[24 + 2 * n + 1]);
        const double hzs = plane ? 0.0 : sg * bdC * c * iTz, hes = plane ? 0.0 : sg * bdC * c * iTe;
        hz[n] = make_double2(v[32 + 2 * n] * hzs, v[32 + 2 * n + 1] * hzs);
        he[n] = make_double2(v[40 + 2 * n] * hes, v[40 + 2 * n + 1] * hes);
      }
    }
  }
}

// ------------------------------------------------------------------ triangle self pairs
// Periodic: q0_lit_coef_bd (q0_lit_coef.c:297-371): polar rule around the node
// over the 3 sub-triangles, G and H (F = 0: the element is plane; the
// tangential derivatives vanish too, q0_lit_dcoef_bd_vt2_cc_DV).  With the
// Jacobian vector J = cw0 2 / (3 sqrt3) the integrands are the quad kernel's.
__global__ void NP_BOUNDS k_q0_self_tri(bem_dom_dev D, const __grid_constant__ bem_qp q, double *__restrict__ G,
                                        double *__restrict__ H, double *__restrict__ selfF, unsigned *status,
                                        unsigned long long *terms) {
  const int p = blockIdx.x;
  const int t = p >> 2, tn = p & 3;
  const int te = abs(D.sid[t]) - 1;
  if (!bem_is_tri(D, te) || tn == 3) return;
  extern __shared__ double2 wts_s[];  // BEM_WT_SMEM bytes of dynamic shared memory
  const double2 *wts = bem_wtab_stage(q, wts_s);
  __syncthreads();
  bem_el el;
  bem_load_el(D.cr, D.cw, te, el);
  double zt, et, r[5], th[5];
  bem_tri_node(tn, zt, et);
  bem_tri_node_r_th(zt, et, r, th);
  double J[3];
  for (int d = 0; d < 3; ++d) J[d] = el.cw[d][0] * (2.0 / (3.0 * BEM_SQ3));
  const double aJ = sqrt(dot3(J, J));
  double v[16];
#pragma unroll
  for (int c = 0; c < 16; ++c) v[c] = 0.0;
  unsigned st = 0;
  unsigned long long nterm = 0, npt = 0;
  for (int pt = threadIdx.x; pt < 384 * BEM_GLN; pt += NP_THREADS) {
    const int idx = pt / BEM_GLN, ir = pt % BEM_GLN;
    const polar_pt tp = polar_theta(th, idx);
    const double rm = bem_rmax(r[tp.j], r[tp.j + 1], th[tp.j], th[tp.j + 1], tp.th);
    if (rm < 0.0) st |= BEM_ST_GEOMETRY;
    double sth, cth;
    sincos(tp.th, &sth, &cth);
    const double rr = 0.5 * rm * (c_q.xl[ir] + 1.0);
    const double w = tp.wth * 0.5 * rm * c_q.wl[ir];
    const double z = rr * cth + zt, e = rr * sth + et;
    double K[3];
    bem_K(el, rr, cth, sth, zt, et, K);
    bem_gval gv;
    const int rc = bem_qpgf(q, rr * K[0], rr * K[1], rr * K[2], gv, wts);
    if (rc < 0) st |= (rc == -12 || rc == -23) ? BEM_ST_RAYLEIGH : BEM_ST_QPGF_LIMIT;
    nterm += rc > 0 ? (unsigned long long)rc : 0ULL;
    ++npt;
    const cplx g = cscale(gv.g, aJ * rr * w);
    const cplx h = cscale(cadd(cadd(cscale(gv.gx, J[0]), cscale(gv.gy, J[1])), cscale(gv.gz, J[2])), rr * w);
    double N[4];
    bem_Nn3(z, e, N);
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      v[2 * a] += g.re * N[a];
      v[2 * a + 1] += g.im * N[a];
      v[8 + 2 * a] += h.re * N[a];
      v[8 + 2 * a + 1] += h.im * N[a];
    }
  }
  count_work(terms + 2, nterm, npt);
  set_status(status, st);
  __shared__ double sm[16 * (NP_THREADS / 32) + 16];
  block_reduce<16>(v, sm);
  if (threadIdx.x < 16) {
    const size_t N = (size_t)D.ne * 4;
    const int c = threadIdx.x;
    double *dst = c < 8 ? G : H;
    const int a = (c & 7) >> 1, part = c & 1;
    dst[2 * ((size_t)p * N + 4 * t + a) + part] = v[c];
  } else if (threadIdx.x < 19) {
    selfF[3 * p + (threadIdx.x - 16)] = 0.0;
  }
}

// Free space: lit_coef_bd (lit_coef.c:290-350) for G (H, F vanish on the plane
// element) and the principal-value tangential derivatives of G,
// lit_dcoef_bd_tz0_PV / _te0_PV (lit_dcoef.c:461-640, integrands :858-950):
// D-bar-eps (polar, 64 radii from DEPS to the edge), D-eps (closed form in the
// radius over [-pi, pi)) and the PV pair (over [0, pi)); dH vanishes.
__global__ void __launch_bounds__(NP_THREADS) k_fs_self_tri(bem_dom_dev D, double k, double *__restrict__ G,
                                                            double *__restrict__ H, double *__restrict__ dG,
                                                            double *__restrict__ dH, double *__restrict__ selfF,
                                                            unsigned *status, int p0) {
  const int p = p0 + blockIdx.x;
  const int t = p >> 2, tn = p & 3;
  const int te = abs(D.sid[t]) - 1;
  if (!bem_is_tri(D, te) || tn == 3) return;
  bem_el el;
  bem_load_el(D.cr, D.cw, te, el);
  double zt, et, r[5], th[5];
  bem_tri_node(tn, zt, et);
  bem_tri_node_r_th(zt, et, r, th);
  double vz[3], ve[3], cw0[3];
  for (int d = 0; d < 3; ++d) {
    vz[d] = el.cr[d][1];
    ve[d] = el.cr[d][2];
    cw0[d] = el.cw[d][0];
  }
  const double aJ = sqrt(dot3(cw0, cw0)) * (2.0 / (3.0 * BEM_SQ3));
  // accumulators: G (8), dGz (8), dGe (8)
  double v[24];
#pragma unroll
  for (int c = 0; c < 24; ++c) v[c] = 0.0;
  unsigned st = 0;
  // (1) G: 3 x 128 angles x 12 radii from 0 to the edge (lit_sG_r: e^{ik aK r} / aK N)
  for (int pt = threadIdx.x; pt < 384 * BEM_GLN; pt += NP_THREADS) {
    const int idx = pt / BEM_GLN, ir = pt % BEM_GLN;
    const polar_pt tp = polar_theta(th, idx);
    const double rm = bem_rmax(r[tp.j], r[tp.j + 1], th[tp.j], th[tp.j + 1], tp.th);
    if (rm < 0.0) st |= BEM_ST_GEOMETRY;
    double sth, cth;
    sincos(tp.th, &sth, &cth);
    const double rr = 0.5 * rm * (c_q.xl[ir] + 1.0);
    const double w = tp.wth * 0.5 * rm * c_q.wl[ir];
    double K[3];
    bem_K(el, rr, cth, sth, zt, et, K);
    const double aK = sqrt(dot3(K, K));
    const cplx g = cscale(cexpi(k * aK * rr), w / aK);
    double N[4];
    bem_Nn3(rr * cth + zt, rr * sth + et, N);
#pragma unroll
    for (int n = 0; n < 4; ++n) { v[2 * n] += g.re * N[n]; v[2 * n + 1] += g.im * N[n]; }
  }
  // (2) D-bar-eps: 3 x 128 angles x 64 radii from DEPS to the edge (lit_sdG_Db_r)
  for (int pt = threadIdx.x; pt < 384 * BEM_GHN; pt += NP_THREADS) {
    const int idx = pt / BEM_GHN, ir = pt % BEM_GHN;
    const polar_pt tp = polar_theta(th, idx);
    const double rm = bem_rmax(r[tp.j], r[tp.j + 1], th[tp.j], th[tp.j + 1], tp.th);
    if (rm < 0.0) st |= BEM_ST_GEOMETRY;
    double sth, cth;
    sincos(tp.th, &sth, &cth);
    const double rr = 0.5 * (rm - BEM_DEPS) * c_q.xh[ir] + 0.5 * (rm + BEM_DEPS);
    const double w = tp.wth * 0.5 * (rm - BEM_DEPS) * c_q.wh[ir];
    double K[3];
    bem_K(el, rr, cth, sth, zt, et, K);
    const double aK = sqrt(dot3(K, K)), iK = 1.0 / aK;
    const double kR = k * aK * rr;
    const cplx cbce = cmul(cmk(-1.0, kR), cexpi(kR));
    const double f = w / rr * iK * iK * iK;  // (K.v / aK) / aK^2 / r
    const cplx gz = cscale(cbce, f * dot3(K, vz)), ge = cscale(cbce, f * dot3(K, ve));
    double N[4];
    bem_Nn3(rr * cth + zt, rr * sth + et, N);
#pragma unroll
    for (int n = 0; n < 4; ++n) {
      v[8 + 2 * n] += gz.re * N[n];  v[8 + 2 * n + 1] += gz.im * N[n];
      v[16 + 2 * n] += ge.re * N[n]; v[16 + 2 * n + 1] += ge.im * N[n];
    }
  }
  // (3) D-eps, times i/k: 4 x 64 angles over [-pi, pi) (lit_sdG_De_theta)
  // (4) PV pair, times -1/k: 2 x 64 angles over [0, pi) (lit_sdG_DP_theta)
  for (int idx = threadIdx.x; idx < 384; idx += NP_THREADS) {
    const bool de = idx < 256;
    const int qd = de ? idx >> 6 : (idx - 256) >> 6, m = idx & 63;
    const double tht = 0.25 * CUDART_PI * c_q.xh[m] + (de ? (-0.75 + 0.5 * qd) : (0.25 + 0.5 * qd)) * CUDART_PI;
    const double wth = 0.25 * CUDART_PI * c_q.wh[m];
    double sth, cth;
    sincos(tht, &sth, &cth);
    double K[3];
    for (int d = 0; d < 3; ++d) K[d] = el.cr[d][1] * cth + el.cr[d][2] * sth;
    const double aK = sqrt(dot3(K, K)), iK = 1.0 / aK;
    const double keK = k * BEM_DEPS * aK;
    double sk, ck;
    sincos(keK, &sk, &ck);
    double dN[4];
    bem_dNn3(cth, sth, dN);
    const double i4 = iK * iK * iK * iK;  // (K.v / aK) / aK^3
    cplx f;
    if (de) {
      // (keK + i) sin keK + (2 - i keK) cos keK - 2, times i / k
      const cplx c = cmk(keK * sk + 2.0 * ck - 2.0, sk - keK * ck);
      f = cscale(cmk(-c.im, c.re), wth * i4 / k);
    } else {
      f = cmk(-wth * i4 * sk / k, 0.0);
    }
    const cplx gz = cscale(f, dot3(K, vz)), ge = cscale(f, dot3(K, ve));
#pragma unroll
    for (int n = 0; n < 4; ++n) {
      v[8 + 2 * n] += gz.re * dN[n];  v[8 + 2 * n + 1] += gz.im * dN[n];
      v[16 + 2 * n] += ge.re * dN[n]; v[16 + 2 * n + 1] += ge.im * dN[n];
    }
  }
  set_status(status, st);
  __shared__ double sm[24 * (NP_THREADS / 32) + 24];
  block_reduce<24>(v, sm);
  if (threadIdx.x == 0) {
    const size_t N = (size_t)D.ne * 4;
    const double c = BEM_I_FP * aJ;
    const double iTz = 1.0 / sqrt(dot3(vz, vz)), iTe = 1.0 / sqrt(dot3(ve, ve));
    if (G) {
      double2 *g2 = reinterpret_cast<double2 *>(G + 2 * ((size_t)p * N + 4 * t));
      double2 *h2 = reinterpret_cast<double2 *>(H + 2 * ((size_t)p * N + 4 * t));
      for (int n = 0; n < 4; ++n) {
        g2[n] = make_double2(v[2 * n] * c, v[2 * n + 1] * c);
        h2[n] = make_double2(0.0, 0.0);
      }
      selfF[3 * p] = selfF[3 * p + 1] = selfF[3 * p + 2] = 0.0;
    }
    if (dG) {
      const size_t r = 2 * (size_t)(p - p0);
      double2 *gz = reinterpret_cast<double2 *>(dG + 2 * (r * N + 4 * t));
      double2 *ge = reinterpret_cast<double2 *>(dG + 2 * ((r + 1) * N + 4 * t));
      double2 *hz = reinterpret_cast<double2 *>(dH + 2 * (r * N + 4 * t));
      double2 *he = reinterpret_cast<double2 *>(dH + 2 * ((r + 1) * N + 4 * t));
      for (int n = 0; n < 4; ++n) {
        gz[n] = make_double2(-c * iTz * v[8 + 2 * n], -c * iTz * v[8 + 2 * n + 1]);
        ge[n] = make_double2(-c * iTe * v[16 + 2 * n], -c * iTe * v[16 + 2 * n + 1]);
        hz[n] = make_double2(0.0, 0.0);
        he[n] = make_double2(0.0, 0.0);
      }
    }
  }
}

// ------------------------------------------------------------------ diagonal / dF
__global__ void k_diag(bem_dom_dev D, int exterior, const double *__restrict__ rowF, const int *__restrict__ near_n,
                       const double *__restrict__ nearF, const double *__restrict__ selfF, double *__restrict__ H,
                       double *__restrict__ dF, unsigned *status) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= D.ne * 4 || bem_pad_row(D, p)) return;
  double F = rowF[3 * p], Fz = rowF[3 * p + 1], Fe = rowF[3 * p + 2];
  const int n = near_n[p];
  for (int k = 0; k < n; ++k) {
    const double *nf = nearF + ((size_t)p * D.near_cap + k) * 3;
    F += nf[0]; Fz += nf[1]; Fe += nf[2];
  }
  F += selfF[3 * p]; Fz += selfF[3 * p + 1]; Fe += selfF[3 * p + 2];
  const double d = exterior ? 1.0 + F : F;
  const size_t N = (size_t)D.ne * 4;
  H[2 * ((size_t)p * N + p)] += d;
  dF[3 * p] = d;
  dF[3 * p + 1] = Fz;
  dF[3 * p + 2] = Fe;
  if (!isfinite(d) || !isfinite(Fz) || !isfinite(Fe)) set_status(status, BEM_ST_NONFINITE);
}

// ------------------------------------------------------------------ point evaluators (tests)
__global__ void k_faddeeva(const double *__restrict__ z, int n, double *__restrict__ w) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const cplx r = bem_faddeeva(z[2 * i], z[2 * i + 1]);
  w[2 * i] = r.re;
  w[2 * i + 1] = r.im;
}

__global__ void __launch_bounds__(128) k_qpgf_points(const __grid_constant__ bem_qp q, const double *__restrict__ r, int n, double *__restrict__ G,
                                                     double *__restrict__ dG, int *__restrict__ ret) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  bem_gval v;
  const int e = bem_qpgf(q, r[3 * i], r[3 * i + 1], r[3 * i + 2], v);
  ret[i] = e;
  G[2 * i] = v.g.re; G[2 * i + 1] = v.g.im;
  dG[6 * i + 0] = v.gx.re; dG[6 * i + 1] = v.gx.im;
  dG[6 * i + 2] = v.gy.re; dG[6 * i + 3] = v.gy.im;
  dG[6 * i + 4] = v.gz.re; dG[6 * i + 5] = v.gz.im;
}

// ------------------------------------------------------------------ real-space term table
// One block per interval j of width BEM_WT_H: A(y), B(y) (ew_real_ab) at the
// BEM_WT_DEG Chebyshev nodes of the interval, then the Chebyshev coefficients
// (discrete cosine sums).
__global__ void k_wtab_build(double k, double ve, double *__restrict__ out) {
  __shared__ double fa[BEM_WT_DEG], fb[BEM_WT_DEG];
  const int j = blockIdx.x, m = threadIdx.x;
  const double n = BEM_WT_DEG;
  const double tm = cos(CUDART_PI * (m + 0.5) / n);
  const double2 ab = ew_real_ab(k, ve, k * ve, (j + 0.5 * (1.0 + tm)) * BEM_WT_H);
  fa[m] = ab.x;
  fb[m] = ab.y;
  __syncthreads();
  double sa = 0.0, sb = 0.0;
  for (int mm = 0; mm < BEM_WT_DEG; ++mm) {
    const double c = cos(CUDART_PI * m * (mm + 0.5) / n);
    sa += fa[mm] * c;
    sb += fb[mm] * c;
  }
  const double f = (m == 0 ? 1.0 : 2.0) / n;
  out[2 * ((size_t)j * BEM_WT_DEG + m)] = sa * f;
  out[2 * ((size_t)j * BEM_WT_DEG + m) + 1] = sb * f;
}

// ------------------------------------------------------------------ spectral order table
// Block (order, interval j), thread m: the two channels of ew_spec_tab at the
// m-th Chebyshev node of the interval, then the Chebyshev coefficients.  For an
// evanescent order M = (f1 - f2) / d is twice the mean of erfcx' over
// [bv - |d|, bv + |d|] (64-point Gauss-Legendre; erfcx' < 0 everywhere, so no
// cancellation) times e^{-bv^2 - d^2}.
__global__ void k_stab_build(const __grid_constant__ bem_qp q, double ve, double *__restrict__ out) {
  __shared__ double fp[BEM_ST_DEG], fm[BEM_ST_DEG];
  const int ord = blockIdx.x, j = blockIdx.y, m = threadIdx.x;
  const int n1 = q.st_n1lo + ord / q.st_n2cnt, n2 = q.st_n2lo + ord % q.st_n2cnt;
  const double anx = bem_an(-q.kx, n1, q.g1x, n2, q.g2x), any = bem_an(-q.ky, n1, q.g1y, n2, q.g2y);
  const double bn2 = __dadd_rn(__dadd_rn(__dmul_rn(q.k, q.k), -__dmul_rn(anx, anx)), -__dmul_rn(any, any));
  double P = 0.0, M = 0.0;
  const double tm = cos(CUDART_PI * (m + 0.5) / BEM_ST_DEG);
  const double d = (j - 0.5 * q.st_nint + 0.5 * (1.0 + tm)) * BEM_ST_H;  // intervals cover [-D, D)
  if (bn2 > 0.0) {
    // propagating: Q = e^{bv^2 - d^2} w(bv + i d)
    const double bv = sqrt(bn2) * ve;
    const cplx w = bem_faddeeva(bv, d);
    const double ef = exp(bv * bv - d * d);
    P = ef * w.re;
    M = ef * w.im;
  } else if (bn2 < 0.0) {
    const double bn = sqrt(-bn2), bv = bn * ve;
    const double e0 = exp(-(bv * bv + d * d));
    P = e0 * (erfcx(bv + d) + erfcx(bv - d)) / bn;
    double sg = 0.0;
    for (int k = 0; k < BEM_GHN; ++k) {
      const double x = bv + d * c_q.xh[k];
      sg += c_q.wh[k] * (2.0 * x * erfcx(x) - 1.1283791670955125739);  // erfcx'(x); 2/sqrt(pi)
    }
    M = e0 * sg;
  }
  fp[m] = P;
  fm[m] = M;
  __syncthreads();
  double sp = 0.0, sm = 0.0;
  for (int mm = 0; mm < BEM_ST_DEG; ++mm) {
    const double c = cos(CUDART_PI * m * (mm + 0.5) / BEM_ST_DEG);
    sp += fp[mm] * c;
    sm += fm[mm] * c;
  }
  const double f = (m == 0 ? 1.0 : 2.0) / BEM_ST_DEG;
  double *o = out + 2 * (((size_t)ord * q.st_nint + j) * BEM_ST_DEG + m);
  o[0] = sp * f;
  o[1] = sm * f;
}

// ------------------------------------------------------------------ host launchers
extern "C" int bem_launch_stab(const bem_qp *q, double *out, cudaStream_t st) {
  if (q->st_n1cnt <= 0 || q->st_n2cnt <= 0 || q->st_nint <= 0) return 0;
  k_stab_build<<<dim3(q->st_n1cnt * q->st_n2cnt, q->st_nint), BEM_ST_DEG, 0, st>>>(*q, q->eta_run, out);
  bem_count_launches(1);
  return cudaPeekAtLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int bem_launch_wtab(double k, double ve, double *out, cudaStream_t st) {
  k_wtab_build<<<BEM_WT_N, BEM_WT_DEG, 0, st>>>(k, ve, out);
  bem_count_launches(1);
  return cudaPeekAtLastError() == cudaSuccess ? 0 : -1;
}

// n-point Gauss-Legendre rule on [-1, 1], nodes ascending: Newton's method on
// P_n (three-term recurrence) from the Chebyshev-like guess cos(pi (i + 3/4) /
// (n + 1/2)), weights 2 / ((1 - x^2) P_n'(x)^2); symmetric pairs are set from
// one root so that the rule is exactly symmetric.
static void gauss_legendre(int n, double *x, double *w) {
  for (int i = 0; i < (n + 1) / 2; ++i) {
    double z = cos(CUDART_PI * (i + 0.75) / (n + 0.5)), dp = 1.0;
    for (int it = 0; it < 100; ++it) {
      double p0 = 1.0, p1 = z;
      for (int m = 2; m <= n; ++m) {
        const double p2 = ((2.0 * m - 1.0) * z * p1 - (m - 1.0) * p0) / m;
        p0 = p1;
        p1 = p2;
      }
      dp = n * (z * p1 - p0) / (z * z - 1.0);
      const double dz = p1 / dp;
      z -= dz;
      if (fabs(dz) < 1e-17) break;
    }
    // derivative at the converged root
    {
      double p0 = 1.0, p1 = z;
      for (int m = 2; m <= n; ++m) {
        const double p2 = ((2.0 * m - 1.0) * z * p1 - (m - 1.0) * p0) / m;
        p0 = p1;
        p1 = p2;
      }
      dp = n * (z * p1 - p0) / (z * z - 1.0);
    }
    const double wi = 2.0 / ((1.0 - z * z) * dp * dp);
    x[i] = -z; w[i] = wi;           // z > 0: the i-th largest root
    x[n - 1 - i] = z; w[n - 1 - i] = wi;
  }
  if (n & 1) x[n / 2] = 0.0;
}

extern "C" int bem_set_constants(const double *xl, const double *wl, const double *xh, const double *wh) {
  bem_quad qq;
  for (int i = 0; i < BEM_GLN; ++i) { qq.xl[i] = xl[i]; qq.wl[i] = wl[i]; }
  for (int i = 0; i < BEM_GHN; ++i) { qq.xh[i] = xh[i]; qq.wh[i] = wh[i]; }
  // 8-point Gauss-Legendre rule on [-1, 1] (nodes and weights to 22 digits)
  const double x8[4] = {0.1834346424956498049395, 0.5255324099163289858177, 0.7966664774136267395916,
                        0.9602898564975362316836};
  const double w8[4] = {0.3626837833783619829652, 0.3137066458778872873380, 0.2223810344533744705444,
                        0.1012285362903762591525};
  // the tiers' n-point rules, nodes ascending: 8 points from the table above,
  // the others by gauss_legendre
  for (int t = 0; t < BEM_NTIER; ++t) {
    const int n = BEM_TIER_N0 - t;
    for (int i = 0; i < BEM_TIER_N0; ++i) qq.xt[t][i] = qq.wt[t][i] = 0.0;
    if (n == 8) {
      for (int i = 0; i < 4; ++i) {
        qq.xt[t][3 - i] = -x8[i]; qq.wt[t][3 - i] = w8[i];
        qq.xt[t][4 + i] = x8[i]; qq.wt[t][4 + i] = w8[i];
      }
    } else {
      gauss_legendre(n, qq.xt[t], qq.wt[t]);
    }
  }
  const double zt[4] = {-BEM_P44, BEM_P44, BEM_P44, -BEM_P44}, et[4] = {-BEM_P44, -BEM_P44, BEM_P44, BEM_P44};
  for (int i = 0; i < 4; ++i) { qq.zt[i] = zt[i]; qq.et[i] = et[i]; }
  // 9-point product Gauss rule on [-1,1]^2 (nodes 0, +-sqrt(3/5); weights 25/81, 40/81, 64/81),
  // ordered as the reference's zt_49/et_49 (bem3_aw_qd2.c:997-1008)
  const double b = 0.7745966692414833770359, w0 = 25.0 / 81.0, w1 = 40.0 / 81.0, w2 = 64.0 / 81.0;
  const double z9[9] = {-b, b, b, -b, 0.0, b, 0.0, -b, 0.0}, e9[9] = {-b, -b, b, b, -b, 0.0, b, 0.0, 0.0};
  const double w9[9] = {w0, w0, w0, w0, w1, w1, w1, w1, w2};
  for (int i = 0; i < 9; ++i) { qq.z9[i] = z9[i]; qq.e9[i] = e9[i]; qq.w9[i] = w9[i]; }
  bem_wconst wc;
  wc.relerr = BEM_MEPS;
  wc.a = CUDART_PI / sqrt(-log(wc.relerr * 0.5));
  wc.a2 = wc.a * wc.a;
  wc.c = 2.0 / CUDART_PI * wc.a;
  for (int n = 1; n <= BEM_W_TAB; ++n) wc.tab[n - 1] = exp(-wc.a2 * n * n);
  if (cudaMemcpyToSymbol(c_q, &qq, sizeof(qq)) != cudaSuccess) return -1;
  if (cudaMemcpyToSymbol(c_w, &wc, sizeof(wc)) != cudaSuccess) return -1;
  return 0;
}

extern "C" int bem_launch_faddeeva(const double *z, int n, double *w, cudaStream_t st) {
  if (n <= 0) return 0;
  k_faddeeva<<<(n + 127) / 128, 128, 0, st>>>(z, n, w);
  bem_count_launches(1);
  return cudaPeekAtLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int bem_launch_qpgf(const bem_qp *q, const double *r, int n, double *G, double *dG, int *ret, cudaStream_t st) {
  if (n <= 0) return 0;
  k_qpgf_points<<<(n + 127) / 128, 128, 0, st>>>(*q, r, n, G, dG, ret);
  bem_count_launches(1);
  return cudaPeekAtLastError() == cudaSuccess ? 0 : -1;
}

static bem_far far_params(const bem_dom_dev *D, const bem_qp *q, int periodic) {
  bem_far fr;
  fr.on = periodic && D->far_rule;
  fr.d1x = q->d1x; fr.d1y = q->d1y; fr.d2x = q->d2x; fr.d2y = q->d2y;
  fr.idet = q->idet;
  fr.k = q->k;
  return fr;
}

// The periodic kernels keep a copy of the real-space term table in dynamic
// shared memory (BEM_WT_SMEM bytes), which takes some of them past the 48 KB
// a block gets without asking.
// blocks per node of the near-singular kernels: each strides over the node's
// listed pairs (a grid over the table's whole capacity would start mostly
// empty blocks)
static int near_grid_y(const bem_dom_dev *D) { return D->near_cap < 32 ? D->near_cap : 32; }

template <class BA>
static int q0_smem_attrs_bt() {
  const int b = (int)BEM_WT_SMEM;
  const cudaFuncAttribute a = cudaFuncAttributeMaxDynamicSharedMemorySize;
  if (cudaFuncSetAttribute(k_q0_far<10, BA>, a, b) != cudaSuccess || cudaFuncSetAttribute(k_q0_far<9, BA>, a, b) != cudaSuccess ||
      cudaFuncSetAttribute(k_q0_far<8, BA>, a, b) != cudaSuccess || cudaFuncSetAttribute(k_q0_far<7, BA>, a, b) != cudaSuccess ||
      cudaFuncSetAttribute(k_q0_far<6, BA>, a, b) != cudaSuccess || cudaFuncSetAttribute(k_q0_regular<BA>, a, b) != cudaSuccess ||
      cudaFuncSetAttribute(k_q0_near<BA>, a, b) != cudaSuccess || cudaFuncSetAttribute(k_q0_self<BA>, a, b) != cudaSuccess)
    return -1;
  return 0;
}
static int q0_smem_attrs() {
  const int b = (int)BEM_WT_SMEM;
  const cudaFuncAttribute a = cudaFuncAttributeMaxDynamicSharedMemorySize;
  if (q0_smem_attrs_bt<bat_none>() || q0_smem_attrs_bt<bem_bat>()) return -1;
  if (cudaFuncSetAttribute(k_q0_regular_tri, a, b) != cudaSuccess || cudaFuncSetAttribute(k_q0_self_tri, a, b) != cudaSuccess)
    return -1;
  return 0;
}

// tier NF's kernel over its list (L.e set: grid_list blocks striding over it)
// or over the pair range [p0, p0 + np)
template <int NF, class BA>
static void launch_far(const bem_dom_dev *D, const bem_qp *q, bem_scratch *S, double *G, double *H, long long p0,
                       long long np, bem_plist L, unsigned grid_list, const BA &B, cudaStream_t st) {
  using F = far_shape<NF>;
  L.type = 1 + F::T;
  const unsigned grid = L.e ? grid_list : (unsigned)((np + F::PB - 1) / F::PB);
  if (grid == 0) return;
  k_q0_far<NF, BA><<<grid, F::TB, BEM_WT_SMEM, st>>>(*D, *q, S->flag, G, H, S->status, S->terms, p0, np, L, B);
  bem_count_launches(1);
}
template <class BA = bat_none>
static void launch_far_tiers(const bem_dom_dev *D, const bem_qp *q, bem_scratch *S, double *G, double *H, long long p0,
                             long long np, const bem_plist &L, unsigned grid_list, cudaStream_t st,
                             const BA &B = BA{}) {
  launch_far<10>(D, q, S, G, H, p0, np, L, grid_list, B, st);
  launch_far<9>(D, q, S, G, H, p0, np, L, grid_list, B, st);
  launch_far<8>(D, q, S, G, H, p0, np, L, grid_list, B, st);
  launch_far<7>(D, q, S, G, H, p0, np, L, grid_list, B, st);
  launch_far<6>(D, q, S, G, H, p0, np, L, grid_list, B, st);
}
static const bat_none k_nobat = {};

extern "C" int bem_launch_assemble(const bem_dom_dev *D, const bem_qp *q, int periodic, int exterior, double k,
                                   bem_scratch *S, double *G, double *H, double *dG, double *dH, double *dF,
                                   cudaStream_t st, cudaEvent_t *ev) {
  if (periodic && q0_smem_attrs()) return -1;
  // ev (optional): 6 events recorded around classify | regular | near | self | diag
  const int N = D->ne * 4;
  if (D->ne <= 0) return 0;
  if (D->has_tri) {
    // triangles leave padding rows and columns zero (the reference's calloc'ed matrices)
    const size_t nn = (size_t)N * N;
    if (cudaMemsetAsync(G, 0, 2 * nn * sizeof(double), st) != cudaSuccess ||
        cudaMemsetAsync(H, 0, 2 * nn * sizeof(double), st) != cudaSuccess ||
        cudaMemsetAsync(dF, 0, 3 * (size_t)N * sizeof(double), st) != cudaSuccess)
      return -1;
    if (dG && (cudaMemsetAsync(dG, 0, 4 * nn * sizeof(double), st) != cudaSuccess ||
               cudaMemsetAsync(dH, 0, 4 * nn * sizeof(double), st) != cudaSuccess))
      return -1;
  }
  const long long npairs = (long long)N * D->ne;
  // compacted pair lists for the periodic domain when the scratch holds them
  const bool lists = periodic && S->plist && S->pcount && (unsigned long long)npairs <= S->pcap &&
                     npairs <= 0xffffffffLL;
  if (lists && cudaMemsetAsync(S->pcount, 0, 2 * BEM_NLIST * sizeof(unsigned), st) != cudaSuccess) return -1;
  if (ev) cudaEventRecord(ev[0], st);
  k_classify<<<N, 128, 0, st>>>(*D, far_params(D, q, periodic), S->rowF, S->near_s, S->near_n, S->flag, S->status,
                                lists ? S->pcount : nullptr);
  bem_count_launches(1);
  if (lists) {
    k_plist_fill<<<N, 128, 0, st>>>(*D, S->flag, S->plist, S->pcount, S->pcap);
    bem_count_launches(1);
  }
  if (ev) cudaEventRecord(ev[1], st);
  if (periodic) {
    if (lists) {
      // one resident wave (RP_MINB / FP_MINB blocks per SM) striding over each list
      int dev = 0, nsm = 0;
      if (cudaGetDevice(&dev) != cudaSuccess ||
          cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || nsm <= 0)
        return -1;
      const unsigned grid = RP_MINB * (unsigned)nsm, grid_far = FP_MINB * (unsigned)nsm;
      const bem_plist Lreg = {S->plist, S->pcount, 0};
      k_q0_regular<bat_none><<<grid, RP_THREADS, BEM_WT_SMEM, st>>>(*D, *q, S->flag, G, H, S->status, S->terms, 0, npairs, Lreg,
                                                                         k_nobat);
      bem_count_launches(1);
      if (D->far_rule) launch_far_tiers(D, q, S, G, H, 0, npairs, Lreg, grid_far, st);
      if (D->has_tri) {
        k_q0_regular_tri<<<grid, RP_THREADS, BEM_WT_SMEM, st>>>(*D, *q, S->flag, G, H, S->status, S->terms, 0, npairs, Lreg);
        bem_count_launches(1);
      }
    } else {
      const bem_plist L0 = {nullptr, nullptr, 0};
      const long long chunk = 1LL << 26;  // keep grid.x well inside limits
      for (long long p0 = 0; p0 < npairs; p0 += chunk) {
        const long long np = npairs - p0 < chunk ? npairs - p0 : chunk;
        k_q0_regular<bat_none><<<(unsigned)((np + 1) / 2), RP_THREADS, BEM_WT_SMEM, st>>>(*D, *q, S->flag, G, H, S->status, S->terms,
                                                                             p0, np, L0, k_nobat);
        bem_count_launches(1);
        if (D->far_rule) launch_far_tiers(D, q, S, G, H, p0, np, L0, 0, st);
        if (D->has_tri) {
          k_q0_regular_tri<<<(unsigned)((np + 1) / 2), RP_THREADS, BEM_WT_SMEM, st>>>(*D, *q, S->flag, G, H, S->status, S->terms,
                                                                            p0, np, L0);
          bem_count_launches(1);
        }
      }
    }
    if (ev) cudaEventRecord(ev[2], st);
    k_q0_near<bat_none><<<dim3(N, near_grid_y(D)), NP_THREADS, BEM_WT_SMEM, st>>>(*D, *q, S->near_s, S->near_n, G, H, S->nearF,
                                                                              S->status, S->terms, k_nobat);
    bem_count_launches(1);
    if (ev) cudaEventRecord(ev[3], st);
    k_q0_self<bat_none><<<N, NP_THREADS, BEM_WT_SMEM, st>>>(*D, *q, G, H, S->selfF, S->status, S->terms, k_nobat);
    bem_count_launches(1);
    if (D->has_tri) {
      k_q0_self_tri<<<N, NP_THREADS, BEM_WT_SMEM, st>>>(*D, *q, G, H, S->selfF, S->status, S->terms);
      bem_count_launches(1);
    }
  } else {
    k_fs_regular<<<(unsigned)((npairs + 127) / 128), 128, 0, st>>>(*D, k, S->flag, G, H, dG, dH, 0, N);
    bem_count_launches(1);
    if (ev) cudaEventRecord(ev[2], st);
    k_fs_near<<<dim3(N, near_grid_y(D)), NP_THREADS, 0, st>>>(*D, k, S->near_s, S->near_n, G, H, dG, dH, S->nearF, 0);
    bem_count_launches(1);
    if (ev) cudaEventRecord(ev[3], st);
    k_fs_self<<<N, NP_THREADS, 0, st>>>(*D, k, G, H, dG, dH, S->selfF, S->status, 0);
    bem_count_launches(1);
    if (D->has_tri) {
      k_fs_self_tri<<<N, NP_THREADS, 0, st>>>(*D, k, G, H, dG, dH, S->selfF, S->status, 0);
      bem_count_launches(1);
    }
  }
  if (ev) cudaEventRecord(ev[4], st);
  k_diag<<<(N + 127) / 128, 128, 0, st>>>(*D, exterior, S->rowF, S->near_n, S->nearF, S->selfF, H, dF, S->status);
  bem_count_launches(1);
  if (ev) cudaEventRecord(ev[5], st);
  return cudaPeekAtLastError() == cudaSuccess ? 0 : -1;
}

// The periodic domain of a batch of nb problems on one body, media, lattice
// and frequency (bem_bat).  One classification, with q (instance 0's
// parameters: pair flags, rule tiers, lists and geometric sums depend on the
// geometry, the lattice and k only), then each kernel launched once for up to
// BEM_BAT_MAX instances: the regular-pair kernels stride over the lists
// instance after instance, the near-singular and self kernels take the
// instance from blockIdx.z; the diagonal per instance.  qps, Gh, Hh: the
// instances' parameters and output pointers, on the host.  Quad meshes with
// pair lists only (-2 otherwise).
extern "C" int bem_launch_assemble_batch(const bem_dom_dev *D, const bem_qp *q, int nb, const bem_qp *qps,
                                         double *const *Gh, double *const *Hh, bem_scratch *S, double *dF,
                                         cudaStream_t st) {
  if (q0_smem_attrs()) return -1;
  const int N = D->ne * 4;
  if (D->ne <= 0 || nb <= 0) return 0;
  if (D->has_tri) return -2;
  const long long npairs = (long long)N * D->ne;
  if (!(S->plist && S->pcount && (unsigned long long)npairs <= S->pcap && npairs <= 0xffffffffLL)) return -2;
  if (cudaMemsetAsync(S->pcount, 0, 2 * BEM_NLIST * sizeof(unsigned), st) != cudaSuccess) return -1;
  k_classify<<<N, 128, 0, st>>>(*D, far_params(D, q, 1), S->rowF, S->near_s, S->near_n, S->flag, S->status,
                                S->pcount);
  bem_count_launches(1);
  k_plist_fill<<<N, 128, 0, st>>>(*D, S->flag, S->plist, S->pcount, S->pcap);
  bem_count_launches(1);
  int dev = 0, nsm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || nsm <= 0)
    return -1;
  const bem_plist Lreg = {S->plist, S->pcount, 0};
  bem_bat B;  // 20 KB on the host stack, copied into each launch's argument block
  for (int b0 = 0; b0 < nb; b0 += BEM_BAT_MAX) {
    B.nb = nb - b0 < BEM_BAT_MAX ? nb - b0 : BEM_BAT_MAX;
    for (int i = 0; i < B.nb; ++i) {
      B.qp[i] = qps[b0 + i];
      B.G[i] = Gh[b0 + i];
      B.H[i] = Hh[b0 + i];
    }
    k_q0_regular<bem_bat><<<RP_MINB * (unsigned)nsm, RP_THREADS, BEM_WT_SMEM, st>>>(
        *D, *q, S->flag, nullptr, nullptr, S->status, S->terms, 0, npairs, Lreg, B);
    bem_count_launches(1);
    if (D->far_rule) launch_far_tiers(D, q, S, nullptr, nullptr, 0, npairs, Lreg, FP_MINB * (unsigned)nsm, st, B);
    k_q0_near<bem_bat><<<dim3(N, near_grid_y(D), B.nb), NP_THREADS, BEM_WT_SMEM, st>>>(
        *D, *q, S->near_s, S->near_n, nullptr, nullptr, S->nearF, S->status, S->terms, B);
    bem_count_launches(1);
    k_q0_self<bem_bat><<<dim3(N, 1, B.nb), NP_THREADS, BEM_WT_SMEM, st>>>(*D, *q, nullptr, nullptr, S->selfF,
                                                                       S->status, S->terms, B);
    bem_count_launches(1);
  }
  for (int b = 0; b < nb; ++b) {
    k_diag<<<(N + 127) / 128, 128, 0, st>>>(*D, 1, S->rowF, S->near_n, S->nearF, S->selfF, Hh[b], dF, S->status);
    bem_count_launches(1);
  }
  return cudaPeekAtLastError() == cudaSuccess ? 0 : -1;
}

// Time the periodic regular-pair kernel on a sample of the pairs (nchunk
// chunks of frac / nchunk of all pairs, spread over the node range) for the
// Ewald-parameter autotuner; the pair flags must be current (k_classify).
extern "C" int bem_time_regular(const bem_dom_dev *D, const bem_qp *q, bem_scratch *S, double *G, double *H,
                                double frac, int nchunk, cudaStream_t st, float *ms) {
  if (q0_smem_attrs()) return -1;
  const long long npairs = (long long)D->ne * 4 * D->ne;
  const long long len = (long long)(npairs * frac / nchunk) + 1;
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return -1;
  cudaEventRecord(e0, st);
  for (int c = 0; c < nchunk; ++c) {
    const long long p0 = npairs * c / nchunk;
    const long long np = p0 + len <= npairs ? len : npairs - p0;
    if (np > 0) {
      // the kernels of the assembly itself (over pair ranges, not lists):
      // quad sources, the shorter-rule tiers, and triangle sources when there are any
      const bem_plist L0 = {nullptr, nullptr, 0};
      k_q0_regular<bat_none><<<(unsigned)((np + 1) / 2), RP_THREADS, BEM_WT_SMEM, st>>>(*D, *q, S->flag, G, H, S->status, S->terms,
                                                                           p0, np, L0, k_nobat);
      bem_count_launches(1);
      if (D->far_rule) launch_far_tiers(D, q, S, G, H, p0, np, L0, 0, st);
      if (D->has_tri) {
        k_q0_regular_tri<<<(unsigned)((np + 1) / 2), RP_THREADS, BEM_WT_SMEM, st>>>(*D, *q, S->flag, G, H, S->status, S->terms,
                                                                          p0, np, L0);
        bem_count_launches(1);
      }
    }
  }
  cudaEventRecord(e1, st);
  int rc = cudaEventSynchronize(e1) == cudaSuccess && cudaEventElapsedTime(ms, e0, e1) == cudaSuccess ? 0 : -1;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (cudaPeekAtLastError() != cudaSuccess) rc = -1;
  return rc;
}

// The free-space kernels over the rows p0 .. p0 + np - 1 writing only dG and
// dH (row 2 (p - p0) of each): the derivative rows of an interior domain
// recomputed a block of rows at a time for the particle velocity, instead of
// kept (2 x 2N x N complex).  The pair flags and near lists must be current
// (bem_launch_classify).
extern "C" int bem_launch_fs_deriv(const bem_dom_dev *D, double k, bem_scratch *S, int p0, int np, double *dG,
                                   double *dH, cudaStream_t st) {
  if (np <= 0 || D->ne <= 0) return 0;
  const long long npairs = (long long)np * D->ne;
  k_fs_regular<<<(unsigned)((npairs + 127) / 128), 128, 0, st>>>(*D, k, S->flag, nullptr, nullptr, dG, dH, p0, np);
  bem_count_launches(1);
  k_fs_near<<<dim3(np, near_grid_y(D)), NP_THREADS, 0, st>>>(*D, k, S->near_s, S->near_n, nullptr, nullptr, dG, dH,
                                                          S->nearF, p0);
  bem_count_launches(1);
  k_fs_self<<<np, NP_THREADS, 0, st>>>(*D, k, nullptr, nullptr, dG, dH, S->selfF, S->status, p0);
  bem_count_launches(1);
  if (D->has_tri) {
    k_fs_self_tri<<<np, NP_THREADS, 0, st>>>(*D, k, nullptr, nullptr, dG, dH, S->selfF, S->status, p0);
    bem_count_launches(1);
  }
  return cudaPeekAtLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int bem_launch_classify(const bem_dom_dev *D, const bem_qp *q, int periodic, bem_scratch *S, cudaStream_t st) {
  if (D->ne <= 0) return 0;
  k_classify<<<D->ne * 4, 128, 0, st>>>(*D, far_params(D, q, periodic), S->rowF, S->near_s, S->near_n, S->flag, S->status,
                                        nullptr);
  bem_count_launches(1);
  return cudaPeekAtLastError() == cudaSuccess ? 0 : -1;
}

#include "bem_post.cuh"
