// Global system, boundary values and post-processing on the device.
//
//   k_gather       dense A (n x n, n = 2 NN, row-major) from the per-domain
//                  G and H: main-domain side [ H | -G ], sub-domain side
//                  [ hk2 H | G ], hk2 = k2(main)/k2(sub)
//                  (create_matrix_csr_dac, bem3_aw_qd2_solve_bieq.c:244-345)
//   k_rhs          b = sum(-hk2 H Pi - G dPi) over sub-domain-side sources whose
//                  main domain is 0 (same function, :287-319)
//   k_store        X -> P, dP per domain (tmatrix_bd_store, :370-427)
//   k_pv_interior  tangential derivatives from the dG, dH rows, 3x3 inverse,
//                  particle velocity and the interface condition for domain 0
//                  (q_solve_pv_bv, :655-750; dpdt_fcm :516; inv_matrix_33 :493)
//   k_pv_exterior  domain-0 velocity from the interface condition
//   k_dpv_rhs      B = H pv (3 right-hand sides) for the dpv solve (solve_dpv_bv, :533-653)
//   k_force0       radiation force and torque, 4-point rule at the element
//                  nodes (force_FN_aqd2 + bil_force_4p, bem3_aw_qd2_force.c:4-120)
// The LU factorisations themselves are the device LU of bem_lu.cu (bem_capi.cu).
#include "bem_count.h"
#include <cuda_runtime.h>
#include <stdint.h>
#include "bem_solve.h"

struct zc { double re, im; };
__device__ __forceinline__ zc zmk(double a, double b) { zc z; z.re = a; z.im = b; return z; }
__device__ __forceinline__ zc zmul(zc a, zc b) { return zmk(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
__device__ __forceinline__ zc zadd(zc a, zc b) { return zmk(a.re + b.re, a.im + b.im); }
__device__ __forceinline__ zc zsub(zc a, zc b) { return zmk(a.re - b.re, a.im - b.im); }
__device__ __forceinline__ zc zld(const double *p) { return zmk(p[0], p[1]); }
__device__ __forceinline__ void zst(double *p, zc v) { p[0] = v.re; p[1] = v.im; }
__device__ __forceinline__ zc zdiv(zc a, zc b) {
  const double d = b.re * b.re + b.im * b.im;
  return zmk((a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d);
}

// one thread per (row p, source column c = 4 s + l) of domain d
__global__ void k_gather(bem_sys_dev S, int d, const double *__restrict__ G, const double *__restrict__ H, double *__restrict__ A) {
  const int Nd = S.dom_ne[d] * 4;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)Nd * Nd) return;
  const int p = (int)(idx / Nd), c = (int)(idx % Nd);
  const int row = S.rowidx[S.dom_off[d] * 4 + p];
  if (row < 0) return;
  const int s = c >> 2, l = c & 3;
  const int asd = abs(S.sid[S.dom_off[d] + s]) - 1;
  if (l >= S.npe[asd]) return;
  const int col = S.eni[asd * 4 + l];
  const size_t n = (size_t)S.n;
  const zc h = zld(H + 2 * ((size_t)p * Nd + c)), g = zld(G + 2 * ((size_t)p * Nd + c));
  double *ap = A + 2 * ((size_t)row * n + col);
  double *aq = A + 2 * ((size_t)row * n + S.NN + col);
  if (d == S.md[asd]) {
    zst(ap, h);
    zst(aq, zmk(-g.re, -g.im));
  } else {
    zst(ap, zmul(zld(S.hk2 + 2 * asd), h));
    zst(aq, g);
  }
}

// one warp per row p of domain d
__global__ void k_rhs(bem_sys_dev S, int d, const double *__restrict__ G, const double *__restrict__ H, double *__restrict__ b) {
  const int Nd = S.dom_ne[d] * 4;
  const int p = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x & 31;
  if (p >= Nd) return;
  const int row = S.rowidx[S.dom_off[d] * 4 + p];
  if (row < 0) return;
  zc acc = zmk(0, 0);
  for (int c = lane; c < Nd; c += 32) {
    const int s = c >> 2, l = c & 3;
    const int asd = abs(S.sid[S.dom_off[d] + s]) - 1;
    if (l >= S.npe[asd]) continue;
    if (d == S.md[asd] || S.md[asd] != 0) continue;
    const zc h = zld(H + 2 * ((size_t)p * Nd + c)), g = zld(G + 2 * ((size_t)p * Nd + c));
    const zc t1 = zmul(zmul(zld(S.hk2 + 2 * asd), h), zld(S.Pi + 2 * (asd * 4 + l)));
    const zc t2 = zmul(g, zld(S.dPi + 2 * (asd * 4 + l)));
    acc = zsub(acc, zadd(t1, t2));
  }
  for (int o = 16; o > 0; o >>= 1) {
    acc.re += __shfl_down_sync(0xffffffffu, acc.re, o);
    acc.im += __shfl_down_sync(0xffffffffu, acc.im, o);
  }
  if (lane == 0) zst(b + 2 * row, acc);
}

// X -> P, dP of domain d: one thread per element node
__global__ void k_store(bem_sys_dev S, int d, const double *__restrict__ X, double *__restrict__ P, double *__restrict__ dP) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= S.dom_ne[d] * 4) return;
  const int s = i >> 2, l = i & 3;
  const int asd = abs(S.sid[S.dom_off[d] + s]) - 1;
  if (l >= S.npe[asd]) { zst(P + 2 * i, zmk(0, 0)); zst(dP + 2 * i, zmk(0, 0)); return; }
  const int e = S.eni[asd * 4 + l];
  const zc x0 = zld(X + 2 * e), x1 = zld(X + 2 * (S.NN + e));
  if (d == S.md[asd]) {
    zst(P + 2 * i, x0);
    zst(dP + 2 * i, x1);
  } else {
    const zc hk2 = zld(S.hk2 + 2 * asd);
    zc p = zmul(hk2, x0), dp = zmk(-x1.re, -x1.im);
    if (S.md[asd] == 0) {
      p = zadd(p, zmul(hk2, zld(S.Pi + 2 * (asd * 4 + l))));
      dp = zsub(dp, zld(S.dPi + 2 * (asd * 4 + l)));
    }
    zst(P + 2 * i, p);
    zst(dP + 2 * i, dp);
  }
}

// inverse of the 3x3 matrix with rows (vn, vtz, vte) (inv_matrix_33)
__device__ __forceinline__ void inv33(double *ma, const double *vn, const double *vz, const double *ve) {
  const double idet = 1.0 / (vn[0] * vz[1] * ve[2] + vn[1] * vz[2] * ve[0] + vn[2] * vz[0] * ve[1] -
                             (vn[2] * vz[1] * ve[0] + vn[1] * vz[0] * ve[2] + vn[0] * vz[2] * ve[1]));
  ma[0] = vz[1] * ve[2] - vz[2] * ve[1];
  ma[1] = -vn[1] * ve[2] + vn[2] * ve[1];
  ma[2] = vn[1] * vz[2] - vn[2] * vz[1];
  ma[3] = -vz[0] * ve[2] + vz[2] * ve[0];
  ma[4] = vn[0] * ve[2] - vn[2] * ve[0];
  ma[5] = -vn[0] * vz[2] + vn[2] * vz[0];
  ma[6] = vz[0] * ve[1] - vz[1] * ve[0];
  ma[7] = -vn[0] * ve[1] + vn[1] * ve[0];
  ma[8] = vn[0] * vz[1] - vn[1] * vz[0];
  for (int i = 0; i < 9; ++i) ma[i] *= idet;
}

// one warp per collocation row p of interior domain d
// rows p0 .. p0 + np - 1; dG, dH hold rows 2 (p - p0) and 2 (p - p0) + 1
__global__ void k_pv_interior(bem_sys_dev S, int d, const double *__restrict__ dG, const double *__restrict__ dH,
                              const double *__restrict__ dF, const double *__restrict__ P, const double *__restrict__ dP,
                              double *__restrict__ pv, double *__restrict__ tpv, int p0, int np) {
  const int Nd = S.dom_ne[d] * 4;
  const int p = p0 + blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x & 31;
  if (p >= p0 + np || p >= Nd) return;
  const int t = p >> 2, tn = p & 3;
  const int at = S.sid[S.dom_off[d] + t];
  const int atd = abs(at) - 1;
  if (tn >= S.npe[atd]) return;
  zc az = zmk(0, 0), ae = zmk(0, 0);
  const size_t r2 = 2 * (size_t)(p - p0);
  const double *rz = dG + 2 * r2 * Nd, *re = dG + 2 * (r2 + 1) * Nd;
  const double *hz = dH + 2 * r2 * Nd, *he = dH + 2 * (r2 + 1) * Nd;
  for (int c = lane; c < Nd; c += 32) {
    const zc dp = zld(dP + 2 * c), pp = zld(P + 2 * c);
    az = zadd(az, zsub(zmul(zld(rz + 2 * c), dp), zmul(zld(hz + 2 * c), pp)));
    ae = zadd(ae, zsub(zmul(zld(re + 2 * c), dp), zmul(zld(he + 2 * c), pp)));
  }
  for (int o = 16; o > 0; o >>= 1) {
    az.re += __shfl_down_sync(0xffffffffu, az.re, o);
    az.im += __shfl_down_sync(0xffffffffu, az.im, o);
    ae.re += __shfl_down_sync(0xffffffffu, ae.re, o);
    ae.im += __shfl_down_sync(0xffffffffu, ae.im, o);
  }
  if (lane != 0) return;
  const double f0 = dF[3 * p], f1 = dF[3 * p + 1], f2 = dF[3 * p + 2];
  const zc Pp = zld(P + 2 * p), dPp = zld(dP + 2 * p);
  const zc dPz = zmk((az.re - Pp.re * f1) / f0, (az.im - Pp.im * f1) / f0);
  const zc dPe = zmk((ae.re - Pp.re * f2) / f0, (ae.im - Pp.im * f2) / f0);
  // unit tangents at the node (tz_te_bd_node) and the signed unit normal
  double vz[3], ve[3], vn[3], a[9];
  const double *cr = S.cr + (size_t)atd * 12;
  double nz = 0, ne = 0, nn = 0;
  for (int i = 0; i < 3; ++i) {
    vz[i] = cr[i * 4 + 1] + cr[i * 4 + 3] * S.et44[tn];
    ve[i] = cr[i * 4 + 2] + cr[i * 4 + 3] * S.zt44[tn];
    vn[i] = (at < 0 ? -1.0 : 1.0) * S.wen[(size_t)atd * 12 + tn * 3 + i];
    nz += vz[i] * vz[i]; ne += ve[i] * ve[i]; nn += vn[i] * vn[i];
  }
  nz = sqrt(nz); ne = sqrt(ne); nn = sqrt(nn);
  for (int i = 0; i < 3; ++i) { vz[i] /= nz; ve[i] /= ne; vn[i] /= nn; }
  inv33(a, vn, vz, ve);
  zc v[3];
  for (int i = 0; i < 3; ++i) {
    const zc s = zadd(zadd(zmk(dPp.re * a[i * 3], dPp.im * a[i * 3]), zmk(dPz.re * a[i * 3 + 1], dPz.im * a[i * 3 + 1])),
                      zmk(dPe.re * a[i * 3 + 2], dPe.im * a[i * 3 + 2]));
    v[i] = zmk(-s.re, -s.im);
    zst(pv + 2 * (3 * p + i), v[i]);
  }
  if (S.md[atd] == 0) {
    // continuity of the normal velocity and of rho times the tangential velocity
    const double r0 = S.rho0[0], rd = S.rho0[d];
    const double *vi = S.v_inc + 2 * 3 * ((size_t)atd * 4 + tn);
    zc rhs[3] = {zmk(0, 0), zmk(0, 0), zmk(0, 0)};
    for (int i = 0; i < 3; ++i) {
      const zc vinc = zmk(vi[2 * i], vi[2 * i + 1]);
      const zc dv = zsub(v[i], vinc);
      const zc rv = zsub(zmk(rd * v[i].re, rd * v[i].im), zmk(r0 * vinc.re, r0 * vinc.im));
      rhs[0] = zadd(rhs[0], zmk(vn[i] * dv.re, vn[i] * dv.im));
      rhs[1] = zadd(rhs[1], zmk(vz[i] * rv.re, vz[i] * rv.im));
      rhs[2] = zadd(rhs[2], zmk(ve[i] * rv.re, ve[i] * rv.im));
    }
    double rtz[3], rte[3], b2[9];
    for (int i = 0; i < 3; ++i) { rtz[i] = r0 * vz[i]; rte[i] = r0 * ve[i]; }
    inv33(b2, vn, rtz, rte);
    const int e = S.eni[atd * 4 + tn];
    for (int i = 0; i < 3; ++i) {
      const zc o = zadd(zadd(zmk(b2[i * 3] * rhs[0].re, b2[i * 3] * rhs[0].im), zmk(b2[i * 3 + 1] * rhs[1].re, b2[i * 3 + 1] * rhs[1].im)),
                        zmk(b2[i * 3 + 2] * rhs[2].re, b2[i * 3 + 2] * rhs[2].im));
      zst(tpv + 2 * (3 * (size_t)e + i), o);
    }
  }
}

__global__ void k_pv_exterior(bem_sys_dev S, const double *__restrict__ tpv, double *__restrict__ pv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= S.dom_ne[0] * 4) return;
  const int t = i >> 2, tn = i & 3;
  const int atd = abs(S.sid[t]) - 1;
  if (tn >= S.npe[atd]) return;
  const int e = S.eni[atd * 4 + tn];
  for (int c = 0; c < 3; ++c) zst(pv + 2 * (3 * i + c), zld(tpv + 2 * (3 * (size_t)e + c)));
}

// B[c][i] = sum_j H[c][j] pv[j][i], stored column-major (i-th right-hand side contiguous)
__global__ void k_dpv_rhs(int Nd, const double *__restrict__ H, const double *__restrict__ pv, double *__restrict__ B) {
  const int c = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x & 31;
  if (c >= Nd) return;
  zc acc[3] = {zmk(0, 0), zmk(0, 0), zmk(0, 0)};
  const double *hr = H + 2 * (size_t)c * Nd;
  for (int j = lane; j < Nd; j += 32) {
    const zc h = zld(hr + 2 * j);
    for (int i = 0; i < 3; ++i) acc[i] = zadd(acc[i], zmul(h, zld(pv + 2 * (3 * j + i))));
  }
  for (int i = 0; i < 3; ++i)
    for (int o = 16; o > 0; o >>= 1) {
      acc[i].re += __shfl_down_sync(0xffffffffu, acc[i].re, o);
      acc[i].im += __shfl_down_sync(0xffffffffu, acc[i].im, o);
    }
  if (lane == 0)
    for (int i = 0; i < 3; ++i) zst(B + 2 * ((size_t)i * Nd + c), acc[i]);
}

// column-major B (N x 3) -> dpv[j][i]
__global__ void k_dpv_store(int Nd, const double *__restrict__ B, double *__restrict__ dpv) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= Nd) return;
  for (int i = 0; i < 3; ++i) zst(dpv + 2 * (3 * j + i), zld(B + 2 * ((size_t)i * Nd + j)));
}

// Domains with triangles: the dpv system keeps only real nodes (solve_dpv_bv,
// bem3_aw_qd2_solve_bieq.c:556-600 skips row and column 3 of each triangle).
// inv[r] = full index of compact index r.
__global__ void k_compress_mat(const double *__restrict__ G, int N, const int *__restrict__ inv, int nn,
                               double *__restrict__ Gc) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)nn * nn) return;
  const int r = (int)(idx / nn), c = (int)(idx % nn);
  zst(Gc + 2 * idx, zld(G + 2 * ((size_t)inv[r] * N + inv[c])));
}
// column-major right-hand sides: to = 0 compact <- full, 1 full <- compact (padding rows 0)
__global__ void k_move_rows(const double *__restrict__ src, double *__restrict__ dst, int N, const int *__restrict__ inv,
                            int nn, int nrhs, int to_full) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (to_full) {
    if (r >= N) return;
    for (int i = 0; i < nrhs; ++i) zst(dst + 2 * ((size_t)i * N + r), zmk(0, 0));
    return;
  }
  if (r >= nn) return;
  for (int i = 0; i < nrhs; ++i) zst(dst + 2 * ((size_t)i * nn + r), zld(src + 2 * ((size_t)i * N + inv[r])));
}
__global__ void k_scatter_rows(const double *__restrict__ src, double *__restrict__ dst, int N, const int *__restrict__ inv,
                               int nn, int nrhs) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nn) return;
  for (int i = 0; i < nrhs; ++i) zst(dst + 2 * ((size_t)i * N + inv[r]), zld(src + 2 * ((size_t)i * nn + r)));
}

// radiation force and torque with node values (bil_force_4p, bem3_aw_qd2_force.c:73-120): one block.
// Triangles (lit_force_4p, :167-228): the 3 nodes with weight 25/96 and the centre with
// weight -27/96, whose p and v are boundary values (ctr: per domain-0 element, the
// centre's S0, S2, F from k_bdval, or -1; pw: the incident plane wave).
__global__ void k_force0(bem_sys_dev S, const double *__restrict__ P0, const double *__restrict__ pv0, const double *rc,
                         double c0, double rho0, const int *__restrict__ ctr, const double *__restrict__ cbd,
                         const double *__restrict__ pw, double *__restrict__ out) {
  const double c1 = 0.25 / (c0 * c0 * rho0), c2 = 0.25 * rho0, c3 = 0.5 * rho0;
  const zc k2 = zld(S.k2);
  double acc[6] = {0, 0, 0, 0, 0, 0};
  const int n = S.dom_ne[0] * 4;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const int t = i >> 2, tn = i & 3;
    const int asd = abs(S.sid[t]) - 1;
    const bool tri = S.npe[asd] == 3;
    zc p, v[3];
    double rb[3], wb[3], wt = 1.0;  // 4-point rule weights (wt_44) are all 1
    if (tri && tn == 3) {
      if (!ctr) continue;
      // centre of the triangle: r = cr0, W = cw0, boundary values from k_bdval
      const double *b = cbd + 9 * (size_t)ctr[t];
      const double cf = 1.0 / (1.0 + b[8]);
      const double *crp = S.cr + (size_t)asd * 12;
      for (int d = 0; d < 3; ++d) { rb[d] = crp[d * 4]; wb[d] = S.wen[(size_t)asd * 12 + d]; }
      const double *R = pw + 2;
      const double r0z = -R[6] * (rb[0] - pw[11]) - R[7] * (rb[1] - pw[12]) + R[8] * (rb[2] - pw[13]);
      double sz, cz;
      sincos(pw[14] * r0z, &sz, &cz);
      const zc pinc = zmul(zmk(pw[0], pw[1]), zmk(cz, sz));
      const zc vz = zmk(pinc.re / pw[15], pinc.im / pw[15]);
      p = zadd(zmk(-(k2.re * b[0] - k2.im * b[1]) * cf, -(k2.re * b[1] + k2.im * b[0]) * cf), pinc);
      for (int l = 0; l < 3; ++l) v[l] = zadd(zmk(b[2 + 2 * l] * cf, b[3 + 2 * l] * cf), zmk(vz.re * R[l * 3 + 2], vz.im * R[l * 3 + 2]));
      wt = 0.5 * (-27.0 / 48.0);
    } else {
      if (tn >= S.npe[asd]) continue;
      for (int d = 0; d < 3; ++d) { rb[d] = S.ren[(size_t)asd * 12 + tn * 3 + d]; wb[d] = S.wen[(size_t)asd * 12 + tn * 3 + d]; }
      p = zsub(zld(S.p_inc + 2 * (asd * 4 + tn)), zmul(zld(P0 + 2 * i), k2));
      for (int l = 0; l < 3; ++l) v[l] = zadd(zld(S.v_inc + 2 * (3 * (asd * 4 + tn) + l)), zld(pv0 + 2 * (3 * i + l)));
      if (tri) wt = 0.5 * (25.0 / 48.0);
    }
    const double *r = rb, *w = wb;
    const double t1 = c1 * (p.re * p.re + p.im * p.im) - c2 * (v[0].re * v[0].re + v[0].im * v[0].im + v[1].re * v[1].re +
                                                               v[1].im * v[1].im + v[2].re * v[2].re + v[2].im * v[2].im);
    double T[9];
    for (int l = 0; l < 3; ++l)
      for (int m = 0; m < 3; ++m) T[l * 3 + m] = c3 * (v[l].re * v[m].re + v[l].im * v[m].im);
    T[0] += t1; T[4] += t1; T[8] += t1;
    double Tw[3];
    for (int l = 0; l < 3; ++l) Tw[l] = T[l * 3] * w[0] + T[l * 3 + 1] * w[1] + T[l * 3 + 2] * w[2];
    for (int l = 0; l < 3; ++l) acc[l] += Tw[l] * wt;
    const double dx = r[0] - rc[0], dy = r[1] - rc[1], dz = r[2] - rc[2];
    acc[3] += (dy * Tw[2] - dz * Tw[1]) * wt;
    acc[4] += (dz * Tw[0] - dx * Tw[2]) * wt;
    acc[5] += (dx * Tw[1] - dy * Tw[0]) * wt;
  }
  __shared__ double sm[6][256];
  for (int c = 0; c < 6; ++c) sm[c][threadIdx.x] = acc[c];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      for (int c = 0; c < 6; ++c) sm[c][threadIdx.x] += sm[c][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int c = 0; c < 6; ++c) out[c] = sm[c][0];
}

// ------------------------------------------------------------------ launchers
extern "C" int bem_launch_gather(const bem_sys_dev *S, int d, const double *G, const double *H, double *A, double *b,
                                 cudaStream_t st) {
  const long long Nd = (long long)S->dom_ne_h[d] * 4;
  if (Nd == 0) return 0;
  if (A) {
    k_gather<<<(unsigned)((Nd * Nd + 255) / 256), 256, 0, st>>>(*S, d, G, H, A);
    bem_count_launches(1);
  }
  k_rhs<<<(unsigned)((Nd + 7) / 8), 256, 0, st>>>(*S, d, G, H, b);
  bem_count_launches(1);
  return cudaPeekAtLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int bem_launch_store(const bem_sys_dev *S, int d, const double *X, double *P, double *dP, cudaStream_t st) {
  const int n = S->dom_ne_h[d] * 4;
  if (n == 0) return 0;
  k_store<<<(n + 127) / 128, 128, 0, st>>>(*S, d, X, P, dP);
  bem_count_launches(1);
  return cudaPeekAtLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int bem_launch_pv(const bem_sys_dev *S, int d, const double *dG, const double *dH, const double *dF,
                             const double *P, const double *dP, double *pv, double *tpv, cudaStream_t st) {
  const int n = S->dom_ne_h[d] * 4;
  if (n == 0) return 0;
  if (d == 0) {
    k_pv_exterior<<<(n + 127) / 128, 128, 0, st>>>(*S, tpv, pv);
    bem_count_launches(1);
    return cudaPeekAtLastError() == cudaSuccess ? 0 : -1;
  }
  return bem_launch_pv_rows(S, d, dG, dH, dF, P, dP, pv, tpv, 0, n, st);
}

extern "C" int bem_launch_pv_rows(const bem_sys_dev *S, int d, const double *dG, const double *dH, const double *dF,
                                  const double *P, const double *dP, double *pv, double *tpv, int p0, int np,
                                  cudaStream_t st) {
  if (np <= 0) return 0;
  k_pv_interior<<<(np + 7) / 8, 256, 0, st>>>(*S, d, dG, dH, dF, P, dP, pv, tpv, p0, np);
  bem_count_launches(1);
  return cudaPeekAtLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int bem_launch_dpv_rhs(int Nd, const double *H, const double *pv, double *B, cudaStream_t st) {
  if (Nd == 0) return 0;
  k_dpv_rhs<<<(Nd + 7) / 8, 256, 0, st>>>(Nd, H, pv, B);
  bem_count_launches(1);
  return cudaPeekAtLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int bem_launch_dpv_store(int Nd, const double *B, double *dpv, cudaStream_t st) {
  if (Nd == 0) return 0;
  k_dpv_store<<<(Nd + 127) / 128, 128, 0, st>>>(Nd, B, dpv);
  bem_count_launches(1);
  return cudaPeekAtLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int bem_launch_compress(const double *G, int N, const int *inv, int nn, double *Gc, cudaStream_t st) {
  const long long n2 = (long long)nn * nn;
  if (n2 == 0) return 0;
  k_compress_mat<<<(unsigned)((n2 + 255) / 256), 256, 0, st>>>(G, N, inv, nn, Gc);
  bem_count_launches(1);
  return cudaPeekAtLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int bem_launch_rows(const double *src, double *dst, int N, const int *inv, int nn, int nrhs, int to_full,
                               cudaStream_t st) {
  if (to_full) {
    k_move_rows<<<(N + 127) / 128, 128, 0, st>>>(src, dst, N, inv, nn, nrhs, 1);
    bem_count_launches(1);
    k_scatter_rows<<<(nn + 127) / 128, 128, 0, st>>>(src, dst, N, inv, nn, nrhs);
    bem_count_launches(1);
  } else {
    k_move_rows<<<(nn + 127) / 128, 128, 0, st>>>(src, dst, N, inv, nn, nrhs, 0);
    bem_count_launches(1);
  }
  return cudaPeekAtLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int bem_launch_force0(const bem_sys_dev *S, const double *P0, const double *pv0, const double *rc, double c0,
                                 double rho0, const int *ctr, const double *cbd, const double *pw, double *out,
                                 cudaStream_t st) {
  k_force0<<<1, 256, 0, st>>>(*S, P0, pv0, rc, c0, rho0, ctr, cbd, pw, out);
  bem_count_launches(1);
  return cudaPeekAtLastError() == cudaSuccess ? 0 : -1;
}
