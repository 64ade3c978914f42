// Post-processing on the device: fields at points off the boundary and
// boundary values on the elements (for the 9-point radiation force).
// Included at the end of bem_assemble.cu so that it shares that file's
// constant tables (quadrature rules, Faddeeva constants).
//
// Field at a point r (pv_s_dbieq_aqd2 / pv_s_bieq_aqd2 / phi_s_aqd2,
// bem3_aw_qd2_field.c:3-297): for every source element of the point's domain
// the coefficients CC = (G[4], H[4], F) and their gradients with respect to r
// (q0_bil_dcoef_grad_*, q0_bil_dcoef_grad.c; bil_dcoef_grad_*, bil_dcoef_grad.c)
// are contracted at once with the element's boundary values, so one kernel
// returns per point
//   S0    = sum (G dP - H P)                     (phi before normalisation)
//   S1[j] = sum (dG/dr_j dP - dH/dr_j P)         (grad phi before normalisation)
//   F, dF[j]                                     (solid-angle term and gradient)
//   S2[j] = sum (G dpv_j - H pv_j)               (near-boundary velocity)
// The host applies the reference's normalisation, near-boundary switch and
// Bloch phase.  Rules: type 0 4 nodes, 1 9-point, 2 12x12 GL, 3 64x64 GL.
#pragma once

#define FIELD_THREADS 128

struct fld_acc { double s0r, s0i, s1[6], f, df[3], s2[6]; };  // 18 doubles

// rule point idx of a source element: parameter point, weight, node flag
__device__ __forceinline__ int rule_points(int type) {
  return type == 0 ? 4 : (type == 1 ? 9 : (type == 2 ? BEM_GLN * BEM_GLN : BEM_GHN * BEM_GHN));
}

__device__ __forceinline__ void rule_point(int type, int i, double &z, double &e, double &w) {
  if (type == 0) { z = c_q.zt[i]; e = c_q.et[i]; w = 1.0; }
  else if (type == 1) { z = c_q.z9[i]; e = c_q.e9[i]; w = c_q.w9[i]; }
  else if (type == 2) { z = c_q.xl[i / BEM_GLN]; e = c_q.xl[i % BEM_GLN]; w = c_q.wl[i / BEM_GLN] * c_q.wl[i % BEM_GLN]; }
  else { z = c_q.xh[i / BEM_GHN]; e = c_q.xh[i % BEM_GHN]; w = c_q.wh[i / BEM_GHN] * c_q.wh[i % BEM_GHN]; }
}

// Rules on a triangle source (q0_lit_coef_4p / _7p / _GL / _GH, q0_lit_coef.c:10-250):
// type 0: the 3 nodes and the centre (weights 25/48 x 3, -27/48), 1: 7-point rule,
// 2, 3: the 3-part 12 x 12 / 64 x 64 rules.  w multiplies W = cw0 (twice the area).
__device__ __forceinline__ int tri_rule_points(int type) {
  return type == 0 ? 4 : (type == 1 ? 7 : 3 * (type == 2 ? BEM_GLN * BEM_GLN : BEM_GHN * BEM_GHN));
}
__device__ __forceinline__ void tri_rule_point(int type, int i, double &z, double &e, double &w) {
  if (type == 0) {
    if (i < 3) bem_tri_node(i, z, e);
    else z = e = 0.0;
    w = 0.5 * (i < 3 ? 25.0 / 48.0 : -27.0 / 48.0);
  } else if (type == 1) {
    // the 7-point rule (zt_37, et_37, wt_37, bem3_aw_qd2.c:1012-1021)
    const double n0 = 0.3480702390148154917985, n1 = 0.2052130961576726346557;
    const double n2 = 0.6028753385763033130539, n3 = 0.3554395089236065568357;
    const double v0 = 0.1259391805448271525957, v1 = 0.1323941527885061807376, v2 = 0.225;
    const double zz[7] = {-n0, 2.0 * n0, -n0, n1, -2.0 * n1, n1, 0.0}, ee[7] = {-n2, 0.0, n2, n3, 0.0, -n3, 0.0};
    z = zz[i];
    e = ee[i];
    w = 0.5 * (i < 3 ? v0 : (i < 6 ? v1 : v2));
  } else {
    const int n = type == 2 ? BEM_GLN : BEM_GHN;
    const double *x = type == 2 ? c_q.xl : c_q.xh, *wq = type == 2 ? c_q.wl : c_q.wh;
    const int part = i / (n * n), ij = i % (n * n), a = ij / n, b = ij % n;
    bem_tri_point(part, x[a], x[b], z, e);
    w = wq[a] * wq[b] * bem_tri_wfac(x[a], x[b]);
  }
}

// boundary values of source element s interpolated at (z,e); type 0 uses the
// node value itself (the 4-point rule sits on the nodes; the triangle's centre
// point takes the mean of its 3 nodes)
__device__ __forceinline__ void interp_bv(int type, int i, double z, double e, int s, const double *P, const double *dP,
                                          const double *pv, const double *dpv, cplx &Pn, cplx &dPn, cplx pvn[3],
                                          cplx dpvn[3], bool tri = false) {
  double N[4];
  if (type == 0 && !(tri && i == 3)) {
    for (int a = 0; a < 4; ++a) N[a] = a == i ? 1.0 : 0.0;
  } else {
    bem_Nn(tri, z, e, N);
  }
  Pn = dPn = cmk(0, 0);
  for (int c = 0; c < 3; ++c) pvn[c] = dpvn[c] = cmk(0, 0);
  for (int a = 0; a < 4; ++a) {
    const size_t o = (size_t)s * 4 + a;
    Pn = cadd(Pn, cscale(cmk(P[2 * o], P[2 * o + 1]), N[a]));
    dPn = cadd(dPn, cscale(cmk(dP[2 * o], dP[2 * o + 1]), N[a]));
    for (int c = 0; c < 3; ++c) {
      pvn[c] = cadd(pvn[c], cscale(cmk(pv[2 * (3 * o + c)], pv[2 * (3 * o + c) + 1]), N[a]));
      dpvn[c] = cadd(dpvn[c], cscale(cmk(dpv[2 * (3 * o + c)], dpv[2 * (3 * o + c) + 1]), N[a]));
    }
  }
}

template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double *sm /* NV*(FIELD_THREADS/32) + NV */) {
#pragma unroll
  for (int c = 0; c < NV; ++c) {
    double x = v[c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0) sm[c * (FIELD_THREADS / 32) + (threadIdx.x >> 5)] = x;
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    double x = 0.0;
    for (int w = 0; w < FIELD_THREADS / 32; ++w) x += sm[threadIdx.x * (FIELD_THREADS / 32) + w];
    sm[NV * (FIELD_THREADS / 32) + threadIdx.x] = x;
  }
  __syncthreads();
#pragma unroll
  for (int c = 0; c < NV; ++c) v[c] = sm[NV * (FIELD_THREADS / 32) + c];
  __syncthreads();
}

// one block per field point; threads over (source element, rule point)
// grad = 1: S1 and dF with the second-derivative Green's function (q0_dcoef_rt_grad,
// d3hm_qpgf_d2_v2); 0: the potential sums S0, S2, F alone with the
// first-derivative one (q0_coef_rt, d3hm_qpgf_d2_v1), as phi_s_aqd2 and
// pv_s_bieq_aqd2 form them: the two lattice sums stop differently next to
// the lattice plane, so each caller gets the one the reference uses.
__global__ void __launch_bounds__(FIELD_THREADS) k_field(bem_dom_dev D, const __grid_constant__ bem_qp q, int periodic, int grad, double k, int type,
                                                         const double *__restrict__ pts, const double *__restrict__ P,
                                                         const double *__restrict__ dP, const double *__restrict__ pv,
                                                         const double *__restrict__ dpv, double *__restrict__ out,
                                                         unsigned *status) {
  const int ip = blockIdx.x;
  const double rt[3] = {pts[3 * ip], pts[3 * ip + 1], pts[3 * ip + 2]};
  const int nr = D.has_tri ? max(rule_points(type), tri_rule_points(type)) : rule_points(type);
  double a[18];
#pragma unroll
  for (int c = 0; c < 18; ++c) a[c] = 0.0;
  unsigned st = 0;
  for (long long it = threadIdx.x; it < (long long)D.ne * nr; it += FIELD_THREADS) {
    const int s = (int)(it / nr), i = (int)(it % nr);
    const int se = abs(D.sid[s]) - 1;
    // triangle sources: q0_lit_dcoef_grad_* / lit_dcoef_grad_* (q0_lit_dcoef_grad.c, lit_dcoef_grad.c)
    const bool stri = D.has_tri && D.npe[se] == 3;
    if (i >= (stri ? tri_rule_points(type) : rule_points(type))) continue;
    const double sg = D.sid[s] < 0 ? -1.0 : 1.0;
    double z, e, w, vR[3], vW[3];
    if (stri) tri_rule_point(type, i, z, e, w);
    else rule_point(type, i, z, e, w);
    if (type == 0) {  // the rule's points are the ren entries (a triangle's centre is its 4th)
      for (int d = 0; d < 3; ++d) {
        vR[d] = __ldg(D.ren + (size_t)se * 12 + i * 3 + d);
        vW[d] = __ldg(D.wen + (size_t)se * 12 + i * 3 + d);
      }
    } else {
      bem_el el;
      bem_load_el(D.cr, D.cw, se, el);
      bem_rw_ref(el, z, e, vR, vW);
    }
    for (int d = 0; d < 3; ++d) vR[d] = __dsub_rn(vR[d], rt[d]);
    const double aR = sqrt(dot3(vR, vR)), iR = 1.0 / aR;
    const double aW = sqrt(dot3(vW, vW));
    const double rdW = dot3(vR, vW) * iR;
    cplx Pn, dPn, pvn[3], dpvn[3];
    interp_bv(type, i, z, e, s, P, dP, pv, dpv, Pn, dPn, pvn, dpvn, stri);
    cplx G, H, dG[3], dH[3];
    if (periodic && !grad) {
      bem_gval gv;
      const int rc = bem_qpgf(q, vR[0], vR[1], vR[2], gv);
      if (rc < 0) st |= (rc == -12 || rc == -23) ? BEM_ST_RAYLEIGH : BEM_ST_QPGF_LIMIT;
      G = cscale(gv.g, aW);
      H = cadd(cadd(cscale(gv.gx, vW[0]), cscale(gv.gy, vW[1])), cscale(gv.gz, vW[2]));
      for (int j = 0; j < 3; ++j) dG[j] = dH[j] = cmk(0.0, 0.0);
    } else if (periodic) {
      bem_gval2 gv;
      const int rc = bem_qpgf2(q, vR[0], vR[1], vR[2], gv);
      if (rc < 0) st |= (rc == -12 || rc == -23) ? BEM_ST_RAYLEIGH : BEM_ST_QPGF_LIMIT;
      G = cscale(gv.g, aW);
      H = cadd(cadd(cscale(gv.d[0], vW[0]), cscale(gv.d[1], vW[1])), cscale(gv.d[2], vW[2]));
      // d/d rt = -d/d R; second derivatives ordered xx, yy, zz, xy, yz, zx
      const cplx *d2 = gv.d2;
      const cplx hx = cadd(cadd(cscale(d2[0], vW[0]), cscale(d2[3], vW[1])), cscale(d2[5], vW[2]));
      const cplx hy = cadd(cadd(cscale(d2[3], vW[0]), cscale(d2[1], vW[1])), cscale(d2[4], vW[2]));
      const cplx hz = cadd(cadd(cscale(d2[5], vW[0]), cscale(d2[4], vW[1])), cscale(d2[2], vW[2]));
      for (int j = 0; j < 3; ++j) dG[j] = cscale(gv.d[j], -aW);
      dH[0] = cscale(hx, -1.0);
      dH[1] = cscale(hy, -1.0);
      dH[2] = cscale(hz, -1.0);
    } else {
      // free space (bil_dcoef_grad_*): G = e^{ikR}/(4 pi R) |W|, H = (ikR-1) e^{ikR} (R.W)/(4 pi R^3)
      const cplx ce = cexpi(k * aR), cb = cmk(-1.0, k * aR), cbce = cmul(cb, ce);
      const double tD = rdW * iR * iR, i3 = iR * iR * iR;
      G = cscale(ce, BEM_I_FP * iR * aW);
      H = cscale(cbce, sg * BEM_I_FP * tD);
      const cplx kk3 = cmk(k * k * aR * aR + 3.0 * cb.re, 3.0 * cb.im);
      for (int j = 0; j < 3; ++j) {
        const double rj = vR[j] * iR;
        dG[j] = cscale(cbce, -BEM_I_FP * iR * iR * rj * aW);
        dH[j] = cscale(cmul(ce, csub(cscale(kk3, rj * rdW), cscale(cb, vW[j]))), sg * BEM_I_FP * i3);
      }
    }
    const cplx t0 = csub(cmul(G, dPn), cmul(H, Pn));
    a[0] += w * t0.re;
    a[1] += w * t0.im;
    for (int j = 0; j < 3; ++j) {
      const cplx t1 = csub(cmul(dG[j], dPn), cmul(dH[j], Pn));
      a[2 + 2 * j] += w * t1.re;
      a[3 + 2 * j] += w * t1.im;
      const cplx t2 = csub(cmul(G, dpvn[j]), cmul(H, pvn[j]));
      a[12 + 2 * j] += w * t2.re;
      a[13 + 2 * j] += w * t2.im;
    }
    const double i3 = iR * iR * iR;
    a[8] += sg * w * rdW * iR * iR;
    for (int j = 0; j < 3; ++j) a[9 + j] += sg * w * i3 * (3.0 * vR[j] * iR * rdW - vW[j]);
  }
  set_status(status, st);
  __shared__ double sm[18 * (FIELD_THREADS / 32) + 18];
  block_sum<18>(a, sm);
  if (threadIdx.x < 18) {
    double v = a[threadIdx.x];
    if (threadIdx.x >= 8 && threadIdx.x < 12) v *= BEM_I_FP;  // F and dF carry 1/4pi
    out[18 * (size_t)ip + threadIdx.x] = v;
  }
}

// Boundary sums of one domain at parameter points (z,e) of its elements
// (pv_s_bd_aqd2, bem3_aw_qd2_field.c:394-433): regular sources with the chosen
// rule, the element itself with the singular polar rule.  periodic = 1: the
// host domain with the quasi-periodic Green's function (q0_coef_bd,
// d3qd2_elem.c:684, self pair q0_bil_coef_bd); 0: an interior domain in free
// space with wave number k (coef_bd, d3qd2_elem.c:187, self pair bil_coef_bd,
// bil_coef.c:244-342).  out per target: S0 (2), S2 (6), F.
__global__ void __launch_bounds__(FIELD_THREADS) k_bdval(bem_dom_dev D, const __grid_constant__ bem_qp q, int periodic, double k, int type,
                                                         const int *__restrict__ tgt_t,
                                                         const double *__restrict__ tgt_ze, const double *__restrict__ P,
                                                         const double *__restrict__ dP, const double *__restrict__ pv,
                                                         const double *__restrict__ dpv, double *__restrict__ out,
                                                         unsigned *status) {
  const int ip = blockIdx.x;
  const int t = tgt_t[ip];
  const double zt = tgt_ze[2 * ip], et = tgt_ze[2 * ip + 1];
  const int te = abs(D.sid[t]) - 1;
  bem_el elt;
  bem_load_el(D.cr, D.cw, te, elt);
  double rt[3], wt_[3];
  bem_rw_ref(elt, zt, et, rt, wt_);
  const int nr = D.has_tri ? max(rule_points(type), tri_rule_points(type)) : rule_points(type);
  double a[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) a[c] = 0.0;
  unsigned st = 0;
  // regular sources
  for (long long it = threadIdx.x; it < (long long)D.ne * nr; it += FIELD_THREADS) {
    const int s = (int)(it / nr), i = (int)(it % nr);
    const int se = abs(D.sid[s]) - 1;
    if (s == t) continue;
    const bool stri = D.has_tri && D.npe[se] == 3;
    if (i >= (stri ? tri_rule_points(type) : rule_points(type))) continue;
    const double sg = D.sid[s] < 0 ? -1.0 : 1.0;
    double z, e, w, vR[3], vW[3];
    if (stri) tri_rule_point(type, i, z, e, w);
    else rule_point(type, i, z, e, w);
    if (type == 0 && !(stri && i == 3)) {
      for (int d = 0; d < 3; ++d) {
        vR[d] = __ldg(D.ren + (size_t)se * 12 + i * 3 + d);
        vW[d] = __ldg(D.wen + (size_t)se * 12 + i * 3 + d);
      }
    } else {
      bem_el el;
      bem_load_el(D.cr, D.cw, se, el);
      bem_rw_ref(el, z, e, vR, vW);
    }
    for (int d = 0; d < 3; ++d) vR[d] = __dsub_rn(vR[d], rt[d]);
    const double aR = sqrt(dot3(vR, vR)), iR = 1.0 / aR;
    const double aW = sqrt(dot3(vW, vW));
    const double tD = dot3(vR, vW) * iR * iR * iR;
    cplx G, H;
    if (periodic) {
      bem_gval gv;
      const int rc = bem_qpgf(q, vR[0], vR[1], vR[2], gv);
      if (rc < 0) st |= (rc == -12 || rc == -23) ? BEM_ST_RAYLEIGH : BEM_ST_QPGF_LIMIT;
      G = cscale(gv.g, aW);
      H = cadd(cadd(cscale(gv.gx, vW[0]), cscale(gv.gy, vW[1])), cscale(gv.gz, vW[2]));
    } else {
      // bil_coef_4p / _9p / _GL / _GH (bil_coef.c:24-243)
      const cplx ce = cexpi(k * aR);
      G = cscale(ce, BEM_I_FP * iR * aW);
      H = cscale(cmul(cmk(-1.0, k * aR), ce), sg * BEM_I_FP * tD);
    }
    cplx Pn, dPn, pvn[3], dpvn[3];
    interp_bv(type, i, z, e, s, P, dP, pv, dpv, Pn, dPn, pvn, dpvn, stri);
    const cplx t0 = csub(cmul(G, dPn), cmul(H, Pn));
    a[0] += w * t0.re;
    a[1] += w * t0.im;
    for (int j = 0; j < 3; ++j) {
      const cplx t2 = csub(cmul(G, dpvn[j]), cmul(H, pvn[j]));
      a[2 + 2 * j] += w * t2.re;
      a[3 + 2 * j] += w * t2.im;
    }
    a[8] += sg * w * tD * BEM_I_FP;
  }
  // the element itself: polar rule around (zt, et); a triangle has 3 sub-triangles
  // and the constant Jacobian vector cw0 2 / (3 sqrt3) (q0_lit_coef_bd, lit_coef_bd)
  const bool ttri = D.has_tri && D.npe[te] == 3;
  double r[5], th[5];
  if (ttri) bem_tri_node_r_th(zt, et, r, th);
  else bem_node_r_th(zt, et, r, th);
  const bool plane = D.plane[te] != 0;
  const double sgt = D.sid[t] < 0 ? -1.0 : 1.0, bdC = bem_bdC(elt);
  for (int pt = threadIdx.x; pt < (ttri ? 384 : 512) * BEM_GLN; pt += FIELD_THREADS) {
    const int idx = pt / BEM_GLN, ir = pt % BEM_GLN;
    const polar_pt tp = polar_theta(th, idx);
    const double rm = bem_rmax(r[tp.j], r[tp.j + 1], th[tp.j], th[tp.j + 1], tp.th);
    if (rm < 0.0) st |= BEM_ST_GEOMETRY;
    double sth, cth;
    sincos(tp.th, &sth, &cth);
    const double rr = 0.5 * rm * (c_q.xl[ir] + 1.0);
    const double w = tp.wth * 0.5 * rm * c_q.wl[ir] * rr;
    const double z = rr * cth + zt, e = rr * sth + et;
    double K[3], vR[3], vW[3];
    bem_K(elt, rr, cth, sth, zt, et, K);
    for (int d = 0; d < 3; ++d) {
      vR[d] = rr * K[d];
      vW[d] = ttri ? elt.cw[d][0] * (2.0 / (3.0 * BEM_SQ3)) : elt.cw[d][0] + elt.cw[d][1] * z + elt.cw[d][2] * e;
    }
    const double aW = sqrt(dot3(vW, vW));
    cplx G, H;
    if (periodic) {
      bem_gval gv;
      const int rc = bem_qpgf(q, vR[0], vR[1], vR[2], gv);
      if (rc < 0) st |= (rc == -12 || rc == -23) ? BEM_ST_RAYLEIGH : BEM_ST_QPGF_LIMIT;
      G = cscale(gv.g, aW);
      H = cadd(cadd(cscale(gv.gx, vW[0]), cscale(gv.gy, vW[1])), cscale(gv.gz, vW[2]));
    } else {
      // bil_sG_r, bil_sH_r (lit_sG_r) with the Jacobian rr of the polar map taken out of w
      const double aK = sqrt(dot3(K, K)), kR = k * aK * rr;
      const cplx ce = cexpi(kR);
      G = cscale(ce, BEM_I_FP * aW / (aK * rr));
      H = plane ? cmk(0.0, 0.0)
                : cscale(cmul(cmk(-1.0, kR), ce), sgt * BEM_I_FP * bdC * cth * sth / (aK * aK * aK * rr));
    }
    cplx Pn, dPn, pvn[3], dpvn[3];
    interp_bv(1, 0, z, e, t, P, dP, pv, dpv, Pn, dPn, pvn, dpvn, ttri);
    const cplx t0 = csub(cmul(G, dPn), cmul(H, Pn));
    a[0] += w * t0.re;
    a[1] += w * t0.im;
    for (int j = 0; j < 3; ++j) {
      const cplx t2 = csub(cmul(G, dpvn[j]), cmul(H, pvn[j]));
      a[2 + 2 * j] += w * t2.re;
      a[3 + 2 * j] += w * t2.im;
    }
  }
  // the element's own F (geometric polar rule, zero for plane elements)
  if (!plane) a[8] += sgt * polar_F_partial(elt, zt, et, st) * BEM_I_FP * bdC;
  set_status(status, st);
  __shared__ double sm[9 * (FIELD_THREADS / 32) + 9];
  block_sum<9>(a, sm);
  if (threadIdx.x < 9) out[9 * (size_t)ip + threadIdx.x] = a[threadIdx.x];
}

// Radiation force and torque from boundary values at the rule points of the
// domain-0 elements (bil_force_9p, bem3_aw_qd2_force.c:122-165): one block.
__global__ void k_force_bd(bem_dom_dev D, int ntgt, const int *__restrict__ tgt_t, const double *__restrict__ tgt_ze,
                           const double *__restrict__ wts, const double *__restrict__ bdv, const double *__restrict__ pw,
                           double k2r, double k2i, const double *rc, double c0, double rho0, double *__restrict__ out) {
  // pw: amplitude (re, im), R[9], tv[3], k0, rho0 c0
  const double c1 = 0.25 / (c0 * c0 * rho0), c2 = 0.25 * rho0, c3 = 0.5 * rho0;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int ip = threadIdx.x; ip < ntgt; ip += blockDim.x) {
    const int te = abs(D.sid[tgt_t[ip]]) - 1;
    bem_el el;
    bem_load_el(D.cr, D.cw, te, el);
    double r[3], w[3];
    bem_rw_ref(el, tgt_ze[2 * ip], tgt_ze[2 * ip + 1], r, w);
    const double *b = bdv + 9 * (size_t)ip;
    const double cf = 1.0 / (1.0 + b[8]);
    // incident plane wave at r (calc_apw_pv, aw_pw.c:129-157)
    const double *R = pw + 2;
    const double rcx = r[0] - pw[11], rcy = r[1] - pw[12], rcz = r[2] - pw[13];
    const double r0z = -R[6] * rcx - R[7] * rcy + R[8] * rcz;
    const cplx pinc = cmul(cmk(pw[0], pw[1]), cexpi(pw[14] * r0z));
    const cplx vz = cscale(pinc, 1.0 / pw[15]);
    // p = -k2 S0 / (1+F) + p_inc;  v = S2 / (1+F) + v_inc
    const cplx S0 = cmk(b[0] * cf, b[1] * cf);
    const cplx p = cadd(cscale(cmul(cmk(k2r, k2i), S0), -1.0), pinc);
    cplx v[3];
    for (int l = 0; l < 3; ++l) v[l] = cadd(cmk(b[2 + 2 * l] * cf, b[3 + 2 * l] * cf), cscale(vz, R[l * 3 + 2]));
    const double t1 = c1 * (p.re * p.re + p.im * p.im) -
                      c2 * (v[0].re * v[0].re + v[0].im * v[0].im + v[1].re * v[1].re + v[1].im * v[1].im +
                            v[2].re * v[2].re + v[2].im * v[2].im);
    double T[9];
    for (int l = 0; l < 3; ++l)
      for (int m = 0; m < 3; ++m) T[l * 3 + m] = c3 * (v[l].re * v[m].re + v[l].im * v[m].im);
    T[0] += t1; T[4] += t1; T[8] += t1;
    double Tw[3];
    for (int l = 0; l < 3; ++l) Tw[l] = (T[l * 3] * w[0] + T[l * 3 + 1] * w[1] + T[l * 3 + 2] * w[2]) * wts[ip];
    for (int l = 0; l < 3; ++l) acc[l] += Tw[l];
    const double dx = r[0] - rc[0], dy = r[1] - rc[1], dz = r[2] - rc[2];
    acc[3] += dy * Tw[2] - dz * Tw[1];
    acc[4] += dz * Tw[0] - dx * Tw[2];
    acc[5] += dx * Tw[1] - dy * Tw[0];
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

extern "C" int bem_launch_field(const bem_dom_dev *D, const bem_qp *q, int periodic, int grad, double k, int type,
                                int npts, const double *pts, const double *P, const double *dP, const double *pv,
                                const double *dpv, double *out, unsigned *status, cudaStream_t st) {
  if (npts <= 0) return 0;
  k_field<<<npts, FIELD_THREADS, 0, st>>>(*D, *q, periodic, grad, k, type, pts, P, dP, pv, dpv, out, status);
  return cudaPeekAtLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int bem_launch_bdval(const bem_dom_dev *D, const bem_qp *q, int periodic, double k, int type, int ntgt,
                                const int *tgt_t,
                                const double *tgt_ze, const double *P, const double *dP, const double *pv,
                                const double *dpv, double *out, unsigned *status, cudaStream_t st) {
  if (ntgt <= 0) return 0;
  k_bdval<<<ntgt, FIELD_THREADS, 0, st>>>(*D, *q, periodic, k, type, tgt_t, tgt_ze, P, dP, pv, dpv, out, status);
  return cudaPeekAtLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int bem_launch_force_bd(const bem_dom_dev *D, int ntgt, const int *tgt_t, const double *tgt_ze,
                                   const double *wts, const double *bdv, const double *pw, double k2r, double k2i,
                                   const double *rc, double c0, double rho0, double *out, cudaStream_t st) {
  k_force_bd<<<1, 256, 0, st>>>(*D, ntgt, tgt_t, tgt_ze, wts, bdv, pw, k2r, k2i, rc, c0, rho0, out);
  return cudaPeekAtLastError() == cudaSuccess ? 0 : -1;
}
