// Element geometry and quadrature tables on the device.
//
// Bilinear element (d3qd2_src/d3qd2_elem.c:890-1028):
//   r(z,e) = cr0 + cr1 z + cr2 e + cr3 z e,  W(z,e) = cw0 + cw1 z + cw2 e
//   interpolation functions with nodes at (+-1/sqrt3, +-1/sqrt3)  (bil_Nn, :903)
#pragma once
#include <cuda_runtime.h>

#define BEM_GLN 12
#define BEM_GHN 64
#define BEM_CBD_SDF 0.5        // near-singular switch on |dF/dt|   (d3qd2_const.h:80)
#define BEM_CDFH 1.0e-3        // central-difference step           (d3qd2_const.h:35)
#define BEM_DEPS 0.1           // radius of the PV disc D_eps        (d3qd2_const.h:34)
#define BEM_I_FP 7.957747154594766788444e-2  // 1/(4 pi)
#define BEM_P44 0.5773502691896257645091     // 1/sqrt(3)
#define BEM_MAXNEAR 256        // most near-singular sources a collocation node can hold (bem_dom_dev.near_cap)

// Shorter rules of the periodic domain's regular pairs (k_q0_far): tier t is
// the (BEM_TIER_N0 - t)-point Gauss-Legendre rule, t = 0 .. BEM_NTIER - 1
// (10, 9, 8, 7 and 6 points)
#define BEM_NTIER 5
#define BEM_TIER_N0 10
struct bem_quad {
  double xl[BEM_GLN], wl[BEM_GLN];
  double xt[BEM_NTIER][BEM_TIER_N0], wt[BEM_NTIER][BEM_TIER_N0];
  double xh[BEM_GHN], wh[BEM_GHN];
  double zt[4], et[4];        // collocation node parameters (zt_44, et_44)
  double z9[9], e9[9], w9[9]; // 9-point rule (zt_49, et_49, wt_49)
};
static __constant__ bem_quad c_q;  // one copy per translation unit

// element constants of element e (0-based), 21 doubles
struct bem_el { double cr[3][4]; double cw[3][3]; };

__device__ __forceinline__ void bem_load_el(const double *__restrict__ cr, const double *__restrict__ cw, int e, bem_el &el) {
#pragma unroll
  for (int d = 0; d < 3; ++d) {
#pragma unroll
    for (int c = 0; c < 4; ++c) el.cr[d][c] = __ldg(cr + (size_t)e * 12 + d * 4 + c);
#pragma unroll
    for (int c = 0; c < 3; ++c) el.cw[d][c] = __ldg(cw + (size_t)e * 9 + d * 3 + c);
  }
}

// interpolation function N_n(z,e) (bil_Nn)
__device__ __forceinline__ void bem_Nn4(double z, double e, double N[4]) {
  const double ia = 1.0 / BEM_P44;
  const double zm = 1.0 - z * ia, zp = 1.0 + z * ia, em = 1.0 - e * ia, ep = 1.0 + e * ia;
  N[0] = 0.25 * zm * em;
  N[1] = 0.25 * zp * em;
  N[2] = 0.25 * zp * ep;
  N[3] = 0.25 * zm * ep;
}

__device__ __forceinline__ void bem_rw(const bem_el &el, double z, double e, double r[3], double w[3]) {
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    r[d] = el.cr[d][0] + el.cr[d][1] * z + el.cr[d][2] * e + el.cr[d][3] * z * e;
    w[d] = el.cw[d][0] + el.cw[d][1] * z + el.cw[d][2] * e;
  }
}

// The same point with every product and sum rounded separately, in the
// reference's order ((cr0 + cr1 z) + cr2 e) + (cr3 z) e (bil_rw_zeta_eta,
// d3qd2_elem.c:963, r_bd, :18, compiled without fused multiply-add).  The
// boundary-value sums use it so that R = r_s - r_t is bit-identical to the
// reference's: on mirror-symmetric meshes R_z is then exactly 0 where the
// reference's is, and the lattice sums take the same stopping decisions
// (an identically zero z-derivative sum ends the spectral rows at once).
__device__ __forceinline__ void bem_rw_ref(const bem_el &el, double z, double e, double r[3], double w[3]) {
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    r[d] = __dadd_rn(__dadd_rn(__dadd_rn(el.cr[d][0], __dmul_rn(el.cr[d][1], z)), __dmul_rn(el.cr[d][2], e)),
                     __dmul_rn(__dmul_rn(el.cr[d][3], z), e));
    w[d] = el.cw[d][0] + el.cw[d][1] * z + el.cw[d][2] * e;
  }
}

// ---- linear triangles (d3qd2_elem.c:1035-1162): reference triangle with corners
// (-1/2, -sqrt3/2), (1, 0), (-1/2, sqrt3/2); r(z,e) = cr0 + cr1 z + cr2 e
// (cr3 = 0), W = cw0 constant (cw1 = cw2 = 0), so bem_rw, bem_K serve both types.
#define BEM_SQ3 1.732050807568877293528
#define BEM_P34_N0 0.2                       // collocation nodes (-N0,-N1), (2 N0, 0), (-N0, N1)
#define BEM_P34_N1 0.3464101615137754587055

// interpolation functions N_n(z,e), n = 0..2; N[3] = 0 (lit_Nn, d3qd2_elem.c:1047)
__device__ __forceinline__ void bem_Nn3(double z, double e, double N[4]) {
  const double ia = 0.5 / BEM_P34_N0;
  N[0] = (1.0 / 3.0) * (1.0 - ia * (z + BEM_SQ3 * e));
  N[1] = (1.0 / 3.0) * (1.0 + 2.0 * ia * z);
  N[2] = (1.0 / 3.0) * (1.0 - ia * (z - BEM_SQ3 * e));
  N[3] = 0.0;
}
__device__ __forceinline__ void bem_Nn(bool tri, double z, double e, double N[4]) {
  if (tri) bem_Nn3(z, e, N);
  else bem_Nn4(z, e, N);
}
// twice the derivative of N_n along the direction (c, s), the radial factor of the
// principal-value D-eps integrals (lit_dNn_pr_cs, lit_dcoef.c:845)
__device__ __forceinline__ void bem_dNn3(double c, double s, double dN[4]) {
  const double ia = 0.5 / BEM_P34_N0;
  dN[0] = -2.0 / 3.0 * ia * (c + BEM_SQ3 * s);
  dN[1] = 4.0 / 3.0 * ia * c;
  dN[2] = -2.0 / 3.0 * ia * (c - BEM_SQ3 * s);
  dN[3] = 0.0;
}
// The triangle's product Gauss rule (q0_lit_dcoef_v2_cc_GL, q0_lit_dcoef_v2_cc.c:191-219): the
// triangle is cut into 3 quadrilaterals (a vertex, two edge midpoints, the centroid), each
// mapped from [-1,1]^2; point (a, b) of part `part`, Jacobian factor 1 + a/4 + b/4.
__device__ __forceinline__ void bem_tri_point(int part, double a, double b, double &z, double &e) {
  if (part == 0) {
    z = 0.125 * (3.0 + 2.0 * a + 2.0 * b + a * b);
    e = 0.125 * BEM_SQ3 * (-a + b);
  } else if (part == 1) {
    z = 0.0625 * (-3.0 + a - 5.0 * b - a * b);
    e = 0.0625 * BEM_SQ3 * (3.0 + 3.0 * a + b + a * b);
  } else {
    z = 0.0625 * (-3.0 - 5.0 * a + b - a * b);
    e = 0.0625 * BEM_SQ3 * (-3.0 - a - 3.0 * b - a * b);
  }
}
// The same point rounded as the reference rounds it (each operation separately, in
// its order), for the periodic sums whose lattice-plane stopping depends on exact zeros
__device__ __forceinline__ void bem_tri_point_ref(int part, double a, double b, double &z, double &e) {
  const double ab = __dmul_rn(a, b);
  if (part == 0) {
    z = __dmul_rn(0.125, __dadd_rn(__dadd_rn(__dadd_rn(3.0, __dmul_rn(2.0, a)), __dmul_rn(2.0, b)), ab));
    e = __dmul_rn(0.125 * BEM_SQ3, __dadd_rn(-a, b));
  } else if (part == 1) {
    z = __dmul_rn(0.0625, __dadd_rn(__dadd_rn(__dadd_rn(-3.0, a), -__dmul_rn(5.0, b)), -ab));
    e = __dmul_rn(0.0625 * BEM_SQ3, __dadd_rn(__dadd_rn(__dadd_rn(3.0, __dmul_rn(3.0, a)), b), ab));
  } else {
    z = __dmul_rn(0.0625, __dadd_rn(__dadd_rn(__dadd_rn(-3.0, -__dmul_rn(5.0, a)), b), -ab));
    e = __dmul_rn(0.0625 * BEM_SQ3, __dadd_rn(__dadd_rn(__dadd_rn(-3.0, -a), -__dmul_rn(3.0, b)), -ab));
  }
}
// weight of point (a, b) relative to wl_a wl_b with W = cw0: the rule's total is
// |cw0| / 2, the triangle's area (the reference's 1/24 aW normalisation)
__device__ __forceinline__ double bem_tri_wfac(double a, double b) { return (1.0 + 0.25 * a + 0.25 * b) * (1.0 / 24.0); }
// collocation node tn of a triangle (zt_34, et_34)
__device__ __forceinline__ void bem_tri_node(int tn, double &z, double &e) {
  z = tn == 1 ? 2.0 * BEM_P34_N0 : -BEM_P34_N0;
  e = tn == 0 ? -BEM_P34_N1 : (tn == 2 ? BEM_P34_N1 : 0.0);
}
// corner distances and angles seen from (zt, et) (lit_calc_node_r_th, d3qd2_elem.c:1149)
__device__ __forceinline__ void bem_tri_node_r_th(double zt, double et, double r[5], double th[5]) {
  const double ztp = 1.0 - zt, ztm = -0.5 - zt, etp = 0.5 * BEM_SQ3 - et, etm = -0.5 * BEM_SQ3 - et;
  r[0] = sqrt(ztm * ztm + etm * etm);
  r[1] = sqrt(ztp * ztp + et * et);
  r[2] = sqrt(ztm * ztm + etp * etp);
  r[3] = r[0];
  r[4] = r[0];
  th[0] = atan2(etm, ztm);
  th[1] = atan2(-et, ztp);
  th[2] = atan2(etp, ztm);
  th[3] = th[0] + 2.0 * CUDART_PI;
  th[4] = th[3];
}

// corner distances and angles seen from (zt,et) (bil_calc_node_r_th, d3qd2_elem.c:1014)
__device__ __forceinline__ void bem_node_r_th(double zt, double et, double r[5], double th[5]) {
  const double ztp = 1.0 - zt, ztm = -1.0 - zt, etp = 1.0 - et, etm = -1.0 - et;
  r[0] = sqrt(ztm * ztm + etm * etm);
  r[1] = sqrt(ztp * ztp + etm * etm);
  r[2] = sqrt(ztp * ztp + etp * etp);
  r[3] = sqrt(ztm * ztm + etp * etp);
  r[4] = r[0];
  th[0] = atan2(etm, ztm);
  th[1] = atan2(etm, ztp);
  th[2] = atan2(etp, ztp);
  th[3] = atan2(etp, ztm);
  th[4] = th[0] + 2.0 * CUDART_PI;
}

// polar radius of the edge of sub-triangle (r0,th0)-(r1,th1) at angle th
__device__ __forceinline__ double bem_rmax(double r0, double r1, double th0, double th1, double th) {
  return r0 * r1 * sin(th1 - th0) / (r0 * sin(th - th0) - r1 * sin(th - th1));
}

// K(r,theta) = d r(zeta,eta) / d rho along the ray (the bracket in bil_sG_r, bil_coef.c:408)
__device__ __forceinline__ void bem_K(const bem_el &el, double rr, double cth, double sth, double zt, double et, double K[3]) {
  const double cross = rr * cth * sth + zt * sth + et * cth;
#pragma unroll
  for (int d = 0; d < 3; ++d) K[d] = el.cr[d][1] * cth + el.cr[d][2] * sth + el.cr[d][3] * cross;
}
