// Rotation and translation of the loaded body on the device, for serving
// requests that differ from a resident problem only in the body's placement:
// the reference's Rodrigues rotation and translation options of read_aqd2
// (bem3_aw_qd2.c:16-24, 395-422), which turn and move the mesh nodes before
// initialize_aqd2 builds the element constants (bem3_aw_qd2.c:941-1023) and
// the incident field at the collocation nodes (init_boundary_data,
// bem3_aw_qd2.c:1104-1146, with calc_apw_pv / calc_apw_dpdn, aw_pw.c:129-199).
//
// The element constants are linear in the nodes (position rows of cr and the
// collocation points ren) or, for the normal-vector constants cw and wen,
// cross products of node differences, which a rotation M maps to M times
// themselves (det M = 1).  So the kernel turns the resident constants instead
// of rebuilding them from nodes, which gives the reference's values to
// rounding, and evaluates the incident plane wave at the new collocation
// nodes with the formulas of calc_apw_pv / calc_apw_dpdn.  Whether an element
// is plane does not change under a rotation.
#include "bem_count.h"
#include <cuda_runtime.h>
#include <math.h>

struct bem_xform {
  double M[9], t[3];
};

// the incident plane wave (bemgpu_problem.pw: amplitude (re, im), wave
// rotation R[9], translation tv[3], k0, rho0 c0) at r: pressure p, particle
// velocity v and, for a unit normal nrm, dp/dn
__device__ static void plane_wave(const double *pw, const double *r, const double *nrm, double2 *p, double2 *v,
                                  double2 *dpdn) {
  const double *R = pw + 2, *tv = pw + 11;
  const double rc0 = r[0] - tv[0], rc1 = r[1] - tv[1], rc2 = r[2] - tv[2];
  // the reference applies the inverse wave rotation with this sign pattern (aw_pw.c:150-152)
  const double z = -R[6] * rc0 - R[7] * rc1 + R[8] * rc2;
  double s, c;
  sincos(pw[14] * z, &s, &c);
  const double2 pp = make_double2(pw[0] * c - pw[1] * s, pw[0] * s + pw[1] * c);
  *p = pp;
  const double2 vz = make_double2(pp.x / pw[15], pp.y / pw[15]);
  for (int i = 0; i < 3; ++i) v[i] = make_double2(R[3 * i + 2] * vz.x, R[3 * i + 2] * vz.y);
  const double n2 = -R[6] * nrm[0] - R[7] * nrm[1] + R[8] * nrm[2];
  // dp/dn = p i k0 n2
  *dpdn = make_double2(-pp.y * pw[14] * n2, pp.x * pw[14] * n2);
}

__global__ void k_transform(int ne, bem_xform X, double *cr, double *cw, double *ren, double *wen, double *Pi,
                            double *dPi, double *p_inc, double *v_inc, const double *pw, double2 cp) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  const double *M = X.M;
  // cr[e][d][j]: position row j = 0 turns and moves, rows 1..3 (directions) turn
  double a[3][4];
  for (int d = 0; d < 3; ++d)
    for (int j = 0; j < 4; ++j) a[d][j] = cr[(size_t)e * 12 + d * 4 + j];
  for (int d = 0; d < 3; ++d)
    for (int j = 0; j < 4; ++j)
      cr[(size_t)e * 12 + d * 4 + j] = M[3 * d] * a[0][j] + M[3 * d + 1] * a[1][j] + M[3 * d + 2] * a[2][j] +
                                       (j == 0 ? X.t[d] : 0.0);
  double b[3][3];
  for (int d = 0; d < 3; ++d)
    for (int j = 0; j < 3; ++j) b[d][j] = cw[(size_t)e * 9 + d * 3 + j];
  for (int d = 0; d < 3; ++d)
    for (int j = 0; j < 3; ++j)
      cw[(size_t)e * 9 + d * 3 + j] = M[3 * d] * b[0][j] + M[3 * d + 1] * b[1][j] + M[3 * d + 2] * b[2][j];
  for (int nd = 0; nd < 4; ++nd) {
    double *r = ren + (size_t)e * 12 + nd * 3, *w = wen + (size_t)e * 12 + nd * 3;
    const double r0 = r[0], r1 = r[1], r2 = r[2], w0 = w[0], w1 = w[1], w2 = w[2];
    double rn[3], wn[3];
    for (int d = 0; d < 3; ++d) {
      rn[d] = M[3 * d] * r0 + M[3 * d + 1] * r1 + M[3 * d + 2] * r2 + X.t[d];
      wn[d] = M[3 * d] * w0 + M[3 * d + 1] * w1 + M[3 * d + 2] * w2;
      r[d] = rn[d];
      w[d] = wn[d];
    }
    // incident data at the node: Pi = -p / k2, dPi = -dp/dn / k2 (unit normal),
    // p_inc, v_inc as calc_apw_pv
    const double aw = sqrt(wn[0] * wn[0] + wn[1] * wn[1] + wn[2] * wn[2]);
    if (aw != 0.0)
      for (int d = 0; d < 3; ++d) wn[d] /= aw;
    double2 p, v[3], dp;
    plane_wave(pw, rn, wn, &p, v, &dp);
    double *pi = Pi + (size_t)e * 8 + 2 * nd, *dpi = dPi + (size_t)e * 8 + 2 * nd;
    pi[0] = cp.x * p.x - cp.y * p.y;
    pi[1] = cp.x * p.y + cp.y * p.x;
    dpi[0] = cp.x * dp.x - cp.y * dp.y;
    dpi[1] = cp.x * dp.y + cp.y * dp.x;
    p_inc[(size_t)e * 8 + 2 * nd] = p.x;
    p_inc[(size_t)e * 8 + 2 * nd + 1] = p.y;
    for (int d = 0; d < 3; ++d) {
      v_inc[(size_t)e * 24 + nd * 6 + 2 * d] = v[d].x;
      v_inc[(size_t)e * 24 + nd * 6 + 2 * d + 1] = v[d].y;
    }
  }
}

// Rodrigues' rotation about rv by th (the reference's rotate option), then the
// launch; returns the CUDA error of the launch
extern "C" cudaError_t bem_launch_transform(int ne, const double *rv, double th, const double *tv, double *cr,
                                            double *cw, double *ren, double *wen, double *Pi, double *dPi,
                                            double *p_inc, double *v_inc, const double *pw_d, const double *k2,
                                            cudaStream_t st) {
  bem_xform X;
  double nv[3] = {rv[0], rv[1], rv[2]};
  const double an = sqrt(nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2]);
  if (an > 0.0)
    for (int i = 0; i < 3; ++i) nv[i] /= an;
  const double s = sin(th), c = cos(th), u = 1.0 - c;
  X.M[0] = c + nv[0] * nv[0] * u;
  X.M[1] = nv[0] * nv[1] * u - nv[2] * s;
  X.M[2] = nv[2] * nv[0] * u + nv[1] * s;
  X.M[3] = nv[0] * nv[1] * u + nv[2] * s;
  X.M[4] = c + nv[1] * nv[1] * u;
  X.M[5] = nv[1] * nv[2] * u - nv[0] * s;
  X.M[6] = nv[2] * nv[0] * u - nv[1] * s;
  X.M[7] = nv[1] * nv[2] * u + nv[0] * s;
  X.M[8] = c + nv[2] * nv[2] * u;
  for (int i = 0; i < 3; ++i) X.t[i] = tv[i];
  // cp = -1 / k2 of the host medium
  const double den = k2[0] * k2[0] + k2[1] * k2[1];
  const double2 cp = make_double2(-k2[0] / den, k2[1] / den);
  k_transform<<<(ne + 127) / 128, 128, 0, st>>>(ne, X, cr, cw, ren, wen, Pi, dPi, p_inc, v_inc, pw_d, cp);
  bem_count_launches(1);
  return cudaGetLastError();
}
