/* Set-up of the AQD2 object: incident wave, media, element constants, domain
 * lists and incident boundary data.
 *
 *   initialize_aqd2        bem3_aw_qd2.c:60-109
 *   element constants      bem3_aw_qd2.c:941-1023 (bilinear: r = a + b z + c e + d z e,
 *                          W = dr/dz x dr/de = cw0 + cw1 z + cw2 e)
 *   domain element lists   bem3_aw_qd2.c:1085-1102 (sid > 0 main side, < 0 sub side)
 *   incident data          bem3_aw_qd2.c:1104-1146 (Pi = -p/k2 at the nodes)
 *   plane wave             aw_pw.c:103-199
 */
#include "aqd2_internal.h"
#include <sys/time.h>

double aqd2_now(void)
{
  struct timeval tv;
  gettimeofday(&tv, NULL);
  return tv.tv_sec + 1e-6 * tv.tv_usec;
}

void setup_apw(Apw *pw)
{
  ApwD *w = &pw->wd;
  w->omega = 2.0 * M_PI * pw->f;
  w->K0 = pw->c0 * pw->c0 * pw->rho0;
  w->k1 = I * w->omega / w->K0;
  w->k2 = I * w->omega * pw->rho0;
  w->k0 = w->omega / pw->c0;
  w->lambda0 = pw->c0 / pw->f;
  /* propagation direction (sin th cos ps, sin th sin ps, cos th) as the third
     column of a rotation that takes the z axis onto it */
  double ct = cos(pw->theta), st = sin(pw->theta), cp = cos(pw->psi), sp = sin(pw->psi);
  w->R[0] = ct * cp * cp + sp * sp;  w->R[1] = sp * cp * (ct - 1.0);  w->R[2] = st * cp;
  w->R[3] = sp * cp * (ct - 1.0);    w->R[4] = ct * sp * sp + cp * cp; w->R[5] = st * sp;
  w->R[6] = -st * cp;                w->R[7] = -st * sp;               w->R[8] = ct;
  w->kx = w->R[2] * w->k0;
  w->ky = w->R[5] * w->k0;
  w->kz = w->R[8] * w->k0;
}

void calc_apw_pv(double complex *p, double complex *v, double *r, Apw *pw)
{
  const double *R = pw->wd.R;
  double rc[3], r0[3];
  for (int i = 0; i < 3; i++) rc[i] = r[i] - pw->tv[i];
  /* the reference applies the inverse rotation with this sign pattern (aw_pw.c:150-152) */
  r0[0] = R[0] * rc[0] + R[1] * rc[1] - R[2] * rc[2];
  r0[1] = R[3] * rc[0] + R[4] * rc[1] - R[5] * rc[2];
  r0[2] = -R[6] * rc[0] - R[7] * rc[1] + R[8] * rc[2];
  double arg = pw->wd.k0 * r0[2];
  double complex pp = pw->p * (cos(arg) + I * sin(arg));
  double complex vz = pp / (pw->rho0 * pw->c0);
  *p = pp;
  for (int i = 0; i < 3; i++) v[i] = R[i * 3 + 2] * vz;
}

void calc_apw_dpdn(double complex *p, double complex *dpdn, double *r, double *n, Apw *pw)
{
  const double *R = pw->wd.R;
  double rc[3], r0[3], n2;
  for (int i = 0; i < 3; i++) rc[i] = r[i] - pw->tv[i];
  r0[0] = R[0] * rc[0] + R[1] * rc[1] - R[2] * rc[2];
  r0[1] = R[3] * rc[0] + R[4] * rc[1] - R[5] * rc[2];
  r0[2] = -R[6] * rc[0] - R[7] * rc[1] + R[8] * rc[2];
  n2 = -R[6] * n[0] - R[7] * n[1] + R[8] * n[2];
  double arg = pw->wd.k0 * r0[2];
  double complex pp = pw->p * (cos(arg) + I * sin(arg));
  *p = pp;
  *dpdn = pp * I * pw->wd.k0 * n2;
}

/* Gauss-Legendre rule on [-1, 1]: Newton iteration on P_n from the
 * three-term recurrence, symmetric nodes (same rule as com_src/gauleg.c). */
void aqd2_gauss_legendre(double *x, double *w, int n)
{
  for (int i = 0; i < (n + 1) / 2; i++) {
    double z = cos(M_PI * (i + 0.75) / (n + 0.5)), dp = 0.0, p0 = 0.0, p1 = 0.0;
    for (int it = 0; it < 100; it++) {
      p0 = 1.0;
      p1 = 0.0;
      for (int j = 1; j <= n; j++) {
        double p2 = p1;
        p1 = p0;
        p0 = ((2.0 * j - 1.0) * z * p1 - (j - 1.0) * p2) / j;
      }
      dp = n * (z * p0 - p1) / (z * z - 1.0);
      double z1 = z;
      z = z1 - p0 / dp;
      if (fabs(z - z1) <= 3.0e-16) break;
    }
    x[i] = -z;
    x[n - 1 - i] = z;
    w[i] = w[n - 1 - i] = 2.0 / ((1.0 - z * z) * dp * dp);
  }
  if (n % 2 == 1) x[n / 2] = 0.0;
}

void aqd2_init_elem_const(BOUD *bd)
{
  for (int i = 1; i <= bd->Ne; i++) {
    double rc[3][4];
    for (int d = 0; d < 3; d++)
      for (int j = 0; j < 4; j++) rc[d][j] = bd->rn[bd->ed[i][j]][d];
    if (bd->ed[i][3] != 0) {  /* bilinear */
      for (int d = 0; d < 3; d++) {
        bd->cr[i][d][0] = 0.25 * (rc[d][0] + rc[d][1] + rc[d][2] + rc[d][3]);
        bd->cr[i][d][1] = 0.25 * (-rc[d][0] + rc[d][1] + rc[d][2] - rc[d][3]);
        bd->cr[i][d][2] = 0.25 * (-rc[d][0] - rc[d][1] + rc[d][2] + rc[d][3]);
        bd->cr[i][d][3] = 0.25 * (rc[d][0] - rc[d][1] + rc[d][2] - rc[d][3]);
      }
      /* W = (b + d e) x (c + d z): component k from coordinates (a, b) cyclic */
      static const int ca[3] = {1, 2, 0}, cb[3] = {2, 0, 1};
      for (int k = 0; k < 3; k++) {
        const double *A = rc[ca[k]], *B = rc[cb[k]];
        bd->cw[i][k][0] = 0.125 * ((A[0] - A[2]) * (B[1] - B[3]) - (A[1] - A[3]) * (B[0] - B[2]));
        bd->cw[i][k][1] = 0.125 * ((A[2] - A[3]) * (B[0] - B[1]) - (A[0] - A[1]) * (B[2] - B[3]));
        bd->cw[i][k][2] = 0.125 * ((A[1] - A[2]) * (B[0] - B[3]) - (A[0] - A[3]) * (B[1] - B[2]));
      }
    } else {  /* linear triangle */
      for (int d = 0; d < 3; d++) {
        bd->cr[i][d][0] = 1.0 / 3.0 * (rc[d][0] + rc[d][1] + rc[d][2]);
        bd->cr[i][d][1] = 1.0 / 3.0 * (-rc[d][0] + 2.0 * rc[d][1] - rc[d][2]);
        bd->cr[i][d][2] = 1.0 / sqrt(3.0) * (rc[d][2] - rc[d][0]);
        bd->cr[i][d][3] = 0.0;
      }
      bd->cw[i][0][0] = (rc[1][1] - rc[1][0]) * (rc[2][2] - rc[2][0]) - (rc[2][1] - rc[2][0]) * (rc[1][2] - rc[1][0]);
      bd->cw[i][1][0] = (rc[2][1] - rc[2][0]) * (rc[0][2] - rc[0][0]) - (rc[0][1] - rc[0][0]) * (rc[2][2] - rc[2][0]);
      bd->cw[i][2][0] = (rc[0][1] - rc[0][0]) * (rc[1][2] - rc[1][0]) - (rc[1][1] - rc[1][0]) * (rc[0][2] - rc[0][0]);
      for (int k = 0; k < 3; k++) bd->cw[i][k][1] = bd->cw[i][k][2] = 0.0;
    }
  }
  /* 4-point (nodes of the interpolation), 9-point, 4- and 7-point triangle rules */
  const double a = 0.5773502691896257645091, b = 0.7745966692414833770359;
  const double z44[4] = {-a, a, a, -a}, e44[4] = {-a, -a, a, a};
  for (int i = 0; i < 4; i++) { bd->zt_44[i] = z44[i]; bd->et_44[i] = e44[i]; bd->wt_44[i] = 1.0; }
  const double z49[9] = {-b, b, b, -b, 0.0, b, 0.0, -b, 0.0}, e49[9] = {-b, -b, b, b, -b, 0.0, b, 0.0, 0.0};
  const double w0 = 25.0 / 81.0, w1 = 40.0 / 81.0, w2 = 64.0 / 81.0;
  const double w49[9] = {w0, w0, w0, w0, w1, w1, w1, w1, w2};
  for (int i = 0; i < 9; i++) { bd->zt_49[i] = z49[i]; bd->et_49[i] = e49[i]; bd->wt_49[i] = w49[i]; }
  const double t0 = 0.2, t1 = 0.3464101615137754587055;
  const double z34[4] = {-t0, 2.0 * t0, -t0, 0.0}, e34[4] = {-t1, 0.0, t1, 0.0};
  const double w34[4] = {25.0 / 48.0, 25.0 / 48.0, 25.0 / 48.0, -27.0 / 48.0};
  for (int i = 0; i < 4; i++) { bd->zt_34[i] = z34[i]; bd->et_34[i] = e34[i]; bd->wt_34[i] = w34[i]; }
  const double s15 = sqrt(15.0), s3 = sqrt(3.0);
  const double n0 = (s15 + 1.0) / 14.0, n1 = (s15 - 1.0) / 14.0, n2 = s3 * (s15 + 1.0) / 14.0, n3 = s3 * (s15 - 1.0) / 14.0;
  const double z37[7] = {-n0, 2.0 * n0, -n0, n1, -2.0 * n1, n1, 0.0}, e37[7] = {-n2, 0.0, n2, n3, 0.0, -n3, 0.0};
  const double v0 = (155.0 - s15) / 1200.0, v1 = (155.0 + s15) / 1200.0, v2 = 270.0 / 1200.0;
  const double w37[7] = {v0, v0, v0, v1, v1, v1, v2};
  for (int i = 0; i < 7; i++) { bd->zt_37[i] = z37[i]; bd->et_37[i] = e37[i]; bd->wt_37[i] = w37[i]; }
  aqd2_gauss_legendre(bd->xli, bd->wli, GLN);
  aqd2_gauss_legendre(bd->xhi, bd->whi, GHN);
}

void aqd2_r_bd(double *r, int e, double zeta, double eta, BOUD *bd)
{
  double zh = bd->ed[e][3] == 0 ? 0.0 : zeta * eta;
  for (int i = 0; i < 3; i++) r[i] = bd->cr[e][i][0] + bd->cr[e][i][1] * zeta + bd->cr[e][i][2] * eta + bd->cr[e][i][3] * zh;
}

/* bil_check_plane (d3qd2_elem.c:986): the twist vector cr[.][1] is
 * perpendicular to cw[.][2] only for plane elements. */
int aqd2_elem_plane(BOUD *bd, int e)
{
  if (bd->ed[e][3] == 0) return 1;  /* triangles are plane */
  double **cr = bd->cr[e], **cw = bd->cw[e];
  double bdc = cr[0][1] * cw[0][2] + cr[1][1] * cw[1][2] + cr[2][1] * cw[2][2];
  double ab = sqrt(cr[0][1] * cr[0][1] + cr[1][1] * cr[1][1] + cr[2][1] * cr[2][1]);
  double aC = sqrt(cw[0][2] * cw[0][2] + cw[1][2] * cw[1][2] + cw[2][2] * cw[2][2]);
  return fabs(bdc / (ab * aC)) < GEPS ? 1 : 0;
}

static void rotate_translate(AQD2 *qd)
{
  double nv[3] = {qd->rv[0], qd->rv[1], qd->rv[2]};
  double an = sqrt(nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2]);
  if (an > 0.0) for (int i = 0; i < 3; i++) nv[i] /= an;
  double st = sin(qd->th), ct = cos(qd->th), M[9];
  /* Rodrigues' rotation about nv by th */
  M[0] = ct + nv[0] * nv[0] * (1.0 - ct);
  M[1] = nv[0] * nv[1] * (1.0 - ct) - nv[2] * st;
  M[2] = nv[2] * nv[0] * (1.0 - ct) + nv[1] * st;
  M[3] = nv[0] * nv[1] * (1.0 - ct) + nv[2] * st;
  M[4] = ct + nv[1] * nv[1] * (1.0 - ct);
  M[5] = nv[1] * nv[2] * (1.0 - ct) - nv[0] * st;
  M[6] = nv[2] * nv[0] * (1.0 - ct) - nv[1] * st;
  M[7] = nv[1] * nv[2] * (1.0 - ct) + nv[0] * st;
  M[8] = ct + nv[2] * nv[2] * (1.0 - ct);
  for (int s = 1; s <= qd->bd.Nn; s++) {
    double r[3], *p = qd->bd.rn[s];
    for (int i = 0; i < 3; i++) r[i] = M[3 * i] * p[0] + M[3 * i + 1] * p[1] + M[3 * i + 2] * p[2] + qd->tv[i];
    for (int i = 0; i < 3; i++) p[i] = r[i];
  }
}

void initialize_aqd2(AQD2 *qd)
{
  setup_apw(&qd->pw);
  qd->bd.qd.k = qd->pw.wd.k0;
  qd->bd.qd.vk[0] = qd->pw.wd.kx;
  qd->bd.qd.vk[1] = qd->pw.wd.ky;
  qd->bd.qd.vk[2] = qd->pw.wd.kz;
  if (qd->bd.ps != 0) {
    if (qd->bd.qd.vk[0] == 0.0 || qd->bd.qd.vk[1] == 0.0) {
      printf("kx and ky must not be equal to 0 (must satisfy quasi-peridic boundary condition). Exit...\n");
      exit(1);
    }
    if (qd->bd.qd.vk[2] == 0.0) printf("kz must not be equal to 0 (The wave source and the objcet must not overlap). Exit...\n");
  }
  qd->rho0[0] = qd->pw.rho0;
  qd->c0[0] = qd->pw.c0;
  qd->k0[0] = qd->pw.wd.k0;
  qd->K0[0] = qd->pw.wd.K0;
  qd->k1[0] = qd->pw.wd.k1;
  qd->k2[0] = qd->pw.wd.k2;
  for (int i = 1; i <= qd->MN; i++) {
    qd->k0[i] = qd->pw.wd.omega / qd->c0[i];
    qd->K0[i] = qd->rho0[i] * qd->c0[i] * qd->c0[i];
    qd->k1[i] = I * qd->pw.wd.omega / qd->K0[i];
    qd->k2[i] = I * qd->pw.wd.omega * qd->rho0[i];
  }
  double atv = sqrt(qd->tv[0] * qd->tv[0] + qd->tv[1] * qd->tv[1] + qd->tv[2] * qd->tv[2]);
  if (qd->th != 0.0 || atv != 0.0) rotate_translate(qd);
  aqd2_init_elem_const(&qd->bd);
  aqd2_malloc_sub_domain(qd);
  /* element lists: main side first in element order, sign marks the sub side */
  for (int d = 0; d <= qd->MN; d++) {
    int c = 1;
    for (int i = 1; i <= qd->bd.Ne; i++) {
      if (qd->bd.md[i] == d) qd->bd.sb[d].sid[c++] = i;
      else if (qd->bd.sd[i] == d) qd->bd.sb[d].sid[c++] = -i;
    }
  }
  /* collocation nodes, normals and incident data (4 nodes for quads, 4-point rule points for triangles) */
  double complex cp = -1.0 / qd->pw.wd.k2;
  for (int i = 1; i <= qd->bd.Ne; i++) {
    double **cr = qd->bd.cr[i], **cw = qd->bd.cw[i];
    int tri = qd->bd.ed[i][3] == 0;
    for (int j = 0; j < 4; j++) {
      double z = tri ? qd->bd.zt_34[j] : qd->bd.zt_44[j], e = tri ? qd->bd.et_34[j] : qd->bd.et_44[j];
      double r[3], w[3];
      for (int l = 0; l < 3; l++) {
        if (tri) {
          r[l] = cr[l][0] + cr[l][1] * z + cr[l][2] * e;
          w[l] = cw[l][0];
        } else {
          r[l] = cr[l][0] + cr[l][1] * z + cr[l][2] * e + cr[l][3] * z * e;
          w[l] = cw[l][0] + cw[l][1] * z + cw[l][2] * e;
        }
        qd->bd.ren[i][j][l] = r[l];
        qd->bd.wen[i][j][l] = w[l];
      }
      double aw = sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
      if (aw != 0.0) for (int l = 0; l < 3; l++) w[l] /= aw;
      double complex p, dp;
      calc_apw_dpdn(&p, &dp, r, w, &qd->pw);
      qd->bd.Pi[i][j] = cp * p;
      qd->bd.dPi[i][j] = cp * dp;
    }
  }
}

void domain_id_l_aqd2(int *l1, int *l2, double *rt, AQD2 *qd)
{
  double idet = 1.0 / (qd->bd.qd.vd1[0] * qd->bd.qd.vd2[1] - qd->bd.qd.vd2[0] * qd->bd.qd.vd1[1]);
  *l1 = (int)floor((rt[0] * qd->bd.qd.vd2[1] - rt[1] * qd->bd.qd.vd2[0]) * idet + 0.5);
  *l2 = (int)floor(-(rt[0] * qd->bd.qd.vd1[1] - rt[1] * qd->bd.qd.vd1[0]) * idet + 0.5);
}

void surface_area_aqd2(double *S, int did, int type, AQD2 *qd)
{
  /* sum of |W| over the element's quadrature points (bil_sa_4p/_9p) */
  double sa = 0.0;
  for (int t = 1; t <= qd->bd.sb[did].Ne; t++) {
    int e = abs(qd->bd.sb[did].sid[t]);
    double **cw = qd->bd.cw[e];
    int n = type == 0 ? 4 : 9;
    for (int i = 0; i < n; i++) {
      double z = type == 0 ? qd->bd.zt_44[i] : qd->bd.zt_49[i], eta = type == 0 ? qd->bd.et_44[i] : qd->bd.et_49[i];
      double wt = type == 0 ? qd->bd.wt_44[i] : qd->bd.wt_49[i], w[3];
      for (int l = 0; l < 3; l++) w[l] = cw[l][0] + cw[l][1] * z + cw[l][2] * eta;
      sa += wt * sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
    }
  }
  *S = sa;
}
