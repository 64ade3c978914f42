/* Extra C entry points compiled into oracle/_ref/libbem3ref.so next to the
 * unmodified reference sources.  They let the test suite and the CPU-baseline
 * leg of the benchmark drive the reference's own functions from Python
 * (ctypes) and read back intermediate results.  Nothing here changes what the
 * reference computes: every number still comes from the reference's code.
 *
 * Cited reference entry points:
 *   Faddeeva_w                      qgf2_src/Faddeeva.cc:679
 *   d3hm_qpgf_d2_v1 / _qG / _dqG    qgf2_src/d3_qpgf_d2.c:124, :10, :67
 *   d3hm_qpgf_d2_v1_fd / _v1_ew     qgf2_src/d3_qpgf_d2.c:290, :409
 *   q0_dcoef_bd_node_t2_cc          d3qd2_src/d3qd2_elem.c:830
 *   dcoef_bd_node_t2                d3qd2_src/d3qd2_elem.c:515
 *   create_cmatrix_domain etc.      d3qd2_src/bem3_aw_qd2_solve_bieq.c:124-750
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <complex.h>
#include "bem3_aw_qd2.h"

/* functions with external linkage inside bem3_aw_qd2_solve_bieq.c */
void initalize_cmd(CMD *cm);
void create_cmatrix(CMD *cm, AQD2 *qd);
void create_cmatrix_domain(int did, CMD *cm, AQD2 *qd);
void create_tmatrix_csr(CMD *cm, AQD2 *qd);
void solve_tmatrix_csr(CMD *cm, AQD2 *qd);
void q_solve_pv_bv(CMD *cm, AQD2 *qd);
void solve_pv_bv(CMD *cm, AQD2 *qd);
void solve_dpv_bv(CMD *cm, AQD2 *qd);

size_t ref_sizeof_aqd2(void) { return sizeof(AQD2); }
size_t ref_sizeof_apw(void) { return sizeof(Apw); }

void ref_faddeeva_w(const double *z, int n, double relerr, double *w)
{
  for (int i = 0; i < n; i++) {
    double complex r = Faddeeva_w(z[2 * i] + I * z[2 * i + 1], relerr);
    w[2 * i] = creal(r);
    w[2 * i + 1] = cimag(r);
  }
}

static void fill_qpd(QPD2 *q, const double *p)
{
  /* p = {k, kx, ky, kz, d1x, d1y, d2x, d2y} */
  q->k = p[0];
  q->vk[0] = p[1]; q->vk[1] = p[2]; q->vk[2] = p[3];
  q->vd1[0] = p[4]; q->vd1[1] = p[5];
  q->vd2[0] = p[6]; q->vd2[1] = p[7];
}

/* mode 0: d3hm_qpgf_d2_v1 (auto select), 1: _v1_ew, 2: _v1_fd,
 *      3: d3hm_qpgf_d2_qG, 4: d3hm_qpgf_d2_dqG */
void ref_qpgf(int mode, const double *qp, const double *r, int n, double eps,
              double *G, double *dG, int *ret)
{
  QPD2 q;
  fill_qpd(&q, qp);
  for (int i = 0; i < n; i++) {
    double complex g = 0.0, dg[3] = {0.0, 0.0, 0.0};
    double rr[3] = {r[3 * i], r[3 * i + 1], r[3 * i + 2]};
    int e;
    switch (mode) {
      case 0: e = d3hm_qpgf_d2_v1(&g, dg, rr, eps, &q); break;
      case 1: e = d3hm_qpgf_d2_v1_ew(&g, dg, rr, eps, &q); break;
      case 2: e = d3hm_qpgf_d2_v1_fd(&g, dg, rr, eps, &q); break;
      case 3: e = d3hm_qpgf_d2_qG(&g, rr, eps, &q); break;
      default: e = d3hm_qpgf_d2_dqG(dg, rr, eps, &q); break;
    }
    ret[i] = e;
    G[2 * i] = creal(g); G[2 * i + 1] = cimag(g);
    for (int c = 0; c < 3; c++) { dG[6 * i + 2 * c] = creal(dg[c]); dG[6 * i + 2 * c + 1] = cimag(dg[c]); }
  }
}

/* Run the reference's boundary-value solve on an initialised AQD2 but keep the
 * temporary matrix files (tmpG_*.dat, tmpH_*.dat, tmpdG/dH/dF_*.dat, tmpAval,
 * tmpB ...) in the current directory so the caller can read them.  Mirrors
 * solve_bieq_aqd2 (bem3_aw_qd2_solve_bieq.c:3-51) without finalize_cmd. */
void ref_solve_keep_files(AQD2 *qd)
{
  CMD cm;
  cm.type = 2;
  cm.MN = qd->MN;
  initalize_cmd(&cm);
  create_cmatrix(&cm, qd);
  cm.nn = (size_t)qd->bd.NN;
  cm.na = cm.nn * 2;
  create_tmatrix_csr(&cm, qd);
  solve_tmatrix_csr(&cm, qd);
  if (qd->bd.ps == 1) q_solve_pv_bv(&cm, qd);
  else solve_pv_bv(&cm, qd);
  solve_dpv_bv(&cm, qd);
}

/* Only the coefficient matrices of one domain (files in the current directory). */
void ref_assemble_domain_files(AQD2 *qd, int did)
{
  CMD cm;
  cm.type = 2;
  cm.MN = qd->MN;
  initalize_cmd(&cm);
  create_cmatrix_domain(did, &cm, qd);
}

/* Time-boxed sample of create_cmatrix_domain (bem3_aw_qd2_solve_bieq.c:133-218):
 * the same per-(t, tn, s) element calls for collocation elements t in
 * [t0, t1) of domain did, on nthreads OpenMP threads, results discarded except
 * for a checksum.  Used to time the reference's assembly on a bounded sample. */
double ref_assemble_rows(AQD2 *qd, int did, int t0, int t1)
{
  double chk = 0.0;
  int Ne = qd->bd.sb[did].Ne;
  double complex kc = (double complex)qd->k0[did];
  #pragma omp parallel for schedule(dynamic) reduction(+:chk)
  for (int t = t0; t < t1; t++) {
    double complex CC[9], dCz[9], dCe[9];
    double vtz[3], vte[3];
    int td = qd->bd.sb[did].sid[t];
    int tl = (ELT3 == check_element_type(td, &(qd->bd))) ? 3 : 4;
    for (int tn = 0; tn < tl; tn++) {
      tz_te_bd_node(vtz, vte, td, tn, &(qd->bd));
      for (int s = 1; s <= Ne; s++) {
        int sd = qd->bd.sb[did].sid[s];
        if (did == 0 && qd->bd.ps == 1) q0_dcoef_bd_node_t2_cc(CC, dCz, dCe, td, tn, vtz, vte, sd, kc, 2, &(qd->bd));
        else dcoef_bd_node_t2(CC, dCz, dCe, td, tn, vtz, vte, sd, kc, 2, &(qd->bd));
        chk += creal(CC[0]) + cimag(CC[4]);
      }
    }
  }
  return chk;
}

/* The same loop on a list of collocation elements ts[0..n) (1-based), e.g. a
 * seeded random sample of the domain's rows. */
double ref_assemble_list(AQD2 *qd, int did, const int *ts, int n)
{
  double chk = 0.0;
  int Ne = qd->bd.sb[did].Ne;
  double complex kc = (double complex)qd->k0[did];
  #pragma omp parallel for schedule(dynamic) reduction(+:chk)
  for (int i = 0; i < n; i++) {
    double complex CC[9], dCz[9], dCe[9];
    double vtz[3], vte[3];
    int td = qd->bd.sb[did].sid[ts[i]];
    int tl = (ELT3 == check_element_type(td, &(qd->bd))) ? 3 : 4;
    for (int tn = 0; tn < tl; tn++) {
      tz_te_bd_node(vtz, vte, td, tn, &(qd->bd));
      for (int s = 1; s <= Ne; s++) {
        int sd = qd->bd.sb[did].sid[s];
        if (did == 0 && qd->bd.ps == 1) q0_dcoef_bd_node_t2_cc(CC, dCz, dCe, td, tn, vtz, vte, sd, kc, 2, &(qd->bd));
        else dcoef_bd_node_t2(CC, dCz, dCe, td, tn, vtz, vte, sd, kc, 2, &(qd->bd));
        chk += creal(CC[0]) + cimag(CC[4]);
      }
    }
  }
  return chk;
}

/* One element-pair coefficient call, for unit tests of the per-pair kernels.
 * out: CC[9], dCdtz[9], dCdte[9] as interleaved (re, im). */
void ref_pair_coef(AQD2 *qd, int did, int t, int tn, int s, double *out)
{
  double complex CC[9], dCz[9], dCe[9];
  double vtz[3], vte[3];
  int td = qd->bd.sb[did].sid[t];
  int sd = qd->bd.sb[did].sid[s];
  tz_te_bd_node(vtz, vte, td, tn, &(qd->bd));
  if (did == 0 && qd->bd.ps == 1) q0_dcoef_bd_node_t2_cc(CC, dCz, dCe, td, tn, vtz, vte, sd, (double complex)qd->k0[did], 2, &(qd->bd));
  else dcoef_bd_node_t2(CC, dCz, dCe, td, tn, vtz, vte, sd, (double complex)qd->k0[did], 2, &(qd->bd));
  for (int i = 0; i < 9; i++) {
    out[2 * i] = creal(CC[i]); out[2 * i + 1] = cimag(CC[i]);
    out[18 + 2 * i] = creal(dCz[i]); out[18 + 2 * i + 1] = cimag(dCz[i]);
    out[36 + 2 * i] = creal(dCe[i]); out[36 + 2 * i + 1] = cimag(dCe[i]);
  }
}

/* Pointers into the AQD2 so Python can read the solution arrays. */
int ref_domain_ne(AQD2 *qd, int d) { return qd->bd.sb[d].Ne; }
int ref_mn(AQD2 *qd) { return qd->MN; }
int ref_ne(AQD2 *qd) { return qd->bd.Ne; }
int ref_nn(AQD2 *qd) { return qd->bd.NN; }
/* P,dP as [Ne_d][4] complex; pv,dpv as [Ne_d][4][3] complex (element index 1..Ne_d) */
void ref_get_solution(AQD2 *qd, int d, double *P, double *dP, double *pv, double *dpv)
{
  int Ne = qd->bd.sb[d].Ne;
  for (int s = 1; s <= Ne; s++)
    for (int n = 0; n < 4; n++) {
      size_t o = (size_t)(s - 1) * 4 + n;
      P[2 * o] = creal(qd->bd.sb[d].P[s][n]); P[2 * o + 1] = cimag(qd->bd.sb[d].P[s][n]);
      dP[2 * o] = creal(qd->bd.sb[d].dP[s][n]); dP[2 * o + 1] = cimag(qd->bd.sb[d].dP[s][n]);
      for (int c = 0; c < 3; c++) {
        pv[2 * (3 * o + c)] = creal(qd->bd.sb[d].pv[s][n][c]); pv[2 * (3 * o + c) + 1] = cimag(qd->bd.sb[d].pv[s][n][c]);
        dpv[2 * (3 * o + c)] = creal(qd->bd.sb[d].dpv[s][n][c]); dpv[2 * (3 * o + c) + 1] = cimag(qd->bd.sb[d].dpv[s][n][c]);
      }
    }
}

/* read_aqd2 + initialize_aqd2 from five file names (rotation optional). */
void ref_load(AQD2 *qd, const char *pw, const char *per, const char *med, const char *msh)
{
  char *argv[6] = {(char *)"ref", (char *)pw, (char *)per, (char *)med, (char *)msh, (char *)"unused.dat"};
  read_aqd2(6, argv, qd);
  initialize_aqd2(qd);
}

/* Coefficients CC[9] of source s (1-based index into domain did) at the
 * boundary point (zeta, eta) of element t of the same domain, as the boundary
 * field functions use them (q0_coef_bd / coef_bd, d3qd2_src/d3qd2_elem.c:684,
 * :187).  out = 9 complex numbers. */
void ref_bd_coef(AQD2 *qd, int did, int t, double zeta, double eta, int s, int type, double *out)
{
  double complex CC[9];
  double rt[3];
  int td = qd->bd.sb[did].sid[t], sd = qd->bd.sb[did].sid[s];
  r_bd(rt, td, zeta, eta, &(qd->bd));
  if (did == 0 && qd->bd.ps == 1) q0_coef_bd(CC, rt, td, zeta, eta, sd, (double complex)qd->k0[did], type, &(qd->bd));
  else coef_bd(CC, rt, td, zeta, eta, sd, (double complex)qd->k0[did], type, &(qd->bd));
  for (int i = 0; i < 9; i++) { out[2 * i] = creal(CC[i]); out[2 * i + 1] = cimag(CC[i]); }
}

/* Point of element t (1-based index into domain did) at (zeta, eta) (r_bd, d3qd2_src/d3qd2_elem.c:18). */
void ref_r_bd(AQD2 *qd, int did, int t, double zeta, double eta, double *r)
{
  r_bd(r, qd->bd.sb[did].sid[t], zeta, eta, &(qd->bd));
}
