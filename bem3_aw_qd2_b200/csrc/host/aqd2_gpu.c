/* solve_bieq_aqd2, force_FN_aqd2 and the field functions on the device.
 *
 * The AQD2 object keeps the reference's layout (it is written raw into the
 * .dat file), so device state is kept in a side table keyed by the AQD2
 * address.  solve_bieq_aqd2 flattens the element tables into a
 * bemgpu_problem, runs the assembly and the solves on the GPU and copies
 * P, dP, pv, dpv back into the reference's SUBD arrays.  There is no CPU
 * fallback: a missing or failing GPU is a fatal error, as every failure is in
 * the reference (printf + exit).
 */
#include "aqd2_internal.h"

#define AQD2_MAXCTX 64
static struct { AQD2 *qd; bemgpu_ctx *ctx; } g_tab[AQD2_MAXCTX];
static int g_device = 0;
static int g_precision = -1; /* -1: from the environment (AQD2_PRECISION), else 0 */
static double g_timing[4];
static int g_verbose = 1;

void aqd2_set_verbose(int on) { g_verbose = on; }

void aqd2_set_device(int device) { g_device = device; }
void aqd2_set_precision(int mode) { g_precision = mode; }

static int g_keep_dgh = -1; /* -1: from the environment (AQD2_INTERIOR_DERIVATIVES), else 1 */
void aqd2_set_interior_derivatives(int keep) { g_keep_dgh = keep; }
static int keep_dgh_mode(void)
{
  if (g_keep_dgh >= 0) return g_keep_dgh;
  const char *e = getenv("AQD2_INTERIOR_DERIVATIVES");
  return e ? atoi(e) : 1;
}

static int precision_mode(void)
{
  if (g_precision >= 0) return g_precision;
  const char *e = getenv("AQD2_PRECISION");
  return e ? atoi(e) : 0;
}
void aqd2_last_timing(double *t4) { for (int i = 0; i < 4; i++) t4[i] = g_timing[i]; }

static bemgpu_ctx *ctx_for(AQD2 *qd, int create)
{
  for (int i = 0; i < AQD2_MAXCTX; i++)
    if (g_tab[i].qd == qd) return g_tab[i].ctx;
  if (!create) return NULL;
  for (int i = 0; i < AQD2_MAXCTX; i++)
    if (!g_tab[i].qd) {
      bemgpu_ctx *c = NULL;
      if (bemgpu_create(g_device, NULL, &c) != 0) {
        printf("bem3_aw_qd2: failed to create a CUDA context on device %d. Exit...\n", g_device);
        exit(1);
      }
      if (bemgpu_set_precision(c, precision_mode()) != 0 ||
          bemgpu_set_interior_derivatives(c, keep_dgh_mode(), 0) != 0) {
        printf("bem3_aw_qd2: %s. Exit...\n", bemgpu_error(c));
        exit(1);
      }
      g_tab[i].qd = qd;
      g_tab[i].ctx = c;
      return c;
    }
  printf("bem3_aw_qd2: too many live AQD2 objects. Exit...\n");
  exit(1);
}

struct bemgpu_ctx *aqd2_device_context(AQD2 *qd) { return ctx_for(qd, 0); }

void aqd2_release_device(AQD2 *qd)
{
  for (int i = 0; i < AQD2_MAXCTX; i++)
    if (g_tab[i].qd == qd) {
      bemgpu_destroy(g_tab[i].ctx);
      g_tab[i].qd = NULL;
      g_tab[i].ctx = NULL;
    }
}

static void gpu_check(bemgpu_ctx *c, int rc, const char *what)
{
  if (rc != 0) {
    printf("bem3_aw_qd2 (%s): %s (code %d). Exit...\n", what, bemgpu_error(c), rc);
    exit(1);
  }
}

/* Flatten an initialised AQD2 into a bemgpu_problem whose arrays are malloc'ed
 * here (aqd2_problem_free releases them): element tables, domain lists, media
 * and the incident field at the element nodes (calc_apw_pv, aw_pw.c:129). */
void aqd2_problem_build(AQD2 *qd, bemgpu_problem *pr)
{
  BOUD *bd = &qd->bd;
  int Ne = bd->Ne, nd = qd->MN + 1, tot = 0;
  for (int d = 0; d < nd; d++) tot += bd->sb[d].Ne;
  double *cr = aqd2_calloc(Ne * 12, sizeof(double), "cr"), *cw = aqd2_calloc(Ne * 9, sizeof(double), "cw");
  double *ren = aqd2_calloc(Ne * 12, sizeof(double), "ren"), *wen = aqd2_calloc(Ne * 12, sizeof(double), "wen");
  double *Pi = aqd2_calloc(Ne * 8, sizeof(double), "Pi"), *dPi = aqd2_calloc(Ne * 8, sizeof(double), "dPi");
  double *pinc = aqd2_calloc(Ne * 8, sizeof(double), "pinc"), *vinc = aqd2_calloc(Ne * 24, sizeof(double), "vinc");
  int *npe = aqd2_calloc(Ne, sizeof(int), "npe"), *eni = aqd2_calloc(Ne * 4, sizeof(int), "eni");
  int *md = aqd2_calloc(Ne, sizeof(int), "md"), *sd = aqd2_calloc(Ne, sizeof(int), "sd");
  int *dom_ne = aqd2_calloc(nd, sizeof(int), "dom_ne"), *sid = aqd2_calloc(tot, sizeof(int), "sid");
  double *k2 = aqd2_calloc(2 * nd, sizeof(double), "k2");
  double *k0 = aqd2_calloc(nd, sizeof(double), "k0"), *rho0 = aqd2_calloc(nd, sizeof(double), "rho0");
  double *c0 = aqd2_calloc(nd, sizeof(double), "c0");
  double *xl = aqd2_calloc(GLN, sizeof(double), "xl"), *wl = aqd2_calloc(GLN, sizeof(double), "wl");
  double *xh = aqd2_calloc(GHN, sizeof(double), "xh"), *wh = aqd2_calloc(GHN, sizeof(double), "wh");
  unsigned char *plane = aqd2_calloc(Ne, 1, "plane");
  for (int e = 0; e < Ne; e++) {
    int i = e + 1;
    for (int d = 0; d < 3; d++) {
      for (int k = 0; k < 4; k++) cr[e * 12 + d * 4 + k] = bd->cr[i][d][k];
      for (int k = 0; k < 3; k++) cw[e * 9 + d * 3 + k] = bd->cw[i][d][k];
    }
    for (int n = 0; n < 4; n++) {
      for (int d = 0; d < 3; d++) {
        ren[e * 12 + n * 3 + d] = bd->ren[i][n][d];
        wen[e * 12 + n * 3 + d] = bd->wen[i][n][d];
      }
      Pi[e * 8 + 2 * n] = creal(bd->Pi[i][n]);
      Pi[e * 8 + 2 * n + 1] = cimag(bd->Pi[i][n]);
      dPi[e * 8 + 2 * n] = creal(bd->dPi[i][n]);
      dPi[e * 8 + 2 * n + 1] = cimag(bd->dPi[i][n]);
      double complex p, v[3];
      calc_apw_pv(&p, v, bd->ren[i][n], &qd->pw);
      pinc[e * 8 + 2 * n] = creal(p);
      pinc[e * 8 + 2 * n + 1] = cimag(p);
      for (int d = 0; d < 3; d++) {
        vinc[e * 24 + n * 6 + 2 * d] = creal(v[d]);
        vinc[e * 24 + n * 6 + 2 * d + 1] = cimag(v[d]);
      }
      eni[e * 4 + n] = bd->eni[i][n];
    }
    npe[e] = bd->ed[i][3] == 0 ? 3 : 4;
    md[e] = bd->md[i];
    sd[e] = bd->sd[i];
    plane[e] = (unsigned char)aqd2_elem_plane(bd, i);
  }
  int o = 0;
  for (int d = 0; d < nd; d++) {
    dom_ne[d] = bd->sb[d].Ne;
    for (int s = 1; s <= bd->sb[d].Ne; s++) sid[o++] = bd->sb[d].sid[s];
    k2[2 * d] = creal(qd->k2[d]);
    k2[2 * d + 1] = cimag(qd->k2[d]);
    k0[d] = qd->k0[d];
    rho0[d] = qd->rho0[d];
    c0[d] = qd->c0[d];
  }
  for (int i = 0; i < GLN; i++) { xl[i] = bd->xli[i]; wl[i] = bd->wli[i]; }
  for (int i = 0; i < GHN; i++) { xh[i] = bd->xhi[i]; wh[i] = bd->whi[i]; }
  memset(pr, 0, sizeof(*pr));
  pr->Ne = Ne; pr->NN = bd->NN; pr->MN = qd->MN; pr->ps = bd->ps;
  pr->qp[0] = bd->qd.k; pr->qp[1] = bd->qd.vk[0]; pr->qp[2] = bd->qd.vk[1]; pr->qp[3] = bd->qd.vk[2];
  pr->qp[4] = bd->qd.vd1[0]; pr->qp[5] = bd->qd.vd1[1]; pr->qp[6] = bd->qd.vd2[0]; pr->qp[7] = bd->qd.vd2[1];
  pr->cr = cr; pr->cw = cw; pr->ren = ren; pr->wen = wen; pr->npe = npe; pr->eni = eni; pr->md = md; pr->sd = sd;
  pr->dom_ne = dom_ne; pr->sid = sid; pr->k0 = k0; pr->k2 = k2; pr->rho0 = rho0; pr->c0 = c0;
  pr->Pi = Pi; pr->dPi = dPi; pr->p_inc = pinc; pr->v_inc = vinc;
  pr->xl = xl; pr->wl = wl; pr->xh = xh; pr->wh = wh; pr->plane = plane;
  pr->pw[0] = creal(qd->pw.p);
  pr->pw[1] = cimag(qd->pw.p);
  for (int i = 0; i < 9; i++) pr->pw[2 + i] = qd->pw.wd.R[i];
  for (int i = 0; i < 3; i++) pr->pw[11 + i] = qd->pw.tv[i];
  pr->pw[14] = qd->pw.wd.k0;
  pr->pw[15] = qd->pw.rho0 * qd->pw.c0;
}

void aqd2_problem_free(bemgpu_problem *pr)
{
  free((void *)pr->cr); free((void *)pr->cw); free((void *)pr->ren); free((void *)pr->wen);
  free((void *)pr->Pi); free((void *)pr->dPi); free((void *)pr->p_inc); free((void *)pr->v_inc);
  free((void *)pr->npe); free((void *)pr->eni); free((void *)pr->md); free((void *)pr->sd);
  free((void *)pr->dom_ne); free((void *)pr->sid); free((void *)pr->k2); free((void *)pr->k0);
  free((void *)pr->rho0); free((void *)pr->c0); free((void *)pr->xl); free((void *)pr->wl);
  free((void *)pr->xh); free((void *)pr->wh); free((void *)pr->plane);
  memset(pr, 0, sizeof(*pr));
}

/* flatten AQD2 and upload */
static void load_problem(AQD2 *qd, bemgpu_ctx *c)
{
  bemgpu_problem pr;
  aqd2_problem_build(qd, &pr);
  gpu_check(c, bemgpu_load(c, &pr), "load");
  gpu_check(c, bemgpu_sync(c), "load");
  aqd2_problem_free(&pr);
}

static void download_solution(AQD2 *qd, bemgpu_ctx *c)
{
  for (int d = 0; d <= qd->MN; d++) {
    SUBD *s = &qd->bd.sb[d];
    size_t N = 4 * (size_t)s->Ne;
    double *P = aqd2_calloc(2 * N, sizeof(double), "P"), *dP = aqd2_calloc(2 * N, sizeof(double), "dP");
    double *pv = aqd2_calloc(6 * N, sizeof(double), "pv"), *dpv = aqd2_calloc(6 * N, sizeof(double), "dpv");
    gpu_check(c, bemgpu_get_solution(c, d, P, dP, pv, dpv), "download");
    for (int t = 1; t <= s->Ne; t++)
      for (int n = 0; n < 4; n++) {
        size_t q = (size_t)(t - 1) * 4 + n;
        s->P[t][n] = P[2 * q] + I * P[2 * q + 1];
        s->dP[t][n] = dP[2 * q] + I * dP[2 * q + 1];
        for (int l = 0; l < 3; l++) {
          s->pv[t][n][l] = pv[2 * (3 * q + l)] + I * pv[2 * (3 * q + l) + 1];
          s->dpv[t][n][l] = dpv[2 * (3 * q + l)] + I * dpv[2 * (3 * q + l) + 1];
        }
      }
    free(P); free(dP); free(pv); free(dpv);
  }
}

void solve_bieq_aqd2(AQD2 *qd)
{
  bemgpu_ctx *c = ctx_for(qd, 1);
  if (g_verbose) printf("\nsolve acoustic wave boundary value \n");
  double t0 = aqd2_now();
  load_problem(qd, c);
  double t1 = aqd2_now();
  if (g_verbose) {
    printf("  coefficient matrix          ");
    fflush(stdout);
  }
  gpu_check(c, bemgpu_assemble(c), "assembly");
  gpu_check(c, bemgpu_sync(c), "assembly");
  double t2 = aqd2_now();
  if (g_verbose) {
    printf("finished. Elapsed time : %5g (sec)\n", t2 - t1);
    printf("  solve VP and PV boundary value ");
    fflush(stdout);
  }
  gpu_check(c, bemgpu_solve(c), "solve");
  gpu_check(c, bemgpu_sync(c), "solve");
  unsigned st = bemgpu_status(c);
  if (st) {
    printf("\nbem3_aw_qd2: device status 0x%x (1: lattice-sum limit, 2: Rayleigh anomaly, 4: near-singular table, 8: non-finite, 16: geometry). Exit...\n", st);
    exit(1);
  }
  double t3 = aqd2_now();
  if (g_verbose) printf("finished. Elapsed time : %5g (sec)\n", t3 - t2);
  download_solution(qd, c);
  double t4 = aqd2_now();
  g_timing[0] = t1 - t0; g_timing[1] = t2 - t1; g_timing[2] = t3 - t2; g_timing[3] = t4 - t3;
  if (g_verbose) printf("Total elapsed time : %g (sec)\n", t4 - t0);
}

static void upload_solution(AQD2 *qd, bemgpu_ctx *c)
{
  for (int d = 0; d <= qd->MN; d++) {
    SUBD *s = &qd->bd.sb[d];
    size_t N = 4 * (size_t)s->Ne;
    double *P = aqd2_calloc(2 * N, sizeof(double), "P"), *dP = aqd2_calloc(2 * N, sizeof(double), "dP");
    double *pv = aqd2_calloc(6 * N, sizeof(double), "pv"), *dpv = aqd2_calloc(6 * N, sizeof(double), "dpv");
    for (int t = 1; t <= s->Ne; t++)
      for (int n = 0; n < 4; n++) {
        size_t q = (size_t)(t - 1) * 4 + n;
        P[2 * q] = creal(s->P[t][n]);
        P[2 * q + 1] = cimag(s->P[t][n]);
        dP[2 * q] = creal(s->dP[t][n]);
        dP[2 * q + 1] = cimag(s->dP[t][n]);
        for (int l = 0; l < 3; l++) {
          pv[2 * (3 * q + l)] = creal(s->pv[t][n][l]);
          pv[2 * (3 * q + l) + 1] = cimag(s->pv[t][n][l]);
          dpv[2 * (3 * q + l)] = creal(s->dpv[t][n][l]);
          dpv[2 * (3 * q + l) + 1] = cimag(s->dpv[t][n][l]);
        }
      }
    gpu_check(c, bemgpu_set_solution(c, d, P, dP, pv, dpv), "upload");
    free(P); free(dP); free(pv); free(dpv);
  }
}

/* The device context holding qd's boundary values.  After solve_bieq_aqd2 the
 * context already has them; for an object filled by dat_read_aqd2 the problem
 * and the stored boundary values are uploaded on first use. */
static bemgpu_ctx *ready_ctx(AQD2 *qd)
{
  bemgpu_ctx *c = ctx_for(qd, 0);
  if (c) return c;
  c = ctx_for(qd, 1);
  load_problem(qd, c);
  upload_solution(qd, c);
  return c;
}

static void status_check(bemgpu_ctx *c, const char *what)
{
  unsigned st = bemgpu_status(c);
  if (st) {
    printf("bem3_aw_qd2 (%s): device status 0x%x (1: lattice-sum limit, 2: Rayleigh anomaly, 4: near-singular table, 8: non-finite, 16: geometry). Exit...\n", what, st);
    exit(1);
  }
}

void force_FN_aqd2(double *F, double *N, double *rc, int type, AQD2 *qd)
{
  bemgpu_ctx *c = ready_ctx(qd);
  gpu_check(c, bemgpu_force(c, type, rc, F, N), "force");
  status_check(c, "force");
}

int pv_i_aqd2(double complex *p, double complex *pv, double *rt, int type, AQD2 *qd)
{
  (void)type;
  calc_apw_pv(p, pv, rt, &qd->pw);
  return domain_id_aqd2(rt, qd);
}

int p_i_aqd2(double complex *p, double *rt, int type, AQD2 *qd)
{
  double complex v[3];
  (void)type;
  calc_apw_pv(p, v, rt, &qd->pw);
  return domain_id_aqd2(rt, qd);
}

int phi_i_aqd2(double complex *phi, double *rt, int type, AQD2 *qd)
{
  double complex p, v[3];
  (void)type;
  calc_apw_pv(&p, v, rt, &qd->pw);
  *phi = -p / qd->pw.wd.k2;
  return domain_id_aqd2(rt, qd);
}

static int domain_id_home(double *rt, AQD2 *qd);

/* Element sums of one field point (bem3_aw_qd2_field.c:3-54, 128-297): the
 * point is moved to the home lattice cell (domain_id_l_aqd2), its domain found
 * by the solid-angle test, and the sums of that domain evaluated on the
 * device.  Returns the domain id; o = bemgpu_field's 18 values, ce the Bloch
 * phase of the cell shift.  flags: 0 or BEMGPU_FIELD_POTENTIAL. */
static int field_sums(double o[18], double complex *ce, double *rt, int type, int flags, AQD2 *qd)
{
  int l1 = 0, l2 = 0;
  double r0[3] = {rt[0], rt[1], rt[2]};
  if (type < 0 || type > 3) {
    printf("bem3_aw_qd2: field rule type=%d is not available (0: 4-point, 1: 9-point, 2: GLN-point, 3: GHN-point). Exit...\n", type);
    exit(1);
  }
  if (qd->bd.ps == 1) {
    domain_id_l_aqd2(&l1, &l2, rt, qd);
    r0[0] = rt[0] - l1 * qd->bd.qd.vd1[0] - l2 * qd->bd.qd.vd2[0];
    r0[1] = rt[1] - l1 * qd->bd.qd.vd1[1] - l2 * qd->bd.qd.vd2[1];
  }
  int did = domain_id_home(r0, qd);
  if (did < 0) {
    printf("bem3_aw_qd2: the point (%g, %g, %g) lies in no domain. Exit...\n", rt[0], rt[1], rt[2]);
    exit(1);
  }
  bemgpu_ctx *c = ready_ctx(qd);
  gpu_check(c, bemgpu_field(c, did, type | flags, 1, r0, o), "field");
  status_check(c, "field");
  *ce = 1.0;
  if (l1 != 0 || l2 != 0) {
    double arg = qd->bd.qd.vk[0] * (l1 * qd->bd.qd.vd1[0] + l2 * qd->bd.qd.vd2[0]) +
                 qd->bd.qd.vk[1] * (l1 * qd->bd.qd.vd1[1] + l2 * qd->bd.qd.vd2[1]);
    *ce = cos(arg) + I * sin(arg);
  }
  return did;
}

#define FS_S0(o) ((o)[0] + I * (o)[1])
#define FS_S1(o, j) ((o)[2 + 2 * (j)] + I * (o)[3 + 2 * (j)])
#define FS_S2(o, j) ((o)[12 + 2 * (j)] + I * (o)[13 + 2 * (j)])

int phi_s_aqd2(double complex *phi, double *rt, int type, AQD2 *qd)
{
  double o[18];
  double complex ce;
  int did = field_sums(o, &ce, rt, type, BEMGPU_FIELD_POTENTIAL, qd);
  *phi = FS_S0(o) / (did == 0 ? 1.0 + o[8] : o[8]) * ce;
  return did;
}

int phi_t_aqd2(double complex *phi, double *rt, int type, AQD2 *qd)
{
  double complex p, v[3];
  int did = phi_s_aqd2(phi, rt, type, qd);
  if (did == 0) {
    calc_apw_pv(&p, v, rt, &qd->pw);
    *phi += -p / qd->pw.wd.k2;
  }
  return did;
}

int p_s_aqd2(double complex *p, double *rt, int type, AQD2 *qd)
{
  int did = phi_s_aqd2(p, rt, type, qd);
  *p *= -qd->k2[did];
  return did;
}

int p_t_aqd2(double complex *p, double *rt, int type, AQD2 *qd)
{
  int did = phi_t_aqd2(p, rt, type, qd);
  *p *= -qd->k2[did];
  return did;
}

/* pv_s_aqd2 = pv_s_dbieq_aqd2, or pv_s_bieq_aqd2 near the boundary, where a
 * component of grad F exceeds CBD_CDF (bem3_aw_qd2_field.c:128-144, 231-297). */
int pv_s_aqd2(double complex *p, double complex *pv, double *rt, int type, AQD2 *qd)
{
  double o[18];
  double complex ce;
  int did = field_sums(o, &ce, rt, type, 0, qd);
  double iC = 1.0 / (did == 0 ? 1.0 + o[8] : o[8]);
  double complex P = FS_S0(o);
  if (fabs(o[9]) > AQD2_CBD_CDF || fabs(o[10]) > AQD2_CBD_CDF || fabs(o[11]) > AQD2_CBD_CDF) {
    /* pv_s_bieq_aqd2: the potential sums with the first-derivative Green's function */
    field_sums(o, &ce, rt, type, BEMGPU_FIELD_POTENTIAL, qd);
    iC = 1.0 / (did == 0 ? 1.0 + o[8] : o[8]);
    P = FS_S0(o);
    *p = -qd->k2[did] * P * iC;
    for (int i = 0; i < 3; i++) pv[i] = FS_S2(o, i) * iC;
  } else {
    *p = -qd->k2[did] * P * iC;
    for (int i = 0; i < 3; i++) pv[i] = -(FS_S1(o, i) - P * o[9 + i]) * iC;
  }
  *p *= ce;
  for (int i = 0; i < 3; i++) pv[i] *= ce;
  return did;
}

int pv_t_aqd2(double complex *p, double complex *pv, double *rt, int type, AQD2 *qd)
{
  double complex pi, vi[3];
  int did = pv_s_aqd2(p, pv, rt, type, qd);
  if (did == 0) {
    calc_apw_pv(&pi, vi, rt, &qd->pw);
    *p += pi;
    for (int l = 0; l < 3; l++) pv[l] += vi[l];
  }
  return did;
}

/* Boundary sums at (zeta_t, eta_t) of element t (1-based) of domain did
 * (bem3_aw_qd2_field.c:299-492).  o = bemgpu_boundary_field's 9 values. */
static void bd_sums(double o[9], double *rt, int did, int t, double zeta_t, double eta_t, int type, AQD2 *qd)
{
  if (did < 0 || did > qd->MN || t < 1 || t > qd->bd.sb[did].Ne) {
    printf("bem3_aw_qd2: boundary point of element %d in domain %d is out of range. Exit...\n", t, did);
    exit(1);
  }
  if (type < 0 || type > 3) {
    printf("bem3_aw_qd2: boundary rule type=%d is not available (0..3). Exit...\n", type);
    exit(1);
  }
  bemgpu_ctx *c = ready_ctx(qd);
  int t0 = t - 1;
  double ze[2] = {zeta_t, eta_t};
  gpu_check(c, bemgpu_boundary_field(c, did, type, 1, &t0, ze, o), "boundary field");
  status_check(c, "boundary field");
  aqd2_r_bd(rt, abs(qd->bd.sb[did].sid[t]), zeta_t, eta_t, &qd->bd);
}

void phi_s_bd_aqd2(double complex *phi, int did, int t, double zeta_t, double eta_t, int type, AQD2 *qd)
{
  double o[9], rt[3];
  bd_sums(o, rt, did, t, zeta_t, eta_t, type, qd);
  *phi = (o[0] + I * o[1]) / (did == 0 ? 1.0 + o[8] : o[8]);
}

void phi_t_bd_aqd2(double complex *phi, int did, int t, double zeta_t, double eta_t, int type, AQD2 *qd)
{
  double o[9], rt[3];
  double complex pi, v[3];
  bd_sums(o, rt, did, t, zeta_t, eta_t, type, qd);
  *phi = (o[0] + I * o[1]) / (did == 0 ? 1.0 + o[8] : o[8]);
  if (did == 0) {
    calc_apw_pv(&pi, v, rt, &qd->pw);
    *phi += -pi / qd->pw.wd.k2;
  }
}

void phi_i_bd_aqd2(double complex *phi, int did, int t, double zeta_t, double eta_t, int type, AQD2 *qd)
{
  double complex v[3];
  double rt[3];
  (void)type;
  if (did == 0) {
    aqd2_r_bd(rt, abs(qd->bd.sb[did].sid[t]), zeta_t, eta_t, &qd->bd);
    calc_apw_pv(phi, v, rt, &qd->pw);
    *phi /= -qd->pw.wd.k2;
  } else
    *phi = 0.0;
}

void pv_s_bd_aqd2(double complex *p, double complex *pv, int did, int t, double zeta_t, double eta_t, int type, AQD2 *qd)
{
  double o[9], rt[3];
  bd_sums(o, rt, did, t, zeta_t, eta_t, type, qd);
  double cf = 1.0 / (did == 0 ? 1.0 + o[8] : o[8]);
  *p = -(o[0] + I * o[1]) * cf * qd->k2[did];
  for (int l = 0; l < 3; l++) pv[l] = (o[2 + 2 * l] + I * o[3 + 2 * l]) * cf;
}

void pv_t_bd_aqd2(double complex *p, double complex *pv, int did, int t, double zeta_t, double eta_t, int type, AQD2 *qd)
{
  double o[9], rt[3];
  double complex pi, vi[3];
  bd_sums(o, rt, did, t, zeta_t, eta_t, type, qd);
  double cf = 1.0 / (did == 0 ? 1.0 + o[8] : o[8]);
  *p = -(o[0] + I * o[1]) * cf * qd->k2[did];
  for (int l = 0; l < 3; l++) pv[l] = (o[2 + 2 * l] + I * o[3 + 2 * l]) * cf;
  if (did == 0) {
    calc_apw_pv(&pi, vi, rt, &qd->pw);
    *p += pi;
    for (int l = 0; l < 3; l++) pv[l] += vi[l];
  }
}

void pv_i_bd_aqd2(double complex *p, double complex *pv, int did, int t, double zeta_t, double eta_t, int type, AQD2 *qd)
{
  double rt[3];
  (void)type;
  if (did == 0) {
    aqd2_r_bd(rt, abs(qd->bd.sb[did].sid[t]), zeta_t, eta_t, &qd->bd);
    calc_apw_pv(p, pv, rt, &qd->pw);
  } else {
    *p = 0.0;
    for (int i = 0; i < 3; i++) pv[i] = 0.0;
  }
}

/* Solid-angle domain test (bem3_aw_qd2.c:130-183, 1148-1257): the sum of the
 * solid angles subtended by a domain's boundary is 4 pi inside, 0 outside. */
static int vnorm(double *v)
{
  double a = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  if (a == 0.0) return -1;
  v[0] /= a; v[1] /= a; v[2] /= a;
  return 0;
}
static void cross(double *r, const double *a, const double *b)
{
  r[0] = a[1] * b[2] - a[2] * b[1];
  r[1] = a[2] * b[0] - a[0] * b[2];
  r[2] = a[0] * b[1] - a[1] * b[0];
}
static double dot(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* signed solid angle of the spherical triangle (r0, r1, r2) of unit vectors */
static double tri_angle(const double *r0, const double *r1, const double *r2, int *on)
{
  double n01[3], n12[3], n20[3], nt[3];
  cross(n01, r0, r1);
  cross(n12, r1, r2);
  cross(n20, r2, r0);
  cross(nt, n01, n20);
  double a0 = atan2(sqrt(dot(nt, nt)), -dot(n01, n20));
  cross(nt, n12, n01);
  double a1 = atan2(sqrt(dot(nt, nt)), -dot(n12, n01));
  cross(nt, n20, n12);
  double a2 = atan2(sqrt(dot(nt, nt)), -dot(n20, n12));
  double D = dot(r0, n12);
  if (D > 0.0) return a0 + a1 + a2 - M_PI;
  if (D < 0.0) return -(a0 + a1 + a2 - M_PI);
  *on = 1;
  return 0.0;
}

static int domain_id_home(double *rt, AQD2 *qd)
{
  int nd = qd->MN + 1;
  double *Og = aqd2_calloc(nd, sizeof(double), "Og");
  for (int d = 0; d < nd; d++) {
    for (int i = 1; i <= qd->bd.sb[d].Ne; i++) {
      int e = qd->bd.sb[d].sid[i];
      if (e <= 0) continue;
      int nv = qd->bd.ed[e][3] == 0 ? 3 : 4, on = 0;
      double r[4][3];
      for (int j = 0; j < nv; j++) {
        for (int k = 0; k < 3; k++) r[j][k] = qd->bd.rn[qd->bd.ed[e][j]][k] - rt[k];
        if (vnorm(r[j]) < 0) on = 1;
      }
      double om = 0.0;
      if (!on) {
        om = tri_angle(r[0], r[1], r[2], &on);
        if (!on && nv == 4) om += tri_angle(r[0], r[2], r[3], &on);
      }
      if (on) { free(Og); return d; }
      Og[d] += om;
      Og[qd->bd.sd[e]] -= om;
    }
    if ((d == 0 && fabs(Og[d]) < 2.0 * M_PI) || Og[d] > 2.0 * M_PI) { free(Og); return d; }
  }
  free(Og);
  return -1;
}

int domain_id_aqd2(double *ro, AQD2 *qd)
{
  if (qd->bd.ps == 0) return domain_id_home(ro, qd);
  int l1, l2;
  double rt[3];
  domain_id_l_aqd2(&l1, &l2, ro, qd);
  rt[0] = ro[0] - l1 * qd->bd.qd.vd1[0] - l2 * qd->bd.qd.vd2[0];
  rt[1] = ro[1] - l1 * qd->bd.qd.vd1[1] - l2 * qd->bd.qd.vd2[1];
  rt[2] = ro[2];
  return domain_id_home(rt, qd);
}
