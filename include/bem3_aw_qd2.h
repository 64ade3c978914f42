/* bem3_aw_qd2.h -- drop-in API of the B200 boundary-element solver.
 *
 * Same functions, argument meaning and data structures as the reference's
 * d3qd2_src/bem3_aw_qd2.h:12-97 (with the structs of d3qd2_elem.h:13-65,
 * aw_pw.h:16-34 and d3_qpgf_d2.h:32-36), so the reference's drivers
 * (aw_d3qd2_bv_solver.c, example1.c) compile against it unchanged.  The
 * structs must keep the reference's member order and types: the .dat file
 * stores AQD2 and Apw as raw bytes (bem3_aw_qd2.c:185-224), sizeof(AQD2) =
 * 2720 and sizeof(Apw) = 240 on x86-64.  Device state lives in a side table,
 * never inside AQD2.
 */
#ifndef BEM3_AW_QD2_H_
#define BEM3_AW_QD2_H_

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <complex.h>
#include <time.h>

/* ---- constants kept from the reference's d3qd2_const.h / d3_qpgf_d2.h */
#define MEPS 1.0e-15
#define GEPS 1.0e-15
#define CDFH 1.0e-3
#define I_FP 7.957747154594766788444e-2
#define OPENDID 99
#define ELT3 2
#define ELT4 3
#define GLN 12
#define GHN 64
#define CBD_CDF 10.0
#define CBD_SDF 0.5

/* incident plane wave (aw_pw.h:16-34) */
typedef struct aw_planewave_adata {
  double omega;           /* angular frequency */
  double K0;              /* bulk modulus rho0 c0^2 */
  double complex k1, k2;  /* k1 = i omega/K0, k2 = i omega rho0 */
  double k0, kx, ky, kz;  /* wave number and wave vector */
  double lambda0;         /* wavelength */
  double R[9];            /* rotation matrix of the propagation axis */
} ApwD;

typedef struct aw_planewave {
  double rho0, c0, f;     /* host medium density, sound speed, frequency */
  double complex p;       /* amplitude */
  double tv[3];           /* translation vector */
  double theta, psi;      /* propagation-axis angles */
  ApwD wd;
} Apw;

/* lattice data of the quasi-periodic Green's function (d3_qpgf_d2.h:32-36) */
typedef struct qp_data_v2 {
  double k;
  double vk[3];
  double vd1[2], vd2[2];
} QPD2;

/* per-domain boundary values (d3qd2_elem.h:13-19) */
typedef struct sub_domain_data {
  int Ne;
  int *sid;                     /* signed element ids, [1..Ne] */
  double complex **P, **dP;     /* [element][node] */
  double complex ***pv, ***dpv; /* [element][node][xyz] */
} SUBD;

/* boundary (d3qd2_elem.h:21-46) */
typedef struct boundary_data {
  int ps;
  QPD2 qd;
  int Nn, Ne;
  double **rn;
  int **ed;
  int NN;
  int **eni;
  int *md, *sd, *gd;
  double ***cr, ***cw;
  double ***ren, ***wen;
  double complex **Pi, **dPi;
  double zt_44[4], et_44[4], wt_44[4], zt_49[9], et_49[9], wt_49[9];
  double zt_34[4], et_34[4], wt_34[4], zt_37[7], et_37[7], wt_37[7];
  double xli[GLN], wli[GLN];
  double xhi[GHN], whi[GHN];
  SUBD *sb;
} BOUD;

/* the solver object (d3qd2_elem.h:48-65) */
typedef struct domain_data {
  char ped_fn[128], med_fn[128], msh_fn[128];
  double rv[3], th;
  double tv[3];
  int MN;
  double *rho0, *c0;
  double *k0, *K0;
  double complex *k1, *k2;
  Apw pw;
  BOUD bd;
} AQD2;

#ifdef __cplusplus
extern "C" {
#endif

/* -- set-up and files (bem3_aw_qd2.c) */
void read_aqd2(int argc, char **argv, AQD2 *qd);
void print_aqd2(AQD2 *qd);
void initialize_aqd2(AQD2 *qd);
void finalize_aqd2(AQD2 *qd);
int domain_id_aqd2(double *rt, AQD2 *qd);
void domain_id_l_aqd2(int *l1, int *l2, double *rt, AQD2 *qd);
void dat_write_aqd2(char *fname, AQD2 *qd);
void dat_read_aqd2(char *fname, AQD2 *qd);

/* -- boundary integral equations (bem3_aw_qd2_solve_bieq.c) */
void solve_bieq_aqd2(AQD2 *qd);

/* -- radiation force (bem3_aw_qd2_force.c) */
void force_FN_aqd2(double *F, double *N, double *rc, int type, AQD2 *qd);
void surface_area_aqd2(double *S, int did, int type, AQD2 *qd);

/* -- fields (bem3_aw_qd2_field.c) */
int phi_s_aqd2(double complex *phi, double *rt, int type, AQD2 *qd);
int phi_t_aqd2(double complex *phi, double *rt, int type, AQD2 *qd);
int phi_i_aqd2(double complex *phi, double *rt, int type, AQD2 *qd);
int p_s_aqd2(double complex *p, double *rt, int type, AQD2 *qd);
int p_t_aqd2(double complex *p, double *rt, int type, AQD2 *qd);
int p_i_aqd2(double complex *p, double *rt, int type, AQD2 *qd);
int pv_s_aqd2(double complex *p, double complex *pv, double *rt, int type, AQD2 *qd);
int pv_t_aqd2(double complex *p, double complex *pv, double *rt, int type, AQD2 *qd);
int pv_i_aqd2(double complex *p, double complex *pv, double *rt, int type, AQD2 *qd);

/* -- boundary values at parameter points of element t (1-based) of domain did
 *    (bem3_aw_qd2_field.c:299-492) */
void phi_s_bd_aqd2(double complex *phi, int did, int t, double zeta_t, double eta_t, int type, AQD2 *qd);
void phi_t_bd_aqd2(double complex *phi, int did, int t, double zeta_t, double eta_t, int type, AQD2 *qd);
void phi_i_bd_aqd2(double complex *phi, int did, int t, double zeta_t, double eta_t, int type, AQD2 *qd);
void pv_s_bd_aqd2(double complex *p, double complex *pv, int did, int t, double zeta_t, double eta_t, int type, AQD2 *qd);
void pv_t_bd_aqd2(double complex *p, double complex *pv, int did, int t, double zeta_t, double eta_t, int type, AQD2 *qd);
void pv_i_bd_aqd2(double complex *p, double complex *pv, int did, int t, double zeta_t, double eta_t, int type, AQD2 *qd);

/* -- plane wave (aw_pw.h) */
void read_data_apw(char *fname, Apw *pw);
void print_data_apw(Apw *pw);
void setup_apw(Apw *pw);
void calc_apw_pv(double complex *p, double complex *v, double *r, Apw *pw);
void calc_apw_dpdn(double complex *p, double complex *dpdn, double *r, double *n, Apw *pw);

/* -- additions of this library (no counterpart in the reference) */
/* GPU device used by solve_bieq_aqd2 / force_FN_aqd2 (default 0). */
void aqd2_set_device(int device);
/* Precision of the dense solves of contexts created afterwards (bemgpu.h
 * BEMGPU_FP64 .. BEMGPU_MIXED_FAST; default 0, or the AQD2_PRECISION
 * environment variable). */
void aqd2_set_precision(int mode);
/* Interior derivative rows of contexts created afterwards kept (1) or
 * recomputed in blocks (0) (bemgpu.h bemgpu_set_interior_derivatives;
 * default 1, or the AQD2_INTERIOR_DERIVATIVES environment variable). */
void aqd2_set_interior_derivatives(int keep);
/* 0: solve_bieq_aqd2 prints nothing (default 1: the reference's progress lines). */
void aqd2_set_verbose(int on);
/* Last wall time of the solve phases in seconds: [0] upload, [1] assembly,
 * [2] solve, [3] download. */
void aqd2_last_timing(double *t4);
/* Flatten an initialised AQD2 into a bemgpu_problem (bemgpu.h) with freshly
 * allocated host arrays, e.g. for the request server; aqd2_problem_free
 * releases them. */
struct bemgpu_problem;
void aqd2_problem_build(AQD2 *qd, struct bemgpu_problem *pr);
void aqd2_problem_free(struct bemgpu_problem *pr);
/* The device context that solve_bieq_aqd2 used for qd (NULL before the first
 * solve); its type is declared in bemgpu.h. */
struct bemgpu_ctx *aqd2_device_context(AQD2 *qd);

#ifdef __cplusplus
}
#endif
#endif
