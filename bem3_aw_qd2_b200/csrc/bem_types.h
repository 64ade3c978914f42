/* Plain-C types shared by the host library (C99) and the CUDA kernels.
 *
 * Element tables follow the reference's element constants
 * (d3qd2_src/d3qd2_elem.h:22-45, filled by init_elem_const,
 * d3qd2_src/bem3_aw_qd2.c:941-1023), flattened to contiguous arrays indexed by
 * (absolute element id - 1):
 *   cr [e][3][4]  r(zeta,eta) = cr0 + cr1 zeta + cr2 eta + cr3 zeta eta
 *   cw [e][3][3]  W(zeta,eta) = cw0 + cw1 zeta + cw2 eta   (normal, |W| = Jacobian)
 *   ren[e][4][3]  collocation node coordinates (zeta,eta = +-1/sqrt(3))
 *   wen[e][4][3]  W at the collocation nodes
 */
#ifndef BEM_TYPES_H
#define BEM_TYPES_H

/* geometry of the per-problem table of the real-space Ewald term factors
 * A(y), B(y) (bem_qpgf.cuh): 9 Chebyshev terms on each of 128 intervals of
 * width 1/16 in y in [0, 8); truncation below 5e-17 of the largest value
 * (checked against 30-digit arithmetic), so the table adds nothing to the
 * double rounding */
#define BEM_WT_DEG 9
#define BEM_WT_H 0.0625
#define BEM_WT_N 128
#define BEM_WT_SIZE (2 * BEM_WT_DEG * BEM_WT_N) /* doubles: BEM_WT_DEG x BEM_WT_N complex */
#define BEM_WT_SMEM (BEM_WT_SIZE * 8)           /* its bytes (a kernel's shared-memory copy) */
/* per-problem table of the spectral orders (bem_qpgf.cuh): for each order
 * (n1, n2) of a window around the row centres, 10 Chebyshev terms on
 * intervals of width 1/8 in z / (2 eta_run), two channels */
#define BEM_ST_DEG 10
#define BEM_ST_H 0.125
#define BEM_ST_W 8  /* orders n1 - nc1 and n2 - (row centre) in [-8, 8] */

#ifdef __cplusplus
extern "C" {
#endif

/* Lattice / Bloch data for the quasi-periodic Green's function (the reference's
 * QPD2, qgf2_src/d3_qpgf_d2.h:32-36) plus quantities derived once per
 * (k, k_par, lattice) by bem_qp_prepare(). */
#define BEM_PZ_MAX 24

typedef struct bem_qp {
  double k, kx, ky;             /* wave number and in-plane Bloch wave vector */
  double d1x, d1y, d2x, d2y;    /* lattice vectors */
  double det, idet, aidet;      /* det = d1 x d2, 1/det, |1/det| */
  double g1x, g1y, g2x, g2y;    /* reciprocal lattice vectors */
  double d2sq, g2sq, g1g2;      /* |d2|^2, |g2|^2, g1.g2 */
  double eta0;                  /* the reference's Ewald splitting parameter (before the per-point cap) */
  double eta_run;               /* the one used off the lattice plane (eta0 unless tuned) */
  double sel_cp, sel_bp;        /* spectral-only test: bN/bNp, bNp  */
  double sel_cm, sel_bm;        /*                     bN/bNm, bNm  */
  int nc1;                      /* round(k_par . d1 / 2 pi) */
  int ewald_only;               /* 1: always use the Ewald sum */
  /* optional table of the real-space term factors (A, B) at ve = eta_run,
     x = k eta_run: piecewise Chebyshev, wt_n intervals of width wt_h on
     y in [0, wt_n wt_h), BEM_WT_DEG (A, B) coefficients each; NULL: none */
  const double *wt;
  double wt_h;
  int wt_n;
  /* optional table of the spectral orders at ve = eta_run: orders n1 in
     [st_n1lo, st_n1lo + st_n1cnt), n2 in [st_n2lo, st_n2lo + st_n2cnt),
     st_nint intervals of width BEM_ST_H covering d = z / (2 eta_run) in
     [-st_nint BEM_ST_H / 2, st_nint BEM_ST_H / 2), BEM_ST_DEG coefficient
     pairs each (two channels per order); NULL: none */
  const double *st;
  int st_n1lo, st_n1cnt, st_n2lo, st_n2cnt, st_nint;
  /* residues ef Re w - 1 of the propagating spectral orders (pz_n1, pz_n2) on
     the lattice plane at eta0; pz_n = -1: more orders than the table holds */
  int pz_n;
  int pz_n1[BEM_PZ_MAX], pz_n2[BEM_PZ_MAX];
  double pz_d[BEM_PZ_MAX];
} bem_qp;

/* status word bits written by the kernels (never trapped on the device) */
#define BEM_ST_QPGF_LIMIT   0x01  /* a lattice sum reached its term limit */
#define BEM_ST_RAYLEIGH     0x02  /* beta_n == 0 (Rayleigh anomaly) */
#define BEM_ST_NEAR_OVERFLOW 0x04 /* more near-singular sources in a row than the table holds */
#define BEM_ST_NONFINITE    0x08  /* a non-finite coefficient was produced */
#define BEM_ST_GEOMETRY     0x10  /* negative polar radius in a singular integral */
#define BEM_ST_SOLVE        0x20  /* singular matrix in a factorisation */

#ifdef __cplusplus
}
#endif
#endif
