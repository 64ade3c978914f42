// Host-side set-up of the lattice data of the quasi-periodic Green's function
// (bem_qp), shared by the context API and the allocation-free entry point.
#pragma once
#include <math.h>
#include <string.h>
#include "bem_types.h"

// Residues ef Re w(bn eta0) - 1 of the propagating spectral orders on the
// lattice plane (z = 0), formed with the reference's own expressions and the
// host C library's exp, as the reference forms them inside every call
// (ew_qG2_v1 / ew_qG2_v1_cFn, qgf2_src/d3_qpgf_d2.c:1840-2009; Faddeeva_w on
// the real axis is exp(-x^2), qgf2_src/Faddeeva.cc:684).  Mathematically 0;
// whether the rounded value is exactly 0 decides where the reference's
// spectral rows stop at z = 0, so the device looks the value up instead of
// recomputing it with its own exp.  Orders beyond BEM_PZ_MAX keep pz_n at -1
// and the device falls back to a correctly rounded exp of its own.
static void bem_plane_residues(bem_qp *q) {
  const double vd1[2] = {q->d1x, q->d1y}, vd2[2] = {q->d2x, q->d2y};
  const double detd = vd1[0] * vd2[1] - vd2[0] * vd1[1];
  const double idd = 1.0 / detd;
  double vg1[2], vg2[2];
  vg1[0] = 2.0 * M_PI * idd * vd2[1];
  vg1[1] = -2.0 * M_PI * idd * vd2[0];
  vg2[0] = -2.0 * M_PI * idd * vd1[1];
  vg2[1] = 2.0 * M_PI * idd * vd1[0];
  const double veps = q->eta0;
  // every order with |a_n| < k lies in this box (n_i = (a_n + k_par) . d_i / 2 pi)
  const double kk = q->k + sqrt(q->kx * q->kx + q->ky * q->ky);
  const int N1 = (int)ceil(kk * sqrt(vd1[0] * vd1[0] + vd1[1] * vd1[1]) / (2.0 * M_PI)) + 1;
  const int N2 = (int)ceil(kk * sqrt(vd2[0] * vd2[0] + vd2[1] * vd2[1]) / (2.0 * M_PI)) + 1;
  int n = 0;
  for (int n1 = -N1; n1 <= N1; ++n1)
    for (int n2 = -N2; n2 <= N2; ++n2) {
      double an[2];
      an[0] = -q->kx + (double)n1 * vg1[0] + (double)n2 * vg2[0];
      an[1] = -q->ky + (double)n1 * vg1[1] + (double)n2 * vg2[1];
      const double bn2 = q->k * q->k - an[0] * an[0] - an[1] * an[1];
      if (!(bn2 > 0.0)) continue;
      if (n == BEM_PZ_MAX) { q->pz_n = -1; return; }
      const double bn = sqrt(bn2);
      const double ef = exp(bn2 * veps * veps - 0.0);
      const double x = bn * veps;
      const double wr = exp(-(x * x));
      q->pz_n1[n] = n1;
      q->pz_n2[n] = n2;
      q->pz_d[n] = ef * wr - 1.0;
      ++n;
    }
  q->pz_n = n;
}

// Lattice quantities derived once per (k, k_par, lattice): the reference
// recomputes them inside every Green's-function call (d3_qpgf_d2.c:126-156,
// 1679-1681, 1850-1856).
static void bem_qp_prepare(const double *p, bem_qp *q) {
  memset(q, 0, sizeof(*q));
  q->k = p[0]; q->kx = p[1]; q->ky = p[2];
  q->d1x = p[4]; q->d1y = p[5]; q->d2x = p[6]; q->d2y = p[7];
  q->det = q->d1x * q->d2y - q->d2x * q->d1y;
  q->idet = 1.0 / q->det;
  q->aidet = fabs(q->idet);
  const double cpd = 2.0 * M_PI * q->idet;
  q->g1x = cpd * q->d2y; q->g1y = -cpd * q->d2x;
  q->g2x = -cpd * q->d1y; q->g2y = cpd * q->d1x;
  q->d2sq = q->d2x * q->d2x + q->d2y * q->d2y;
  q->g2sq = q->g2x * q->g2x + q->g2y * q->g2y;
  q->g1g2 = q->g1x * q->g2x + q->g1y * q->g2y;
  const double adp = sqrt(pow(q->d1x + q->d2x, 2) + pow(q->d1y + q->d2y, 2));
  const double adm = sqrt(pow(q->d1x - q->d2x, 2) + pow(q->d1y - q->d2y, 2));
  q->eta0 = sqrt(fabs(q->det) / (4.0 * M_PI) * adp / adm);
  q->eta_run = q->eta0;
  q->nc1 = (int)round((q->kx * q->d1x + q->ky * q->d1y) / (2.0 * M_PI));
  // choice between the Ewald and the pure spectral sum (d3hm_qpgf_d2_v1)
  const double k2 = q->k * q->k;
  const int n1 = q->nc1, n2 = (int)round((q->kx * q->d2x + q->ky * q->d2y) / (2.0 * M_PI));
  const double ad12 = q->d1x * q->d1x + q->d1y * q->d1y, ad22 = q->d2sq;
  const double aNx = -q->kx + n1 * cpd * q->d2y - n2 * cpd * q->d1y;
  const double aNy = -q->ky - n1 * cpd * q->d2x + n2 * cpd * q->d1x;
  const double bN = sqrt(k2 - aNx * aNx - aNy * aNy);
  double aNpx, aNpy, aNmx, aNmy;
  if (ad22 < ad12) {
    aNpx = -q->kx + (n1 + 15) * cpd * q->d2y - n2 * cpd * q->d1y;
    aNpy = -q->ky - (n1 + 15) * cpd * q->d2x + n2 * cpd * q->d1x;
    aNmx = -q->kx + (n1 - 15) * cpd * q->d2y - n2 * cpd * q->d1y;
    aNmy = -q->ky - (n1 - 15) * cpd * q->d2x + n2 * cpd * q->d1x;
  } else {
    aNpx = -q->kx + n1 * cpd * q->d2y - (n2 + 15) * cpd * q->d1y;
    aNpy = -q->ky - n1 * cpd * q->d2x + (n2 + 15) * cpd * q->d1x;
    aNmx = -q->kx + n1 * cpd * q->d2y - (n2 - 15) * cpd * q->d1y;
    aNmy = -q->ky - n1 * cpd * q->d2x + (n2 - 15) * cpd * q->d1x;
  }
  const double bNp = k2 - aNpx * aNpx - aNpy * aNpy;
  const double bNm = k2 - aNmx * aNmx - aNmy * aNmy;
  if (bNp > 0.0 || bNm > 0.0) {
    q->ewald_only = 1;
  } else {
    q->ewald_only = 0;
    q->sel_bp = sqrt(-bNp);
    q->sel_bm = sqrt(-bNm);
    q->sel_cp = bN / q->sel_bp;
    q->sel_cm = bN / q->sel_bm;
  }
  bem_plane_residues(q);
}
