// Device implementation of the Faddeeva function w(z) and of the doubly
// quasi-periodic Helmholtz Green's function G_qp(r) with its gradient.
//
// Both follow the reference's numerical definitions so that the assembled
// matrices agree with the reference to round-off:
//   * w(z) = exp(-z^2) erfc(-iz): computed from the published Zaghloul & Ali
//     series (ACM TOMS 38(2) 2011, "Algorithm 916") for moderate |z| and the
//     Laplace continued fraction (term count from Poppe & Wijers, ACM TOMS 16
//     1990) for large |z|, with the reflection w(z) = 2 exp(-z^2) - w(-z) in the
//     lower half plane.  The requested relative error is the reference's
//     1e-15 (d3qd2_const.h:33 MEPS, passed to Faddeeva_w at
//     qgf2_src/d3_qpgf_d2.c:1835,1993).  erfcx() and erfc() are CUDA's.
//   * G_qp: the reference's selection between the Ewald sum and the pure
//     spectral sum (d3_qpgf_d2.c:124-176), its reduction of r to the home cell
//     and Bloch phase (d3_qpgf_d2.c:409-438, 286-317), its Ewald split
//     parameter with the per-point cap (d3_qpgf_d2.c:1680-1693), and its
//     adaptive truncation of every lattice sum, term by term
//     (d3_qpgf_d2.c:1714-2009 Ewald, 745-885 spectral; stopping tests
//     d3hm_sf_comp_z / d3hm_sf_diff_z at :471-482).
//
// One thread evaluates one point: the lattice loops are short (about 50 real
// space + 50 spectral terms) and every term is FP64 transcendental work, so the
// kernels are bound by the FP64 pipe, not by memory.
#pragma once
#include <cuda_runtime.h>
#include <math_constants.h>
#include "bem_types.h"

#define BEM_MEPS 1.0e-15       // requested relative error of every lattice sum
#define BEM_EFS 0.1            // term test factor, d3_qpgf_d2.h:29
#define BEM_EW_LIMIT 100       // d3_qpgf_d2.h:25
#define BEM_FD_LIMIT 100       // d3_qpgf_d2.h:22
#define BEM_EW_EXPM 3.0        // d3_qpgf_d2.h:26
#define BEM_S_LIMIT 15         // d3_qpgf_d2.h:19
#define BEM_W_TAB 48           // exp(-a^2 n^2) table length
#define BEM_FD_MAX_TERMS 250.0 // spectral-only sum used when it needs fewer terms than this
#define BEM_WT_DEG 14          // Chebyshev terms per interval of the w(x + i y) table
#define BEM_WT_H 0.125         // interval width in y
#define BEM_WT_N 64            // intervals: y in [0, 8)

// Algorithm 916 constants for relerr = 1e-15: a = pi / sqrt(-ln(relerr/2)),
// c = 2a/pi, tab[n-1] = exp(-a^2 n^2).  Filled once by bem_device_init().
struct bem_wconst {
  double a, a2, c, relerr;
  double tab[BEM_W_TAB];
};
// one copy per translation unit; each .cu that launches QPGF kernels uploads it
static __constant__ bem_wconst c_w;

// ---------------------------------------------------------------- complex
struct cplx { double re, im; };
__device__ __forceinline__ cplx cmk(double r, double i) { cplx z; z.re = r; z.im = i; return z; }
__device__ __forceinline__ cplx cadd(cplx a, cplx b) { return cmk(a.re + b.re, a.im + b.im); }
__device__ __forceinline__ cplx csub(cplx a, cplx b) { return cmk(a.re - b.re, a.im - b.im); }
__device__ __forceinline__ cplx cmul(cplx a, cplx b) { return cmk(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
__device__ __forceinline__ cplx cscale(cplx a, double s) { return cmk(a.re * s, a.im * s); }
__device__ __forceinline__ cplx cexpi(double t) { double s, c; sincos(t, &s, &c); return cmk(c, s); }

// ---------------------------------------------------------------- Faddeeva
__device__ __forceinline__ double bem_sinc(double x, double sinx) {
  return fabs(x) < 1e-4 ? 1.0 - x * x * (1.0 / 6.0) : sinx / x;
}

// w(z) for z = xr + i yi.
__device__ __noinline__ cplx bem_faddeeva(double xr, double yi) {
  if (xr == 0.0) return cmk(erfcx(yi), xr);  // w(iy) = erfcx(y), keep the sign of 0
  const double x = fabs(xr), ya = fabs(yi);
  if (ya >= 7.0 || (x >= 6.0 && ya >= 0.1)) {
    // Laplace continued fraction  w(z) = (i/sqrt(pi)) / (z - (1/2)/(z - 1/(z - (3/2)/(z - ...))))
    // evaluated for the upper-half-plane point zs = z (y >= 0) or -z (y < 0).
    const double xs = yi < 0.0 ? -xr : xr;
    const double rho = sqrt((x / 6.3) * (x / 6.3) + (ya / 4.4) * (ya / 4.4));
    int nu = (int)(3.0 + 1442.0 / (26.0 * rho + 77.0)) + 2;
    double wr = xs, wi = ya;
    for (int m = nu; m >= 1; --m) {
      const double h = 0.5 * m / (wr * wr + wi * wi);
      wr = xs - wr * h;
      wi = ya + wi * h;
    }
    const double d = (1.0 / 1.7724538509055160273) / (wr * wr + wi * wi);
    cplx w = cmk(d * wi, d * wr);
    if (yi < 0.0) {  // w(z) = 2 exp(-z^2) - w(-z);  -z^2 = (y^2 - x^2) + 2 i xs y
      const double e = 2.0 * exp((ya - xs) * (ya + xs));
      double s, c;
      sincos(2.0 * xs * yi, &s, &c);
      w = cmk(e * c - w.re, e * s - w.im);
    }
    return w;
  }
  const double a = c_w.a, cc = c_w.c, relerr = c_w.relerr;
  const double y = yi, y2 = y * y;
  double sum1 = 0.0, sum2 = 0.0, sum3 = 0.0, sum4 = 0.0, sum5 = 0.0;
  double expx2;
  if (x < 10.0) {
    // Zaghloul-Ali sums over n >= 1 of exp(-a^2 n^2 - x^2)/(a^2 n^2 + y^2) times
    // 1, exp(-2anx), exp(+2anx) and the a n weighted versions.
    expx2 = exp(-x * x);
    const double e2 = exp(2.0 * a * x), em2 = 1.0 / e2;
    const bool tiny = x < 1e-3;  // sum5 - sum4 would cancel: use sinh directly
    double pp = 1.0, pm = 1.0, dsum = 0.0;
    for (int n = 1; n < 4 * BEM_W_TAB; ++n) {
      const double an = a * n;
      const double ea = n <= BEM_W_TAB ? c_w.tab[n - 1] : exp(-an * an);
      const double coef = ea * expx2 / (an * an + y2);
      pp *= e2;
      pm *= em2;
      sum1 += coef;
      sum2 += coef * pm;
      sum3 += coef * pp;
      if (tiny) {
        dsum += coef * an * 2.0 * sinh(2.0 * an * x);
        if (coef * pp < relerr * sum3) break;
      } else {
        sum4 += coef * pm * an;
        sum5 += coef * pp * an;
        if (coef * pp * an < relerr * sum5) break;
      }
    }
    if (tiny) { sum4 = 0.0; sum5 = dsum; }
  } else {
    // x >= 10 and |y| < 0.1: only the terms near n0 = x/a matter
    expx2 = exp(-x * x);
    const int n0 = (int)floor(x / a + 0.5);
    for (int n = max(1, n0 - 16); n <= n0 + 16; ++n) {
      const double an = a * n, dx = an - x;
      const double t = exp(-dx * dx) / (an * an + y2);
      sum3 += t;
      sum5 += an * t;
    }
  }
  const double ex2erfcx = y > -6.0 ? expx2 * erfcx(y) : 2.0 * exp(y2 - x * x);
  double sxy, s2xy, c2xy;
  sxy = sin(xr * y);
  sincos(2.0 * xr * y, &s2xy, &c2xy);
  const double coef1 = ex2erfcx - cc * y * sum1;
  const double coef2 = cc * xr * expx2;
  const double re = coef1 * c2xy + coef2 * sxy * bem_sinc(xr * y, sxy) + 0.5 * cc * y * (sum2 + sum3);
  const double im = coef2 * bem_sinc(2.0 * xr * y, s2xy) - coef1 * s2xy + 0.5 * cc * copysign(sum5 - sum4, xr);
  return cmk(re, im);
}

// ---------------------------------------------------------------- QPGF
// Relative "unchanged" test on a running sum (d3hm_sf_comp_z, d3_qpgf_d2.c:471)
__device__ __forceinline__ bool bem_same(cplx v1, cplx v2, double eps) {
  return 2.0 * fabs(v1.re - v2.re) <= eps * (fabs(v1.re) + fabs(v2.re)) &&
         2.0 * fabs(v1.im - v2.im) <= eps * (fabs(v1.im) + fabs(v2.im));
}
// Negligible-term test (d3hm_sf_diff_z, d3_qpgf_d2.c:478)
__device__ __forceinline__ bool bem_small(cplx t, cplx s, double eps) {
  return fabs(t.re) <= fabs(s.re) * BEM_EFS * eps && fabs(t.im) <= fabs(s.im) * BEM_EFS * eps;
}

struct bem_gval { cplx g, gx, gy, gz; };

// w(x + i y) from the per-problem table (x = k eta0, 0 <= y < 8): Clenshaw
// recurrence on the interval's Chebyshev series.  Terms with y >= 8 are below
// 1e-27 of the leading one and never reached by the stopping rule; they fall
// back to the direct evaluation.
__device__ __forceinline__ cplx bem_wtab(const bem_qp &q, double x, double y) {
  const double u = y * (1.0 / BEM_WT_H);
  const int j = (int)u;
  if (j >= q.wt_n) return bem_faddeeva(x, y);
  const double t = 2.0 * (u - j) - 1.0, t2 = 2.0 * t;
  const double2 *c = reinterpret_cast<const double2 *>(q.wt) + (size_t)j * BEM_WT_DEG;
  double br = 0.0, bi = 0.0, b1r = 0.0, b1i = 0.0;
#pragma unroll
  for (int k = BEM_WT_DEG - 1; k >= 1; --k) {
    const double2 ck = __ldg(c + k);
    const double nr = ck.x + t2 * br - b1r, ni = ck.y + t2 * bi - b1i;
    b1r = br; b1i = bi;
    br = nr; bi = ni;
  }
  const double2 c0 = __ldg(c);
  return cmk(c0.x + t * br - b1r, c0.y + t * bi - b1i);
}

// Ewald real-space term for lattice point (l1,l2)  (ew_qG1_v1_cFl, d3_qpgf_d2.c:1814).
// ce = exp(i k_par . R_l) is supplied by the caller, which advances it along the
// row by one complex multiplication per term instead of a sincos.
__device__ __forceinline__ void ew_real_term(const bem_qp &q, double px, double py, double rz, cplx ce,
                                             double ke, double ke2, double ive, bool tab, cplx &F, cplx &cf) {
  const double rl = sqrt(px * px + py * py + rz * rz);
  const double irl = 1.0 / rl;
  const double rl2e = rl * 0.5 * ive;
  const double ef = exp(ke2 - rl2e * rl2e);
  const cplx w = tab ? bem_wtab(q, ke, rl2e) : bem_faddeeva(ke, rl2e);
  F = cscale(ce, irl * ef * w.re);
  cf = cscale(ce, irl * irl * ef * (irl * w.re - q.k * w.im + ive * 0.56418958354775628695));
}

// Ewald spectral term for reciprocal point (n1,n2) (ew_qG2_v1_cFn, d3_qpgf_d2.c:1965);
// ce = exp(i alpha_n . r) supplied by the caller (recurrence along n2).
// returns 0 propagating, 1 evanescent, -3 beta_n == 0
__device__ __forceinline__ int ew_spec_term(const bem_qp &q, double anx, double any, double rz, cplx ce,
                                            double ve, cplx &Fn, cplx &dF0, cplx &dF1, cplx &dF2) {
  const double bn2 = q.k * q.k - anx * anx - any * any;
  const double azve = rz / (2.0 * ve);
  if (bn2 > 0.0) {
    const double bn = sqrt(bn2);
    const double ef = exp(bn2 * ve * ve - azve * azve);
    const cplx ff = cexpi(bn * rz);
    const cplx w = bem_faddeeva(bn * ve, azve);
    // Fn = 2 ce / bn (i ef Im w + ff)
    Fn = cscale(cmul(ce, cmk(ff.re, ef * w.im + ff.im)), 2.0 / bn);
    dF0 = cscale(Fn, anx);
    dF1 = cscale(Fn, any);
    dF2 = cscale(cmul(ce, cmk(ef * w.re - ff.re, -ff.im)), 2.0);
    return 0;
  } else if (bn2 < 0.0) {
    const double bn = sqrt(-bn2);
    const double ebz = exp(bn * rz);
    const double f1 = ebz * erfc(bn * ve + azve);
    const double f2 = erfc(bn * ve - azve) / ebz;
    // Fn = ce / (i bn) (f1 + f2)
    Fn = cmul(ce, cmk(0.0, -(f1 + f2) / bn));
    dF0 = cscale(Fn, anx);
    dF1 = cscale(Fn, any);
    dF2 = cscale(ce, f1 - f2);
    return 1;
  }
  return -3;
}

__device__ __forceinline__ cplx cconj(cplx a) { return cmk(a.re, -a.im); }

// Ewald evaluation in the home cell (d3hm_qpgf_d2v1_ew_sd, d3_qpgf_d2.c:1671).
// Returns the number of lattice terms, or a negative reference error code.
// The lattice rows are walked exactly as in the reference (centre, then up,
// then down, each stopped by the reference's tests); the Bloch phases along a
// row are advanced by a unit complex factor, so a row costs one sincos.
__device__ int bem_qpgf_ewald(const bem_qp &q, double rx, double ry, double rz, bem_gval &out) {
  double ve = q.eta0;
  const double r2 = rx * rx + ry * ry + rz * rz;
  if (q.k * q.k * ve * ve - r2 / (4.0 * ve * ve) > BEM_EW_EXPM)
    ve = sqrt(BEM_EW_EXPM + sqrt(q.k * q.k * r2 + BEM_EW_EXPM * BEM_EW_EXPM)) / (1.4142135623730950488 * q.k);
  const double ke = q.k * ve, ke2 = ke * ke, ive = 1.0 / ve;
  const bool tab = q.wt != nullptr && ve == q.eta0;  // table built for x = k eta0
  const double eps = BEM_MEPS;
  int cc = 0;
  const cplx E2 = cexpi(q.kx * q.d2x + q.ky * q.d2y);  // exp(i k_par . d2)

  // ---- real-space sum (ew_qG1_v1, :1714-1812)
  cplx s = cmk(0, 0), sx = cmk(0, 0), sy = cmk(0, 0), sz = cmk(0, 0);
  for (int dir = 0; dir < 3; ++dir) {
    // dir 0: the row l1 = 0; dir 1: l1 = 1, 2, ...; dir 2: l1 = -1, -2, ...
    int l1 = dir == 2 ? -1 : (dir == 1 ? 1 : 0);
    const int step = dir == 2 ? -1 : 1;
    bool done = false;
    for (int it = 0; it < (dir == 0 ? 1 : BEM_EW_LIMIT - 1); ++it, l1 += step) {
      const cplx old = s;
      const int lc = -(int)round(((rx + l1 * q.d1x) * q.d2x + (ry + l1 * q.d1y) * q.d2y) / q.d2sq);
      const cplx pc = cexpi(q.kx * (l1 * q.d1x + lc * q.d2x) + q.ky * (l1 * q.d1y + lc * q.d2y));
      // centre term, then l2 > lc, then l2 < lc
      for (int side = 0; side < 3; ++side) {
        int l2 = side == 0 ? lc : (side == 1 ? lc + 1 : lc - 1);
        const int st = side == 2 ? -1 : 1;
        const cplx E = side == 2 ? cconj(E2) : E2;
        cplx ce = side == 0 ? pc : cmul(pc, E);
        const int nmax = side == 0 ? 1 : BEM_EW_LIMIT - 1;
        int k = 0;
        for (; k < nmax; ++k, l2 += st) {
          const double px = rx + l1 * q.d1x + l2 * q.d2x, py = ry + l1 * q.d1y + l2 * q.d2y;
          cplx F, cf;
          ew_real_term(q, px, py, rz, ce, ke, ke2, ive, tab, F, cf);
          ++cc;
          s = cadd(s, F);
          sx = cadd(sx, cscale(cf, px));
          sy = cadd(sy, cscale(cf, py));
          sz = cadd(sz, cf);
          if (side != 0 && bem_small(F, s, eps)) break;
          ce = cmul(ce, E);
        }
        if (side != 0 && k == nmax) return -21;
      }
      if (dir != 0 && bem_same(s, old, eps)) { done = true; break; }
    }
    if (dir != 0 && !done) return -21;
  }
  const double i4p = 0.07957747154594766788;  // 1/(4 pi)
  out.g = cscale(s, i4p);
  out.gx = cscale(sx, -i4p);
  out.gy = cscale(sy, -i4p);
  out.gz = cscale(sz, -rz * i4p);

  // ---- spectral sum (ew_qG2_v1, :1840-1963)
  const cplx G2 = cexpi(q.g2x * rx + q.g2y * ry);  // exp(i g2 . r)
  cplx t = cmk(0, 0), tx = cmk(0, 0), ty = cmk(0, 0), tz = cmk(0, 0);
  for (int dir = 0; dir < 3; ++dir) {
    int n1 = q.nc1 + (dir == 2 ? -1 : (dir == 1 ? 1 : 0));
    const int step = dir == 2 ? -1 : 1;
    bool done = false;
    for (int it = 0; it < (dir == 0 ? 1 : BEM_EW_LIMIT - 1); ++it, n1 += step) {
      const cplx old = tz;
      const int nc = (int)round(-((-q.kx + n1 * q.g1x) * q.g2x + (-q.ky + n1 * q.g1y) * q.g2y) / q.g2sq);
      const double a0x = -q.kx + n1 * q.g1x, a0y = -q.ky + n1 * q.g1y;
      const cplx pc = cexpi((a0x + nc * q.g2x) * rx + (a0y + nc * q.g2y) * ry);
      int flg = 0;
      for (int side = 0; side < 3; ++side) {
        int n2 = side == 0 ? nc : (side == 1 ? nc + 1 : nc - 1);
        const int st = side == 2 ? -1 : 1;
        const cplx E = side == 2 ? cconj(G2) : G2;
        cplx ce = side == 0 ? pc : cmul(pc, E);
        const int nmax = side == 0 ? 1 : BEM_EW_LIMIT - 1;
        int k = 0;
        for (; k < nmax; ++k, n2 += st) {
          cplx Fn, d0, d1, d2;
          const int e = ew_spec_term(q, a0x + n2 * q.g2x, a0y + n2 * q.g2y, rz, ce, ve, Fn, d0, d1, d2);
          if (e < 0) return -23;
          ++cc;
          t = cadd(t, Fn);
          tx = cadd(tx, d0);
          ty = cadd(ty, d1);
          tz = cadd(tz, d2);
          if (side != 0) {
            if (e > 0) { if (bem_small(d2, tz, eps)) break; }
            else ++flg;
          }
          ce = cmul(ce, E);
        }
        if (side != 0 && k == nmax) return -22;
      }
      if (dir != 0 && flg == 0 && bem_same(tz, old, eps)) { done = true; break; }
    }
    if (dir != 0 && !done) return -22;
  }
  const double c2 = 0.25 * q.aidet;
  out.g = cadd(out.g, cmul(t, cmk(0.0, c2)));
  out.gx = cadd(out.gx, cscale(tx, -c2));
  out.gy = cadd(out.gy, cscale(ty, -c2));
  out.gz = cadd(out.gz, cscale(tz, c2));
  return cc;
}

// Pure spectral sum in the home cell (d3hm_qpgf_d2v1_fd_sd, d3_qpgf_d2.c:745-885).
__device__ int bem_qpgf_spectral(const bem_qp &q, double rx, double ry, double rz, bem_gval &out) {
  if (rz == 0.0) return -14;
  const double eps = BEM_MEPS, az = fabs(rz);
  int cc = 0;
  const cplx G2 = cexpi(q.g2x * rx + q.g2y * ry);  // exp(i g2 . r)
  cplx t = cmk(0, 0), tx = cmk(0, 0), ty = cmk(0, 0), tz = cmk(0, 0);
  for (int dir = 0; dir < 3; ++dir) {
    int n1 = q.nc1 + (dir == 2 ? -1 : (dir == 1 ? 1 : 0));
    const int step = dir == 2 ? -1 : 1;
    bool done = false;
    for (int it = 0; it < (dir == 0 ? 1 : BEM_FD_LIMIT - 1); ++it, n1 += step) {
      const cplx old = tz;
      const int nc = (int)round((q.kx * q.g2x + q.ky * q.g2y - n1 * q.g1g2) / q.g2sq);
      const double a0x = -q.kx + n1 * q.g1x, a0y = -q.ky + n1 * q.g1y;
      const cplx pc = cexpi((a0x + nc * q.g2x) * rx + (a0y + nc * q.g2y) * ry);
      for (int side = 0; side < 3; ++side) {
        int n2 = side == 0 ? nc : (side == 1 ? nc + 1 : nc - 1);
        const int st = side == 2 ? -1 : 1;
        const cplx E = side == 2 ? cconj(G2) : G2;
        cplx ce = side == 0 ? pc : cmul(pc, E);
        const int nmax = side == 0 ? 1 : BEM_FD_LIMIT - 1;
        int k = 0;
        for (; k < nmax; ++k, n2 += st) {
          const double anx = a0x + n2 * q.g2x;
          const double any = a0y + n2 * q.g2y;
          const double bn2 = q.k * q.k - anx * anx - any * any;
          cplx d2, Fn;
          int e;
          if (bn2 > 0.0) {
            const double bn = sqrt(bn2);
            d2 = cmul(ce, cexpi(bn * az));
            Fn = cscale(d2, 1.0 / bn);
            e = 0;
          } else if (bn2 < 0.0) {
            const double bn = sqrt(-bn2);
            d2 = cscale(ce, exp(-bn * az));
            Fn = cmk(d2.im / bn, -d2.re / bn);  // -i d2 / bn
            e = 1;
          } else {
            return -12;
          }
          ++cc;
          t = cadd(t, Fn);
          tx = cadd(tx, cscale(Fn, anx));
          ty = cadd(ty, cscale(Fn, any));
          tz = cadd(tz, d2);
          if (side != 0 && e > 0 && bem_small(d2, tz, eps)) break;
          ce = cmul(ce, E);
        }
        if (side != 0 && k == nmax) return -11;
      }
      if (dir != 0 && bem_same(tz, old, eps)) { done = true; break; }
    }
    if (dir != 0 && !done) return -11;
  }
  const double c = 0.5 * q.aidet;
  out.g = cmul(t, cmk(0.0, c));
  out.gx = cscale(tx, -c);
  out.gy = cscale(ty, -c);
  out.gz = cscale(tz, -c * (rz > 0 ? 1.0 : -1.0));
  return cc;
}

// G_qp and grad G_qp at r (d3hm_qpgf_d2_v1, d3_qpgf_d2.c:124-176 and the cell
// reduction of :409-438).  Returns #terms (> 0) or the reference's negative code.
__device__ int bem_qpgf(const bem_qp &q, double rx, double ry, double rz, bem_gval &out) {
  bool spectral = false;
  if (!q.ewald_only) {
    const double az = fabs(rz);
    spectral = q.sel_cp * exp(-q.sel_bp * az) < BEM_MEPS && q.sel_cm * exp(-q.sel_bm * az) < BEM_MEPS;
    // Where the reference allows the pure spectral sum, both sums converge to
    // 1e-15 and agree to round-off; keep the spectral one only where it is the
    // cheaper: it needs about (36/|z|)^2 |det| / 4 pi terms (|beta_n| |z| < 36)
    // against ~110 costlier Ewald terms.
    if (spectral && (36.0 / az) * (36.0 / az) * fabs(q.det) * 0.0795774715459476679 > BEM_FD_MAX_TERMS) spectral = false;
  }
  const int l1 = (int)floor((rx * q.d2y - ry * q.d2x) * q.idet + 0.5);
  const int l2 = (int)floor(-(rx * q.d1y - ry * q.d1x) * q.idet + 0.5);
  const double hx = rx - l1 * q.d1x - l2 * q.d2x;
  const double hy = ry - l1 * q.d1y - l2 * q.d2y;
  const int e = spectral ? bem_qpgf_spectral(q, hx, hy, rz, out) : bem_qpgf_ewald(q, hx, hy, rz, out);
  if (e > 0 && (l1 != 0 || l2 != 0)) {
    const cplx cf = cexpi(-(q.kx * (l1 * q.d1x + l2 * q.d2x) + q.ky * (l1 * q.d1y + l2 * q.d2y)));
    out.g = cmul(out.g, cf);
    out.gx = cmul(out.gx, cf);
    out.gy = cmul(out.gy, cf);
    out.gz = cmul(out.gz, cf);
  }
  return e;
}
