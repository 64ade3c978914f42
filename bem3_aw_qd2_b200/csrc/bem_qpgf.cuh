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
// |z| below which the spectral rows' stopping tests can meet an exact zero of
// the z-derivative terms (e^{bn z} rounds to 1 for |bn z| < 2^-54): there the
// terms are formed with the reference's rounding and eta0
#define BEM_PLANE_NEAR 1.0e-13
#define BEM_S_LIMIT 15         // d3_qpgf_d2.h:19
#define BEM_W_TAB 48           // exp(-a^2 n^2) table length
#define BEM_FD_MAX_TERMS 250.0 // spectral-only sum used when it needs fewer terms than this

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
#ifndef BEM_FADDEEVA_ATTR
#define BEM_FADDEEVA_ATTR __noinline__
#endif
#ifndef BEM_QPGF_ATTR
#define BEM_QPGF_ATTR
#endif
__device__ BEM_FADDEEVA_ATTR cplx bem_faddeeva(double xr, double yi) {
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

// The real-space Ewald term of a lattice point at distance rl from the
// evaluation point, with x = k ve and y = rl / (2 ve), needs
//   A(y) = e^{x^2 - y^2} Re w(x + i y)
//   B(y) = e^{x^2 - y^2} (Re w / (2 ve) - k y Im w + y / (ve sqrt(pi)))
// (term = A / rl, its radial factor = 2 ve B / rl^3).  Both are functions of y
// alone for a problem's k and ve = eta_run, so they are tabulated once per
// problem (piecewise Chebyshev on [0, 8), coefficients built on the device from
// the Faddeeva function): one Clenshaw recurrence replaces a Faddeeva value and
// an exp per term.  Truncation is below 5e-17 of the largest value (checked
// against 30-digit arithmetic); y >= 8 (terms below 1e-27 of the leading one,
// never reached by the stopping rule) falls back to the direct forms.
__device__ __forceinline__ double2 ew_real_ab(double k, double ve, double x, double y) {
  const cplx w = bem_faddeeva(x, y);
  const double ef = exp(x * x - y * y);
  return make_double2(ef * w.re, ef * (w.re * (0.5 / ve) - k * y * w.im + y * (0.56418958354775628695 / ve)));
}
// wts: the kernel's shared-memory copy of the table (bem_wtab_stage), or null
// to read q.wt through the read-only cache
__device__ __forceinline__ double2 bem_wtab(const bem_qp &q, double ve, double x, double y,
                                            const double2 *wts = nullptr) {
  const double u = y * (1.0 / BEM_WT_H);
  const int j = (int)u;
  if (j >= q.wt_n) return ew_real_ab(q.k, ve, x, y);
  const double t = 2.0 * (u - j) - 1.0, t2 = 2.0 * t;
  double ba = 0.0, bb = 0.0, b1a = 0.0, b1b = 0.0;
  double2 c0;
  if (wts) {
    const double2 *c = wts + j * BEM_WT_DEG;
#pragma unroll
    for (int k = BEM_WT_DEG - 1; k >= 1; --k) {
      const double2 ck = c[k];
      const double na = ck.x + t2 * ba - b1a, nb = ck.y + t2 * bb - b1b;
      b1a = ba; b1b = bb;
      ba = na; bb = nb;
    }
    c0 = c[0];
  } else {
    const double2 *c = reinterpret_cast<const double2 *>(q.wt) + (size_t)j * BEM_WT_DEG;
#pragma unroll
    for (int k = BEM_WT_DEG - 1; k >= 1; --k) {
      const double2 ck = __ldg(c + k);
      const double na = ck.x + t2 * ba - b1a, nb = ck.y + t2 * bb - b1b;
      b1a = ba; b1b = bb;
      ba = na; bb = nb;
    }
    c0 = __ldg(c);
  }
  return make_double2(c0.x + t * ba - b1a, c0.y + t * bb - b1b);
}
// copy the real-space table of q into shared memory (all threads of the
// block take part; the caller synchronises before the first use).  A block
// that evaluates many lattice sums reads its table from there: the lanes of a
// warp look up different intervals, which the read-only cache serves as that
// many separate lines.
__device__ __forceinline__ const double2 *bem_wtab_stage(const bem_qp &q, double2 *wts) {
  if (!q.wt) return nullptr;
  const int cnt = q.wt_n * BEM_WT_DEG;
  const double2 *src = reinterpret_cast<const double2 *>(q.wt);
  for (int e = threadIdx.x; e < cnt; e += blockDim.x) wts[e] = __ldg(src + e);
  return wts;
}

// Ewald real-space term for lattice point (l1,l2)  (ew_qG1_v1_cFl, d3_qpgf_d2.c:1814).
// ce = exp(i k_par . R_l) is supplied by the caller, which advances it along the
// row by one complex multiplication per term instead of a sincos.
__device__ __forceinline__ void ew_real_term(const bem_qp &q, double px, double py, double rz, cplx ce,
                                             double ke, double ke2, double ve, double ive, bool tab, cplx &F,
                                             cplx &cf, const double2 *wts = nullptr) {
  const double r2 = px * px + py * py + rz * rz;
  const double irl = rsqrt(r2), rl = r2 * irl;  // one reciprocal square root for both
  const double rl2e = rl * 0.5 * ive;
  if (tab) {
    const double2 ab = bem_wtab(q, ve, ke, rl2e, wts);
    F = cscale(ce, irl * ab.x);
    cf = cscale(ce, 2.0 * ve * irl * irl * irl * ab.y);
  } else {
    const double ef = exp(ke2 - rl2e * rl2e);
    const cplx w = bem_faddeeva(ke, rl2e);
    F = cscale(ce, irl * ef * w.re);
    cf = cscale(ce, irl * irl * ef * (irl * w.re - q.k * w.im + ive * 0.56418958354775628695));
  }
}

// Ewald spectral term for reciprocal point (n1,n2) (ew_qG2_v1_cFn, d3_qpgf_d2.c:1965);
// ce = exp(i alpha_n . r) supplied by the caller (recurrence along n2).
// returns 0 propagating, 1 evanescent, -3 beta_n == 0
// Quantities that decide a lattice sum's stopping point on the lattice plane
// are rounded as the reference's C code rounds them (each product and sum
// separately, no fused multiply-add), so that exact zeros and exact ties
// come out where the reference's do.
__device__ __forceinline__ double bem_sub2(double r, int l1, double d1, int l2, double d2) {
  return __dadd_rn(__dadd_rn(r, -__dmul_rn((double)l1, d1)), -__dmul_rn((double)l2, d2));
}
// exp(a) rounded to nearest.  Used only where the reference's rounding of
// exp decides a stopping test (the lattice plane below): the reference calls
// the C library's exp, whose results are correctly rounded except in rare
// near-midpoint cases, so a correctly rounded exp reproduces its decisions.
// Method: a = n ln2 + r (|r| <= ln2 / 2, ln2 as a double-double), e = exp(r / 1024) - 1
// by its Taylor series in double-double arithmetic, ten squarings
// (1 + e)^2 = 1 + (2 e + e^2), then 2^n (1 + e) rounded once.
struct bem_dd { double hi, lo; };
__device__ __forceinline__ bem_dd dd_two_sum(double a, double b) {
  const double s = a + b, bb = s - a;
  return {s, (a - (s - bb)) + (b - bb)};
}
__device__ __forceinline__ bem_dd dd_add(bem_dd x, bem_dd y) {
  bem_dd s = dd_two_sum(x.hi, y.hi);
  s.lo += x.lo + y.lo;
  return dd_two_sum(s.hi, s.lo);
}
__device__ __forceinline__ bem_dd dd_mul(bem_dd x, bem_dd y) {
  const double p = x.hi * y.hi;
  const double e = fma(x.hi, y.hi, -p) + (x.hi * y.lo + x.lo * y.hi);
  return dd_two_sum(p, e);
}
__device__ __forceinline__ bem_dd dd_scale(bem_dd x, double s) {  // s a power of two
  return {x.hi * s, x.lo * s};
}
__device__ __noinline__ double bem_exp_cr(double a) {
  if (!(a > -700.0 && a < 700.0)) return exp(a);
  const double ln2_hi = 0.69314718055994528623, ln2_lo = 2.3190468138462995584e-17;
  const double n = rint(a * 1.4426950408889634074);
  // r = a - n ln2 in double-double (n ln2_hi exact as a two-product)
  const double ph = n * ln2_hi, pl = fma(n, ln2_hi, -ph);
  bem_dd r = dd_two_sum(a - ph, -pl);  // a - ph is exact (Sterbenz)
  r = dd_add(r, {-n * ln2_lo, -fma(n, ln2_lo, -n * ln2_lo)});
  r = dd_scale(r, 1.0 / 1024.0);
  // e = r + r^2/2! + ... + r^10/10! (|r| < 3.4e-4: the next term is below 1e-40)
  bem_dd term = r, e = r;
  for (int k = 2; k <= 10; ++k) {
    term = dd_mul(term, r);
    term = dd_mul(term, {1.0 / k, fma(-1.0 / k, (double)k, 1.0) / k});
    e = dd_add(e, term);
  }
  for (int i = 0; i < 10; ++i) e = dd_add(dd_scale(e, 2.0), dd_mul(e, e));
  const bem_dd v = dd_add({1.0, 0.0}, e);
  return ldexp(v.hi + v.lo, (int)n);
}

// a_n = -k_par + n1 g1 + n2 g2 (ew_qG2_v1_cFn, d3_qpgf_d2.c:1970)
__device__ __forceinline__ double bem_an(double mk, int n1, double g1, int n2, double g2) {
  return __dadd_rn(__dadd_rn(mk, __dmul_rn((double)n1, g1)), __dmul_rn((double)n2, g2));
}
// Ewald parameter, capped where k^2 eta^2 - r^2 / 4 eta^2 > EW_EXPM (d3_qpgf_d2.c:1684-1697).
// On and next to the lattice plane the reference's eta0 (its truncation there
// depends on it), elsewhere eta_run (eta0 unless a tuned value is set: both
// sums converge).
__device__ __forceinline__ double bem_ewald_eta(const bem_qp &q, double rx, double ry, double rz) {
  const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(rx, rx), __dmul_rn(ry, ry)), __dmul_rn(rz, rz));
  const double ve = fabs(rz) < BEM_PLANE_NEAR ? q.eta0 : q.eta_run, kk = __dmul_rn(q.k, q.k);
  const double lhs = __dadd_rn(__dmul_rn(__dmul_rn(kk, ve), ve), -__ddiv_rn(r2, __dmul_rn(__dmul_rn(4.0, ve), ve)));
  if (lhs > BEM_EW_EXPM)
    return __ddiv_rn(__dsqrt_rn(__dadd_rn(BEM_EW_EXPM, __dsqrt_rn(__dadd_rn(__dmul_rn(kk, r2), BEM_EW_EXPM * BEM_EW_EXPM)))),
                     __dmul_rn(1.4142135623730950488, q.k));
  return ve;
}

// The lattice-plane forms below run for a few points of a mesh only; they are
// kept out of line so that the hot loops' code stays small.
// Propagating order on the plane: 2 (ef Re w(bn ve) - 1) as the reference rounds it.
__device__ __noinline__ double ew_plane_residue(const bem_qp &q, int n1, int n2, double bn2, double bn, double ve) {
  // On the lattice plane ef Re w(bn ve) - 1 is zero up to rounding; the
  // reference's rows stop on an identically zero z-derivative sum, so the
  // residue must be the reference's rounded value: the host's table at
  // eta0, else formed as the reference forms it (Faddeeva_w on the real
  // axis is exp(-x^2), Faddeeva.cc:684; ef = exp(bn2 ve ve)).
  if (ve == q.eta0)
    for (int i = 0; i < q.pz_n; ++i)
      if (q.pz_n1[i] == n1 && q.pz_n2[i] == n2) return q.pz_d[i];
  const double x = __dmul_rn(bn, ve);
  return __dadd_rn(__dmul_rn(bem_exp_cr(__dmul_rn(__dmul_rn(bn2, ve), ve)), bem_exp_cr(-__dmul_rn(x, x))), -1.0);
}
// Evanescent order next to the plane: f1 = e^{bn z} erfc(bn ve + z/2ve),
// f2 = e^{-bn z} erfc(bn ve - z/2ve), whose difference is zero, or not, by
// rounding alone; the rows' stopping tests see that zero, so both are formed
// exactly as the reference forms them (ebz = exp(bn z), f2 with 1/ebz;
// d3_qpgf_d2.c:2003-2007).
__device__ __noinline__ double2 ew_plane_evanescent(double bn, double ve, double rz, double azve) {
  const double ebz = bem_exp_cr(__dmul_rn(bn, rz)), bvr = __dmul_rn(bn, ve);
  return make_double2(__dmul_rn(ebz, erfc(__dadd_rn(bvr, azve))),
                      __dmul_rn(__ddiv_rn(1.0, ebz), erfc(__dadd_rn(bvr, -azve))));
}

// A spectral order n at d = z / (2 ve), bv = |beta_n| ve, depends on the
// point only through d once k, k_par, the lattice and ve = eta_run are fixed:
//   evanescent (beta_n^2 < 0): f1 + f2 = e^{-bv^2 - d^2} (erfcx(bv + d) + erfcx(bv - d)),
//     f1 - f2 = d e^{-bv^2 - d^2} int_{-1}^{1} erfcx'(bv + d s) ds;
//     tabulated: P = (f1 + f2) / |beta_n| and M = (f1 - f2) / d (no
//     cancellation next to d = 0);
//   propagating (beta_n^2 > 0): Q = e^{bv^2 - d^2} w(bv + i d) = e^{-2 i bv d} erfc(d - i bv);
//     tabulated: Re Q, Im Q.
// The per-problem table holds, per order of a window and per interval of d in
// [-D, D), the Chebyshev series of both channels: one Clenshaw recurrence
// replaces two erfcx, an exp, a square root and a division per evanescent
// term, and a Faddeeva value and an exp per propagating one.  Truncation below
// 1e-16 of each interval's scale (checked against 30-digit arithmetic).
// Returns false where the table does not reach (order or d outside it): the
// caller evaluates directly.
__device__ __forceinline__ bool ew_spec_tab(const bem_qp &q, int n1, int n2, double d, double &c0v, double &c1v) {
  const int i1 = n1 - q.st_n1lo, i2 = n2 - q.st_n2lo;
  const double u = d * (1.0 / BEM_ST_H) + 0.5 * q.st_nint;
  if (!(u >= 0.0)) return false;
  const int j = (int)u;
  if ((unsigned)i1 >= (unsigned)q.st_n1cnt || (unsigned)i2 >= (unsigned)q.st_n2cnt || j >= q.st_nint) return false;
  const double t = 2.0 * (u - j) - 1.0, t2 = 2.0 * t;
  const double2 *c = reinterpret_cast<const double2 *>(q.st) +
                     ((size_t)(i1 * q.st_n2cnt + i2) * q.st_nint + j) * BEM_ST_DEG;
  double b0 = 0.0, b1 = 0.0, b10 = 0.0, b11 = 0.0;
#pragma unroll
  for (int k = BEM_ST_DEG - 1; k >= 1; --k) {
    const double2 ck = __ldg(c + k);
    const double n0 = ck.x + t2 * b0 - b10, n1v = ck.y + t2 * b1 - b11;
    b10 = b0; b11 = b1;
    b0 = n0; b1 = n1v;
  }
  const double2 cz = __ldg(c);
  c0v = cz.x + t * b0 - b10;
  c1v = cz.y + t * b1 - b11;
  return true;
}
// the table applies: built for this ve, and away from the lattice plane
__device__ __forceinline__ bool ew_spec_tab_ok(const bem_qp &q, double ve, double rz) {
  return q.st != nullptr && ve == q.eta_run && fabs(rz) >= BEM_PLANE_NEAR;
}

__device__ __forceinline__ int ew_spec_term(const bem_qp &q, int n1, int n2, double anx, double any, double rz, cplx ce,
                                            double ve, cplx &Fn, cplx &dF0, cplx &dF1, cplx &dF2) {
  const double bn2 = __dadd_rn(__dadd_rn(__dmul_rn(q.k, q.k), -__dmul_rn(anx, anx)), -__dmul_rn(any, any));
  const double azve = rz / (2.0 * ve);
  if (bn2 > 0.0) {
    const double bn = __dsqrt_rn(bn2);
    const cplx ff = cexpi(bn * rz);
    double qr, qi;
    if (ew_spec_tab_ok(q, ve, rz) && ew_spec_tab(q, n1, n2, azve, qr, qi)) {
      Fn = cscale(cmul(ce, cmk(ff.re, qi + ff.im)), 2.0 / bn);
      dF0 = cscale(Fn, anx);
      dF1 = cscale(Fn, any);
      dF2 = cscale(cmul(ce, cmk(qr - ff.re, -ff.im)), 2.0);
      return 0;
    }
    const double ef = exp(bn2 * ve * ve - azve * azve);
    const cplx w = bem_faddeeva(bn * ve, azve);
    // Fn = 2 ce / bn (i ef Im w + ff)
    Fn = cscale(cmul(ce, cmk(ff.re, ef * w.im + ff.im)), 2.0 / bn);
    dF0 = cscale(Fn, anx);
    dF1 = cscale(Fn, any);
    if (rz == 0.0) {
      dF2 = cscale(ce, 2.0 * ew_plane_residue(q, n1, n2, bn2, bn, ve));
    } else {
      dF2 = cscale(cmul(ce, cmk(ef * w.re - ff.re, -ff.im)), 2.0);
    }
    return 0;
  } else if (bn2 < 0.0) {
    // f1 = e^{bn z} erfc(bn ve + z/2ve), f2 = e^{-bn z} erfc(bn ve - z/2ve)
    double P, Mt;
    if (ew_spec_tab_ok(q, ve, rz) && ew_spec_tab(q, n1, n2, azve, P, Mt)) {
      // Fn = ce / (i bn) (f1 + f2) = -i ce P;  f1 - f2 = d M
      Fn = cmul(ce, cmk(0.0, -P));
      dF0 = cscale(Fn, anx);
      dF1 = cscale(Fn, any);
      dF2 = cscale(ce, azve * Mt);
      return 1;
    }
    const double bn = sqrt(-bn2), bv = bn * ve;
    double f1, f2;
    if (fabs(rz) < BEM_PLANE_NEAR) {
      const double2 f = ew_plane_evanescent(bn, ve, rz, azve);
      f1 = f.x;
      f2 = f.y;
    } else {
      // = e^{-Q} erfcx(bn ve +- z/2ve) with Q = bn^2 ve^2 + (z/2ve)^2: one exp
      const double eq = exp(-(bv * bv + azve * azve));
      f1 = eq * erfcx(bv + azve);
      f2 = eq * erfcx(bv - azve);
    }
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
__device__ BEM_QPGF_ATTR int bem_qpgf_ewald(const bem_qp &q, double rx, double ry, double rz, bem_gval &out,
                                            const double2 *wts = nullptr) {
  const double ve = bem_ewald_eta(q, rx, ry, rz);
  const double ke = q.k * ve, ke2 = ke * ke, ive = 1.0 / ve;
  const bool tab = q.wt != nullptr && ve == q.eta_run;  // table built for x = k eta_run
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
          ew_real_term(q, px, py, rz, ce, ke, ke2, ve, ive, tab, F, cf, wts);
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
          const int e = ew_spec_term(q, n1, n2, bem_an(-q.kx, n1, q.g1x, n2, q.g2x),
                                     bem_an(-q.ky, n1, q.g1y, n2, q.g2y), rz, ce, ve, Fn, d0, d1, d2);
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
__device__ BEM_QPGF_ATTR int bem_qpgf_spectral(const bem_qp &q, double rx, double ry, double rz, bem_gval &out) {
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
__device__ BEM_QPGF_ATTR int bem_qpgf(const bem_qp &q, double rx, double ry, double rz, bem_gval &out,
                                      const double2 *wts = nullptr) {
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
  const double hx = bem_sub2(rx, l1, q.d1x, l2, q.d2x);
  const double hy = bem_sub2(ry, l1, q.d1y, l2, q.d2y);
  const int e = spectral ? bem_qpgf_spectral(q, hx, hy, rz, out) : bem_qpgf_ewald(q, hx, hy, rz, out, wts);
  if (e > 0 && (l1 != 0 || l2 != 0)) {
    const cplx cf = cexpi(-(q.kx * (l1 * q.d1x + l2 * q.d2x) + q.ky * (l1 * q.d1y + l2 * q.d2y)));
    out.g = cmul(out.g, cf);
    out.gx = cmul(out.gx, cf);
    out.gy = cmul(out.gy, cf);
    out.gz = cmul(out.gz, cf);
  }
  return e;
}

// ---------------------------------------------------------------- second derivatives
// G_qp, grad G_qp and the second derivatives d2 = {xx, yy, zz, xy, yz, zx}
// (d3hm_qpgf_d2_v2, d3_qpgf_d2.c:178-230; Ewald terms :2011-2399, spectral
// :887-1044).  Used by the field evaluation at points off the boundary.  The
// stopping tests are the reference's for this variant: the real-space and
// Ewald-spectral sums test d2_xx and d2_yy, the pure spectral sum d2_zz.
struct bem_gval2 { cplx g, d[3], d2[6]; };

__device__ __forceinline__ cplx cmuli(cplx a) { return cmk(-a.im, a.re); }  // i a

__device__ int bem_qpgf2_ewald(const bem_qp &q, double rx, double ry, double rz, bem_gval2 &o) {
  const double ve = bem_ewald_eta(q, rx, ry, rz);
  const double ke = q.k * ve, ke2 = ke * ke, ive = 1.0 / ve;
  const bool tab = q.wt != nullptr && ve == q.eta_run;
  const double eps = BEM_MEPS, isp = 0.56418958354775628695;
  int cc = 0;
  const cplx E2 = cexpi(q.kx * q.d2x + q.ky * q.d2y);
  cplx s = cmk(0, 0), sd[3] = {cmk(0, 0), cmk(0, 0), cmk(0, 0)}, s2[6];
  for (int c = 0; c < 6; ++c) s2[c] = cmk(0, 0);
  for (int dir = 0; dir < 3; ++dir) {
    int l1 = dir == 2 ? -1 : (dir == 1 ? 1 : 0);
    const int step = dir == 2 ? -1 : 1;
    bool done = false;
    for (int it = 0; it < (dir == 0 ? 1 : BEM_EW_LIMIT - 1); ++it, l1 += step) {
      const cplx o0 = s2[0], o1 = s2[1];
      const int lc = -(int)round(((rx + l1 * q.d1x) * q.d2x + (ry + l1 * q.d1y) * q.d2y) / q.d2sq);
      const cplx pc = cexpi(q.kx * (l1 * q.d1x + lc * q.d2x) + q.ky * (l1 * q.d1y + lc * q.d2y));
      for (int side = 0; side < 3; ++side) {
        int l2 = side == 0 ? lc : (side == 1 ? lc + 1 : lc - 1);
        const int st = side == 2 ? -1 : 1;
        const cplx E = side == 2 ? cconj(E2) : E2;
        cplx ce = side == 0 ? pc : cmul(pc, E);
        const int nmax = side == 0 ? 1 : BEM_EW_LIMIT - 1;
        int k = 0;
        for (; k < nmax; ++k, l2 += st) {
          const double px = rx + l1 * q.d1x + l2 * q.d2x, py = ry + l1 * q.d1y + l2 * q.d2y;
          const double rl = sqrt(px * px + py * py + rz * rz);
          const double irl = 1.0 / rl, irl2 = irl * irl;
          const double rl2e = rl * 0.5 * ive;
          const double ef = exp(ke2 - rl2e * rl2e);
          // A = ef Re w and the first-derivative factor from the table when it applies
          double A, B1;
          if (tab) {
            const double2 ab = bem_wtab(q, ve, ke, rl2e);
            A = ab.x;
            B1 = 2.0 * ve * irl * irl * irl * ab.y;
          } else {
            const cplx w = bem_faddeeva(ke, rl2e);
            A = ef * w.re;
            B1 = irl2 * ef * (irl * w.re - q.k * w.im + ive * isp);
          }
          const cplx cf1 = cscale(ce, B1);
          const cplx cf2 = cscale(ce, irl2 * (q.k * q.k * irl * 2.0 * A - ive * ive * ive * isp * ef));
          const cplx cf3 = cadd(cscale(cf1, -6.0 * irl2), cf2);
          ++cc;
          s = cadd(s, cscale(ce, irl * A));
          sd[0] = cadd(sd[0], cscale(cf1, px));
          sd[1] = cadd(sd[1], cscale(cf1, py));
          sd[2] = cadd(sd[2], cf1);
          const cplx t0 = cadd(cscale(cf1, 2.0), cscale(cf3, px * px));
          const cplx t1 = cadd(cscale(cf1, 2.0), cscale(cf3, py * py));
          s2[0] = cadd(s2[0], t0);
          s2[1] = cadd(s2[1], t1);
          s2[2] = cadd(s2[2], cadd(cscale(cf1, 2.0), cscale(cf3, rz * rz)));
          s2[3] = cadd(s2[3], cscale(cf3, px * py));
          s2[4] = cadd(s2[4], cscale(cf3, py));
          s2[5] = cadd(s2[5], cscale(cf3, px));
          if (side != 0 && bem_small(t0, s2[0], eps) && bem_small(t1, s2[1], eps)) break;
          ce = cmul(ce, E);
        }
        if (side != 0 && k == nmax) return -21;
      }
      if (dir != 0 && bem_same(s2[0], o0, eps) && bem_same(s2[1], o1, eps)) { done = true; break; }
    }
    if (dir != 0 && !done) return -21;
  }
  const double i4p = 0.07957747154594766788, i8p = 0.5 * i4p;
  o.g = cscale(s, i4p);
  o.d[0] = cscale(sd[0], -i4p);
  o.d[1] = cscale(sd[1], -i4p);
  o.d[2] = cscale(sd[2], -rz * i4p);
  for (int c = 0; c < 4; ++c) o.d2[c] = cscale(s2[c], -i8p);
  o.d2[4] = cscale(s2[4], -rz * i8p);
  o.d2[5] = cscale(s2[5], -rz * i8p);

  const cplx G2 = cexpi(q.g2x * rx + q.g2y * ry);
  cplx t = cmk(0, 0), td[3] = {cmk(0, 0), cmk(0, 0), cmk(0, 0)}, t2[6];
  for (int c = 0; c < 6; ++c) t2[c] = cmk(0, 0);
  const double azve = rz / (2.0 * ve), c2pi = 2.0 * isp * ive;
  for (int dir = 0; dir < 3; ++dir) {
    int n1 = q.nc1 + (dir == 2 ? -1 : (dir == 1 ? 1 : 0));
    const int step = dir == 2 ? -1 : 1;
    bool done = false;
    for (int it = 0; it < (dir == 0 ? 1 : BEM_EW_LIMIT - 1); ++it, n1 += step) {
      const cplx o0 = t2[0], o1 = t2[1];
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
          const double anx = a0x + n2 * q.g2x, any = a0y + n2 * q.g2y;
          const double bn2 = q.k * q.k - anx * anx - any * any;
          const double ef = exp(bn2 * ve * ve - azve * azve);
          cplx Fn, dz, dzz;
          int e;
          if (bn2 > 0.0) {
            const double bn = sqrt(bn2);
            const cplx ff = cexpi(bn * rz);
            const cplx w = bem_faddeeva(bn * ve, azve);
            const cplx F = cmk(2.0 * ff.re, 2.0 * (ef * w.im + ff.im));
            const cplx Gq = cmk(2.0 * (ef * w.re - ff.re), -2.0 * ff.im);
            Fn = cscale(cmul(ce, F), 1.0 / bn);
            dz = cmul(ce, Gq);
            dzz = cmul(ce, cadd(cscale(cmuli(F), bn), cmk(c2pi * ef, 0.0)));
            e = 0;
          } else if (bn2 < 0.0) {
            const double bn = sqrt(-bn2), bv = bn * ve;  // see ew_spec_term
            const double eq = exp(-(bv * bv + azve * azve));
            const double f1 = eq * erfcx(bv + azve), f2 = eq * erfcx(bv - azve);
            Fn = cmul(ce, cmk(0.0, -(f1 + f2) / bn));
            dz = cscale(ce, f1 - f2);
            dzz = cscale(ce, -bn * (f1 + f2) + c2pi * ef);
            e = 1;
          } else {
            return -23;
          }
          ++cc;
          const cplx d0 = cscale(Fn, anx), d1 = cscale(Fn, any);
          const cplx e0 = cscale(d0, anx), e1 = cscale(d1, any);
          t = cadd(t, Fn);
          td[0] = cadd(td[0], d0);
          td[1] = cadd(td[1], d1);
          td[2] = cadd(td[2], dz);
          t2[0] = cadd(t2[0], e0);
          t2[1] = cadd(t2[1], e1);
          t2[2] = cadd(t2[2], dzz);
          t2[3] = cadd(t2[3], cscale(d0, any));
          t2[4] = cadd(t2[4], cscale(dz, any));
          t2[5] = cadd(t2[5], cscale(dz, anx));
          if (side != 0) {
            if (e > 0) { if (bem_small(e0, t2[0], eps) && bem_small(e1, t2[1], eps)) break; }
            else ++flg;
          }
          ce = cmul(ce, E);
        }
        if (side != 0 && k == nmax) return -22;
      }
      if (dir != 0 && flg == 0 && bem_same(t2[0], o0, eps) && bem_same(t2[1], o1, eps)) { done = true; break; }
    }
    if (dir != 0 && !done) return -22;
  }
  const double cd = 0.25 * q.aidet;
  o.g = cadd(o.g, cscale(cmuli(t), cd));
  o.d[0] = cadd(o.d[0], cscale(td[0], -cd));
  o.d[1] = cadd(o.d[1], cscale(td[1], -cd));
  o.d[2] = cadd(o.d[2], cscale(td[2], cd));
  o.d2[0] = cadd(o.d2[0], cscale(cmuli(t2[0]), -cd));
  o.d2[1] = cadd(o.d2[1], cscale(cmuli(t2[1]), -cd));
  o.d2[2] = cadd(o.d2[2], cscale(t2[2], -cd));
  o.d2[3] = cadd(o.d2[3], cscale(cmuli(t2[3]), -cd));
  o.d2[4] = cadd(o.d2[4], cscale(cmuli(t2[4]), cd));
  o.d2[5] = cadd(o.d2[5], cscale(cmuli(t2[5]), cd));
  return cc;
}

__device__ int bem_qpgf2_spectral(const bem_qp &q, double rx, double ry, double rz, bem_gval2 &o) {
  if (rz == 0.0) return -14;
  const double eps = BEM_MEPS, az = fabs(rz);
  int cc = 0;
  const cplx G2 = cexpi(q.g2x * rx + q.g2y * ry);
  cplx t = cmk(0, 0), td[3] = {cmk(0, 0), cmk(0, 0), cmk(0, 0)}, t2[6];
  for (int c = 0; c < 6; ++c) t2[c] = cmk(0, 0);
  for (int dir = 0; dir < 3; ++dir) {
    int n1 = q.nc1 + (dir == 2 ? -1 : (dir == 1 ? 1 : 0));
    const int step = dir == 2 ? -1 : 1;
    bool done = false;
    for (int it = 0; it < (dir == 0 ? 1 : BEM_FD_LIMIT - 1); ++it, n1 += step) {
      const cplx old = t2[2];
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
          const double anx = a0x + n2 * q.g2x, any = a0y + n2 * q.g2y;
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
            Fn = cmk(d2.im / bn, -d2.re / bn);
            e = 1;
          } else {
            return -12;
          }
          ++cc;
          const cplx d0 = cscale(Fn, anx), d1 = cscale(Fn, any), zz = cscale(Fn, bn2);
          t = cadd(t, Fn);
          td[0] = cadd(td[0], d0);
          td[1] = cadd(td[1], d1);
          td[2] = cadd(td[2], d2);
          t2[0] = cadd(t2[0], cscale(d0, anx));
          t2[1] = cadd(t2[1], cscale(d1, any));
          t2[2] = cadd(t2[2], zz);
          t2[3] = cadd(t2[3], cscale(d1, anx));
          t2[4] = cadd(t2[4], cscale(d2, any));
          t2[5] = cadd(t2[5], cscale(d2, anx));
          if (side != 0 && e > 0 && bem_small(zz, t2[2], eps)) break;
          ce = cmul(ce, E);
        }
        if (side != 0 && k == nmax) return -11;
      }
      if (dir != 0 && bem_same(t2[2], old, eps)) { done = true; break; }
    }
    if (dir != 0 && !done) return -11;
  }
  const double c = 0.5 * q.aidet, sz = rz > 0 ? 1.0 : -1.0;
  o.g = cscale(cmuli(t), c);
  o.d[0] = cscale(td[0], -c);
  o.d[1] = cscale(td[1], -c);
  o.d[2] = cscale(td[2], -c * sz);
  for (int m = 0; m < 4; ++m) o.d2[m] = cscale(cmuli(t2[m]), -c);
  o.d2[4] = cscale(cmuli(t2[4]), -c * sz);
  o.d2[5] = cscale(cmuli(t2[5]), -c * sz);
  return cc;
}

__device__ int bem_qpgf2(const bem_qp &q, double rx, double ry, double rz, bem_gval2 &out) {
  bool spectral = false;
  if (!q.ewald_only) {
    const double az = fabs(rz);
    spectral = q.sel_cp * exp(-q.sel_bp * az) < BEM_MEPS && q.sel_cm * exp(-q.sel_bm * az) < BEM_MEPS;
    if (spectral && (36.0 / az) * (36.0 / az) * fabs(q.det) * 0.0795774715459476679 > BEM_FD_MAX_TERMS) spectral = false;
  }
  const int l1 = (int)floor((rx * q.d2y - ry * q.d2x) * q.idet + 0.5);
  const int l2 = (int)floor(-(rx * q.d1y - ry * q.d1x) * q.idet + 0.5);
  const double hx = bem_sub2(rx, l1, q.d1x, l2, q.d2x);
  const double hy = bem_sub2(ry, l1, q.d1y, l2, q.d2y);
  const int e = spectral ? bem_qpgf2_spectral(q, hx, hy, rz, out) : bem_qpgf2_ewald(q, hx, hy, rz, out);
  if (e > 0 && (l1 != 0 || l2 != 0)) {
    const cplx cf = cexpi(-(q.kx * (l1 * q.d1x + l2 * q.d2x) + q.ky * (l1 * q.d1y + l2 * q.d2y)));
    out.g = cmul(out.g, cf);
    for (int c = 0; c < 3; ++c) out.d[c] = cmul(out.d[c], cf);
    for (int c = 0; c < 6; ++c) out.d2[c] = cmul(out.d2[c], cf);
  }
  return e;
}
