// Norms of the FP64 iterative refinement (mixed-precision solves), shared by
// the device reduction and the host stopping test.  Plain C++ with no CUDA
// types, so the CPU tests compile it on its own.
#pragma once
#include <float.h>
#include <math.h>

#ifdef __CUDACC__
#define BEM_HD __host__ __device__
#else
#define BEM_HD
#endif

// One entry's share of the norms md = max |d| (correction) and mx = max |x|
// (solution), |re| + |im| as LAPACK's icamax.  A non-finite correction or
// solution entry makes md infinite: fmax alone would drop a NaN, and a
// refinement whose corrections are all NaN would then look converged.
BEM_HD static inline void bem_refine_norms(double dre, double dim, double xre, double xim, double *md, double *mx) {
  const double a = fabs(dre) + fabs(dim), b = fabs(xre) + fabs(xim);
  if (!(a <= DBL_MAX) || !(b <= DBL_MAX)) {
    *md = INFINITY;
    return;
  }
  *md = fmax(*md, a);
  *mx = fmax(*mx, b);
}

// Relative size of the last correction from the reduced norms: infinite when
// the correction was not finite, so that no tolerance accepts it.
BEM_HD static inline double bem_refine_rel(double md, double mx) {
  if (!(md <= DBL_MAX)) return INFINITY;
  return mx > 0.0 ? md / mx : 0.0;
}
