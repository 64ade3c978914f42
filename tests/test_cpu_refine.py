"""The refinement norms of the mixed-precision solves (csrc/bem_refine.h, the
same functions the device reduction and the host stopping test use) must not
let a non-finite correction look converged: compiled here as plain C and fed
NaN and infinite corrections."""
import os
import subprocess
import tempfile

from conftest import ROOT

CSRC = os.path.join(ROOT, "bem3_aw_qd2_b200", "csrc")

PROGRAM = r"""
#include <stdio.h>
#include "bem_refine.h"
static double run(const double *d, const double *x, int n) {
  double md = 0.0, mx = 0.0;
  for (int i = 0; i < n; ++i) bem_refine_norms(d[2 * i], d[2 * i + 1], x[2 * i], x[2 * i + 1], &md, &mx);
  return bem_refine_rel(md, mx);
}
int main(void) {
  const double nan = NAN, inf = INFINITY;
  double x[6] = {1.0, 0.5, -2.0, 0.0, 0.25, 0.25};
  double ok[6] = {1e-16, 0.0, -2e-16, 1e-16, 0.0, 0.0};
  double one_nan[6] = {1e-16, 0.0, nan, 0.0, 0.0, 0.0};
  double all_nan[6] = {nan, nan, nan, nan, nan, nan};
  double one_inf[6] = {0.0, -inf, 0.0, 0.0, 0.0, 0.0};
  double xnan[6] = {nan, 0.0, 0.0, 0.0, 0.0, 0.0};
  double zero[6] = {0};
  printf("%.17g %.17g %.17g %.17g %.17g %.17g\n", run(ok, x, 3), run(one_nan, x, 3), run(all_nan, x, 3),
         run(one_inf, x, 3), run(ok, xnan, 3), run(zero, zero, 3));
  return 0;
}
"""


def test_refinement_norms_reject_non_finite():
    d = tempfile.mkdtemp(prefix="bem_refine_")
    src, exe = os.path.join(d, "t.c"), os.path.join(d, "t")
    with open(src, "w") as f:
        f.write(PROGRAM)
    subprocess.run(["gcc", "-std=c99", "-O2", "-I" + CSRC, src, "-o", exe, "-lm"], check=True)
    ok, one_nan, all_nan, one_inf, x_nan, zero = [float(v) for v in subprocess.check_output([exe]).split()]
    assert abs(ok - 3e-16 / 2.0) < 1e-30
    # any non-finite correction or solution entry: no tolerance accepts the step
    for rc in (one_nan, all_nan, one_inf, x_nan):
        assert rc == float("inf")
        assert not rc <= 1e-12
    assert zero == 0.0
