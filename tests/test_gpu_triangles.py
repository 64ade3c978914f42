"""Triangle elements (the reference's linear triangles, lit_* / q0_lit_*):
parity of the 80-triangle icosphere on a triangular lattice with the
reference's own solve (tests/golden/make_golden.py, tri80.npz).

Tolerances (stated here, used below): the same as the quad sphere's
  coefficient matrices G, H, dG, dH   1e-10 relative to the row maximum
  dF                                  1e-10 (column 0), 1e-11 absolute (columns 1, 2)
  P, dP, pv, dpv                      1e-9 relative to the array maximum
  force / torque (type 0)             1e-9 relative to |F|
"""
import os
import tempfile

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu
GOLD = os.path.join(ROOT, "tests", "golden")


def rel_rows(a, b):
    scale = np.max(np.abs(b), axis=1, keepdims=True)
    scale[scale == 0] = 1.0
    return float(np.max(np.abs(a - b) / scale))


def rel_max(a, b):
    s = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / (s if s > 0 else 1.0))


@pytest.fixture(scope="module")
def tri80():
    from bem3_aw_qd2_b200 import api, meshgen
    d = tempfile.mkdtemp(prefix="tri80_")
    case = api.Case.from_files(*meshgen.write_inputs(d, **meshgen.CONFIGS["tri80"]))
    case.solve()
    return case, np.load(os.path.join(GOLD, "tri80.npz"))


def test_tri80_matrices(tri80):
    case, g = tri80
    N = 320
    errs = {}
    for d in (0, 1):
        for w in ("G", "H") + (("dG", "dH") if d else ()):
            errs["%s%d" % (w, d)] = rel_rows(case.matrix(d, w, N), g["%s%d" % (w, d)])
    assert max(errs.values()) < 1e-10, errs
    for d in (0, 1):
        dF, ref = case.matrix(d, "dF", N), g["dF%d" % d]
        assert np.max(np.abs(dF[:, 0] - ref[:, 0])) < 1e-10 * np.max(np.abs(ref[:, 0]))
        assert np.max(np.abs(dF[:, 1:] - ref[:, 1:])) < 1e-11


def test_tri80_solution_and_force(tri80):
    case, g = tri80
    for d in (0, 1):
        P, dP, pv, dpv = case.solution(d, 80)
        errs = [rel_max(P, g["P%d" % d]), rel_max(dP, g["dP%d" % d]), rel_max(pv, g["pv%d" % d]),
                rel_max(dpv, g["dpv%d" % d])]
        assert max(errs) < 1e-9, (d, errs)
    F, N = case.force(0)
    s = np.linalg.norm(g["F0"])
    assert np.linalg.norm(F - g["F0"]) < 1e-9 * s
    assert np.linalg.norm(N - g["N0"]) < 1e-9 * s * 0.3
    assert case.status() == 0
