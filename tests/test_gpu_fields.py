"""Parity of the device post-processing with the reference: radiation force
with the 9-point rule (force_FN_aqd2 type 1), field values off the boundary
(phi_s / p_t / pv_s / pv_t_aqd2) and boundary values (phi_s_bd / pv_t_bd_aqd2).
The golden values are the reference's own outputs on the solved 24-quad
cube-sphere (tests/golden/make_golden.py, fields24.npz).

Tolerances (stated here, used below):
  field values                  1e-9 relative to the largest value of the same kind
  boundary values               1e-9 likewise, except at the 9-point rule positions
                                with the 9-point rule (see below): 1e-7
  force (type 1)                1e-7 relative to |F|; torque 1e-7 |F| x 0.3 (the radius)
  domain ids                    equal

Why 1e-7 where the 9-point rule meets its own positions: on this mirror-symmetric
mesh a target at a rule position (zeta, eta in {-b, 0, b}) and the mirrored rule
points of other elements lie on a common lattice plane, R_z = 0 exactly or
within 1e-16.  There the reference's Ewald sum stops on its z-derivative sum,
which is zero or pure rounding noise, so its value depends on rounding: the
reference's own boundary values jump by 5e-7 to 8e-6 when such a target moves
by 1e-14.  The device reproduces the exact-zero decisions (the lattice-plane
test in test_gpu_parity.py); the noise-driven ones (R_z ~ 1e-16) leave ~3e-8.
"""
import os
import tempfile

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu
GOLD = os.path.join(ROOT, "tests", "golden")
TOL = 1e-9
TOL_RULE = 1e-7
B9 = 0.7745966692414833770359


@pytest.fixture(scope="module")
def solved():
    from bem3_aw_qd2_b200 import api, meshgen
    d = tempfile.mkdtemp(prefix="bem24f_")
    files = meshgen.write_inputs(d, **meshgen.CONFIGS["sphere24"])
    case = api.Case.from_files(*files)
    case.solve()
    return case, np.load(os.path.join(GOLD, "fields24.npz")), d


def _close(a, b, scale):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b)))) <= TOL * scale


def test_force_type1(solved):
    case, g, _ = solved
    for tag, rc in (("", (0.0, 0.0, 0.0)), ("c", (0.05, -0.02, 0.1))):
        F, N = case.force(1, rc)
        Fr, Nr = g["F1" + tag], g["N1" + tag]
        sF = np.linalg.norm(Fr)
        assert np.linalg.norm(F - Fr) < TOL_RULE * sF
        assert np.linalg.norm(N - Nr) < TOL_RULE * sF * 0.3
    assert case.status() == 0


def test_field_values(solved):
    case, g, _ = solved
    pts, types = g["pts"], g["types"]
    out = {k: [] for k in ("did", "phi_s", "p_t", "pv_s_p", "pv_s_v", "pv_t_p", "pv_t_v")}
    for p, t in zip(pts, types):
        did, phi, _ = case.field("phi_s", p, int(t))
        out["did"].append(did)
        out["phi_s"].append(phi)
        out["p_t"].append(case.field("p_t", p, int(t))[1])
        _, a, v = case.field("pv_s", p, int(t))
        out["pv_s_p"].append(a)
        out["pv_s_v"].append(v)
        _, a, v = case.field("pv_t", p, int(t))
        out["pv_t_p"].append(a)
        out["pv_t_v"].append(v)
    assert list(out["did"]) == list(g["did"])
    for k in ("phi_s", "p_t", "pv_s_p", "pv_s_v", "pv_t_p", "pv_t_v"):
        ref = g[k]
        got = np.array(out[k])
        # points of each kind are compared against the largest value of that kind
        assert _close(got, ref, np.max(np.abs(ref))), "%s: worst point %d" % (
            k, int(np.argmax(np.max(np.abs(got - ref).reshape(len(ref), -1), axis=1))))


def test_boundary_values(solved):
    case, g, _ = solved
    phi, p, v = [], [], []
    for (did, t, z, e), ty in zip(g["bd"], g["btypes"]):
        phi.append(case.boundary("phi_s_bd", int(did), int(t), float(z), float(e), int(ty))[0])
        a, b = case.boundary("pv_t_bd", int(did), int(t), float(z), float(e), int(ty))
        p.append(a)
        v.append(b)
    # domain 0 and domain 1 values differ in scale; compare each domain on its own
    dom = g["bd"][:, 0].astype(int)
    on_rule = np.array([ty == 1 and all(np.isclose(abs(x), B9) or x == 0.0 for x in (z, e))
                        for (_, _, z, e), ty in zip(g["bd"], g["btypes"])])
    for d in (0, 1):
        m = dom == d
        for got, key in ((np.array(phi), "phi_s_bd"), (np.array(p), "pv_t_bd_p"), (np.array(v), "pv_t_bd_v")):
            ref = g[key]
            scale = np.max(np.abs(ref[m]))
            err = np.abs(got - ref).reshape(len(ref), -1).max(axis=1)
            tol = np.where(on_rule, TOL_RULE, TOL) * scale
            assert np.all(err[m] <= tol[m]), "%s domain %d: %s" % (key, d, err[m] / scale)


def test_dat_file_postprocessing(solved):
    """A solution read back from a .dat file (no solve in this object) gives the
    same force and fields: the boundary values are uploaded on first use."""
    from bem3_aw_qd2_b200 import api
    case, g, d = solved
    path = os.path.join(d, "s24.dat")
    case.dat_write(path)
    other = api.Case.from_dat(path)
    F, N = other.force(1)
    assert np.linalg.norm(F - g["F1"]) < TOL_RULE * np.linalg.norm(g["F1"])
    did, a, v = other.field("pv_t", g["pts"][0], 1)
    assert did == g["did"][0]
    assert abs(a - g["pv_t_p"][0]) <= TOL * np.max(np.abs(g["pv_t_p"]))
    other.close()


@pytest.mark.parametrize("mode", [1, 2, 3, 4])
def test_mixed_precision_matches_fp64(solved, mode):
    """Complex FP32 LU (FP32 / TF32 / TF32x3 trailing updates) with FP64
    refinement: surface values to 1e-11 of the FP64 solve, force and torque of
    both rules to 1e-8 (the radiation-force tolerance of the mixed form)."""
    case, g, _ = solved
    case.set_precision(0)
    case.run_device()
    ref = [case.solution(d, 24) for d in (0, 1)]
    F0, N0 = case.force(0)
    F1, N1 = case.force(1)
    case.set_precision(mode)
    case.run_device()
    it, rc, fb = case.solve_stats()
    assert len(it) == 3 and np.all(fb == 0) and np.all(it >= 1) and np.all(rc <= 1e-12)
    for d in (0, 1):
        for a, b in zip(case.solution(d, 24), ref[d]):
            assert np.max(np.abs(a - b)) <= 1e-11 * np.max(np.abs(b))
    for t, (Fr, Nr) in ((0, (F0, N0)), (1, (F1, N1))):
        F, N = case.force(t)
        assert np.linalg.norm(F - Fr) <= 1e-8 * np.linalg.norm(Fr)
        assert np.linalg.norm(N - Nr) <= 1e-8 * np.linalg.norm(Fr) * 0.3
    case.set_precision(0)
    case.run_device()
