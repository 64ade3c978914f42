"""Triangle elements (the reference's linear triangles, lit_* / q0_lit_*):
parity of the 80-triangle icosphere on a triangular lattice with the
reference's own solve (tests/golden/make_golden.py, tri80.npz).

Tolerances (stated here, used below): the same as the quad sphere's
  coefficient matrices G, H, dG, dH   1e-10 relative to the row maximum
  dF                                  1e-10 (column 0), 1e-11 absolute (columns 1, 2)
  P, dP, pv, dpv                      1e-9 relative to the array maximum
  force / torque (types 0 and 1)      1e-9 relative to |F| (torque x 0.3, the radius)
  field values, boundary values       1e-9 relative to the largest value of the
                                      same kind (boundary values per domain)
Fixtures: tri80.npz (matrices, solution, type-0 force) and fields_tri80.npz
(type-1 force, field and boundary values), both `make_golden.py tri`.
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


@pytest.fixture(scope="module")
def tri80_fields(tri80):
    case, _ = tri80
    return case, np.load(os.path.join(GOLD, "fields_tri80.npz"))


def test_tri80_force_type1(tri80_fields):
    """lit_force_7p: the 7-point rule's boundary values and stress integral."""
    case, g = tri80_fields
    for tag, rc in (("", (0.0, 0.0, 0.0)), ("c", (0.05, -0.02, 0.1))):
        F, N = case.force(1, rc)
        sF = np.linalg.norm(g["F1" + tag])
        assert np.linalg.norm(F - g["F1" + tag]) < 1e-9 * sF, (F, g["F1" + tag])
        assert np.linalg.norm(N - g["N1" + tag]) < 1e-9 * sF * 0.3


def test_tri80_field_values(tri80_fields):
    """phi_s / p_t / pv_s / pv_t off the boundary with rules 0-3 on triangles
    (q0_lit_dcoef_grad_* / lit_dcoef_grad_*): 1e-9 relative to the largest value
    of the same kind."""
    case, g = tri80_fields
    pts, types = g["pts"], g["types"]
    for name, keys in (("phi_s", ("phi_s",)), ("p_t", ("p_t",)), ("pv_s", ("pv_s_p", "pv_s_v")),
                       ("pv_t", ("pv_t_p", "pv_t_v"))):
        got = [case.field(name, tuple(p), int(t)) for p, t in zip(pts, types)]
        assert [r[0] for r in got] == list(g["did"])
        for j, key in enumerate(keys):
            a = np.array([r[1 + j] for r in got])
            ref = g[key]
            assert np.max(np.abs(a - ref)) <= 1e-9 * np.max(np.abs(ref)), (name, key)


def test_tri80_boundary_values(tri80_fields):
    case, g = tri80_fields
    phi, p, v = [], [], []
    for (did, t, z, e), ty in zip(g["bd"], g["btypes"]):
        phi.append(case.boundary("phi_s_bd", int(did), int(t), z, e, int(ty))[0])
        a, b = case.boundary("pv_t_bd", int(did), int(t), z, e, int(ty))
        p.append(a)
        v.append(b)
    # domain 0 and domain 1 values differ in scale; compare each domain on its own
    dom = g["bd"][:, 0].astype(int)
    for d in (0, 1):
        m = dom == d
        for a, key in ((phi, "phi_s_bd"), (p, "pv_t_bd_p"), (v, "pv_t_bd_v")):
            ref = g[key]
            err = np.abs(np.array(a) - ref).reshape(len(ref), -1).max(axis=1)
            assert np.all(err[m] <= 1e-9 * np.max(np.abs(ref[m]))), (key, d, err[m] / np.max(np.abs(ref[m])))


def test_context_reuse_across_problems():
    """One context loads a 24-quad sphere, the 80-triangle sphere, the quad
    sphere again, and the triangles again: device buffers of an earlier
    problem are reused when large enough, grown when not, and every force
    equals the one of a fresh context to 1e-12 of |F| (the same arithmetic
    runs; only the order of floating-point atomics may differ)."""
    import ctypes
    from bem3_aw_qd2_b200 import api, meshgen
    g = api.libs()[1]
    g.bemgpu_load.argtypes = [ctypes.c_void_p, ctypes.POINTER(api.Problem)]
    g.bemgpu_unload.argtypes = [ctypes.c_void_p]
    cases = []
    for name in ("sphere24", "tri80"):
        d = tempfile.mkdtemp(prefix="reuse_%s_" % name)
        cases.append(api.Case.from_files(*meshgen.write_inputs(d, **meshgen.CONFIGS[name])))
    probs = [c.problem() for c in cases]

    def forces(ctx, pr):
        assert g.bemgpu_load(ctx, ctypes.byref(pr)) == 0, g.bemgpu_error(ctx)
        assert g.bemgpu_run(ctx) == 0, g.bemgpu_error(ctx)
        F, N, rc = np.zeros(3), np.zeros(3), np.zeros(3)
        assert g.bemgpu_force(ctx, 0, api._p(rc), api._p(F), api._p(N)) == 0, g.bemgpu_error(ctx)
        assert g.bemgpu_status(ctx) == 0
        return np.concatenate([F, N])

    fresh = []
    for pr in probs:
        ctx = ctypes.c_void_p()
        assert g.bemgpu_create(0, None, ctypes.byref(ctx)) == 0
        fresh.append(forces(ctx, pr))
        g.bemgpu_destroy(ctx)
    ctx = ctypes.c_void_p()
    assert g.bemgpu_create(0, None, ctypes.byref(ctx)) == 0
    try:
        def same(a, b):
            return np.max(np.abs(a - b)) <= 1e-12 * np.linalg.norm(b[:3])
        for i in (0, 1, 0, 1):
            assert same(forces(ctx, probs[i]), fresh[i]), i
        assert g.bemgpu_unload(ctx) == 0
        assert same(forces(ctx, probs[0]), fresh[0])
    finally:
        g.bemgpu_destroy(ctx)
        for c, pr in zip(cases, probs):
            c.free_problem(pr)
