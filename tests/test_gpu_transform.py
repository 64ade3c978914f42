"""Rotation and translation of a device-resident body (bemgpu_transform_mesh)
against the reference's own placement options: the same rotation and
translation given to read_aqd2 (Rodrigues axis, angle, translation; the mesh
is turned before the element constants and incident field are built on the
host) must give the same solution and forces.

Tolerance (stated here, used below): P, dP, pv, dpv within 1e-10 of the array
maximum, forces within 1e-10 relative (the two paths turn the geometry in a
different order, so they agree to rounding, not bit for bit)."""
import ctypes
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-10
RV, TH, TV = (1.0, -2.0, 0.5), 0.7, (0.011, -0.02, 0.031)


def _solution(g, ctx, ne):
    from bem3_aw_qd2_b200 import api
    out = []
    for d in (0, 1):
        arrs = [np.zeros((ne, 4), np.complex128), np.zeros((ne, 4), np.complex128),
                np.zeros((ne, 4, 3), np.complex128), np.zeros((ne, 4, 3), np.complex128)]
        assert g.bemgpu_get_solution(ctx, d, *[api._p(a.view(np.float64)) for a in arrs]) == 0
        out += arrs
    F, N, rc = np.zeros(3), np.zeros(3), np.zeros(3)
    for ty in (0, 1):
        assert g.bemgpu_force(ctx, ty, api._p(rc), api._p(F), api._p(N)) == 0
        out += [F.copy(), N.copy()]
    return out


def test_device_transform_matches_reference_placement():
    from bem3_aw_qd2_b200 import api, meshgen
    h, g = api.libs()
    h.aqd2_set_verbose(0)
    g.bemgpu_load.argtypes = [ctypes.c_void_p, ctypes.POINTER(api.Problem)]
    g.bemgpu_transform_mesh.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_double,
                                        ctypes.POINTER(ctypes.c_double)]
    files = meshgen.write_inputs(tempfile.mkdtemp(prefix="bem_xf_"), **meshgen.CONFIGS["sphere24"])
    plain = api.Case.from_files(*files)
    moved = api.Case.from_files(*files, rotation=RV + (TH,) + TV)
    moved.solve()
    ref = _solution(g, moved.ctx, 24)
    pr = plain.problem()
    ctx = ctypes.c_void_p()
    assert g.bemgpu_create(0, None, ctypes.byref(ctx)) == 0
    try:
        assert g.bemgpu_load(ctx, ctypes.byref(pr)) == 0
        assert g.bemgpu_run(ctx) == 0              # the unmoved body first
        rv, tv = np.array(RV), np.array(TV)
        assert g.bemgpu_transform_mesh(ctx, api._p(rv), TH, api._p(tv)) == 0, g.bemgpu_error(ctx)
        assert g.bemgpu_run(ctx) == 0, g.bemgpu_error(ctx)
        got = _solution(g, ctx, 24)
        for i, (x, y) in enumerate(zip(got, ref)):
            assert np.max(np.abs(x - y)) <= TOL * np.max(np.abs(y)), i
        assert g.bemgpu_status(ctx) == 0
    finally:
        g.bemgpu_destroy(ctx)
        plain.free_problem(pr)
        plain.close()
        moved.close()
