"""Interior-domain reuse: a context that loads a second problem on the same
body, media and frequency but with another in-plane Bloch wave vector keeps
the free-space domain's matrices and dpv factors (bemgpu_interior_reuses) and
must give what a fresh context gives for that problem.

Tolerance (stated here, used below): P, dP, pv, dpv and the force within
1e-13 of the fresh context's (the same kernels on the same inputs)."""
import ctypes
import os
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-13


def _solve(g, ctx, prob, ne):
    from bem3_aw_qd2_b200 import api
    assert g.bemgpu_load(ctx, ctypes.byref(prob)) == 0, g.bemgpu_error(ctx)
    assert g.bemgpu_run(ctx) == 0, g.bemgpu_error(ctx)
    out = []
    for d in (0, 1):
        arrs = [np.zeros((ne, 4), np.complex128), np.zeros((ne, 4), np.complex128),
                np.zeros((ne, 4, 3), np.complex128), np.zeros((ne, 4, 3), np.complex128)]
        assert g.bemgpu_get_solution(ctx, d, *[api._p(a.view(np.float64)) for a in arrs]) == 0
        out += arrs
    F, N, rc = np.zeros(3), np.zeros(3), np.zeros(3)
    assert g.bemgpu_force(ctx, 1, api._p(rc), api._p(F), api._p(N)) == 0
    return out + [F, N]


def _case(theta, phi, wavelength=1.0):
    from bem3_aw_qd2_b200 import api, meshgen
    cfg = dict(meshgen.CONFIGS["sphere24"], theta_deg=theta, phi_deg=phi, wavelength=wavelength)
    return api.Case.from_files(*meshgen.write_inputs(tempfile.mkdtemp(prefix="bem_int_"), **cfg))


def test_interior_matrices_kept_across_bloch_vectors():
    from bem3_aw_qd2_b200 import api
    h, g = api.libs()
    h.aqd2_set_verbose(0)
    g.bemgpu_load.argtypes = [ctypes.c_void_p, ctypes.POINTER(api.Problem)]
    g.bemgpu_interior_reuses.argtypes = [ctypes.c_void_p]
    g.bemgpu_interior_reuses.restype = ctypes.c_longlong
    a, b, c = _case(20.0, 30.0), _case(35.0, 10.0), _case(35.0, 10.0, wavelength=1.1)
    pa, pb, pc = a.problem(), b.problem(), c.problem()
    ctx, fresh = ctypes.c_void_p(), ctypes.c_void_p()
    assert g.bemgpu_create(0, None, ctypes.byref(ctx)) == 0
    assert g.bemgpu_create(0, None, ctypes.byref(fresh)) == 0
    try:
        _solve(g, ctx, pa, 24)
        assert g.bemgpu_interior_reuses(ctx) == 0
        got = _solve(g, ctx, pb, 24)          # same body and frequency, new Bloch vector
        assert g.bemgpu_interior_reuses(ctx) == 1
        ref = _solve(g, fresh, pb, 24)
        for x, y in zip(got, ref):
            assert np.max(np.abs(x - y)) <= TOL * np.max(np.abs(y))
        _solve(g, ctx, pc, 24)                # another frequency: no reuse
        assert g.bemgpu_interior_reuses(ctx) == 1
        got = _solve(g, ctx, pb, 24)          # back to b after c: reassembled, same result
        for x, y in zip(got, ref):
            assert np.max(np.abs(x - y)) <= TOL * np.max(np.abs(y))
        # reuse switched off: the same problem again is assembled in full
        assert g.bemgpu_set_interior_reuse(ctx, 0) == 0
        n0 = g.bemgpu_kernel_launches()
        got = _solve(g, ctx, pb, 24)
        assert g.bemgpu_interior_reuses(ctx) == 1
        assert g.bemgpu_kernel_launches() > n0
        for x, y in zip(got, ref):
            assert np.max(np.abs(x - y)) <= TOL * np.max(np.abs(y))
        # switched on again: the matrices the last load assembled serve the next
        assert g.bemgpu_set_interior_reuse(ctx, 1) == 0
        _solve(g, ctx, pb, 24)
        assert g.bemgpu_interior_reuses(ctx) == 2
    finally:
        g.bemgpu_destroy(ctx)
        g.bemgpu_destroy(fresh)
        for case, p in ((a, pa), (b, pb), (c, pc)):
            case.free_problem(p)
            case.close()
