"""Batches of Bloch vectors (bemgpu_batch_load / _assemble / _select): problems
on one body, media, lattice and frequency that differ only in the incidence
are assembled together (the interior domains once, the periodic domain of all
instances with each kernel launched once) and solved one after another.  Each
instance must give what the same problem gives loaded and run alone.

Cases: the 216-quad sphere at three incidence directions (three in-plane
Bloch wave vectors).  Tolerance (stated here, used below): the periodic
domain's G and H, P, dP, pv, dpv of both domains and the type-0 and type-1
forces within 1e-13 of the single-problem results relative to each array's
largest entry (the same kernels and order of sums; only the launch grouping
differs); torques, which vanish on a sphere up to round-off, within 1e-13 of
|F| times the radius 0.3.  A batch mixing frequencies is refused."""
import ctypes
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-13
DIRS = [(20.0, 30.0), (35.0, 10.0), (5.0, 200.0)]


def _cases(wavelengths=None):
    from bem3_aw_qd2_b200 import api, meshgen
    out = []
    for i, (th, ph) in enumerate(DIRS):
        cfg = dict(meshgen.CONFIGS["sphere216"], theta_deg=th, phi_deg=ph)
        if wavelengths:
            cfg["wavelength"] = wavelengths[i]
        out.append(api.Case.from_files(*meshgen.write_inputs(tempfile.mkdtemp(prefix="bem_bat_"), **cfg)))
    return out


def _results(g, ctx, ne):
    from bem3_aw_qd2_b200 import api
    N = 4 * ne
    out = []
    for w in (0, 1):  # periodic domain's G, H
        m = np.zeros((N, N), np.complex128)
        assert g.bemgpu_get_matrix(ctx, 0, w, api._p(m.view(np.float64))) == 0
        out.append(m)
    for d in (0, 1):
        arrs = [np.zeros((ne, 4), np.complex128), np.zeros((ne, 4), np.complex128),
                np.zeros((ne, 4, 3), np.complex128), np.zeros((ne, 4, 3), np.complex128)]
        assert g.bemgpu_get_solution(ctx, d, *[api._p(a.view(np.float64)) for a in arrs]) == 0
        out += arrs
    for ft in (0, 1):
        F, Nt, rc = np.zeros(3), np.zeros(3), np.zeros(3)
        assert g.bemgpu_force(ctx, ft, api._p(rc), api._p(F), api._p(Nt)) == 0
        out += [F, Nt]
    return out


def _check(got, ref):
    """Arrays in _results order: G, H, 8 solution arrays, then (F, N) of force types 0 and 1."""
    for i, (x, y) in enumerate(zip(got, ref)):
        scale = np.max(np.abs(y))
        if i >= 10 and (i - 10) % 2 == 1:  # a torque: scaled by its force
            scale = max(scale, 0.3 * np.linalg.norm(ref[i - 1]))
        assert np.max(np.abs(x - y)) <= TOL * max(scale, 1e-300), i


def _lib():
    from bem3_aw_qd2_b200 import api
    h, g = api.libs()
    h.aqd2_set_verbose(0)
    g.bemgpu_load.argtypes = [ctypes.c_void_p, ctypes.POINTER(api.Problem)]
    g.bemgpu_batch_load.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.POINTER(api.Problem))]
    g.bemgpu_batch_assemble.argtypes = [ctypes.c_void_p]
    g.bemgpu_batch_select.argtypes = [ctypes.c_void_p, ctypes.c_int]
    g.bemgpu_get_matrix.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    return g


def test_batch_matches_single_problems():
    from bem3_aw_qd2_b200 import api
    g = _lib()
    cases = _cases()
    probs = [c.problem() for c in cases]
    ne = 216
    ctx = ctypes.c_void_p()
    assert g.bemgpu_create(0, None, ctypes.byref(ctx)) == 0
    try:
        # single problems, each in a fresh load
        ref = []
        for p in probs:
            assert g.bemgpu_load(ctx, ctypes.byref(p)) == 0, g.bemgpu_error(ctx)
            assert g.bemgpu_run(ctx) == 0, g.bemgpu_error(ctx)
            ref.append(_results(g, ctx, ne))
        assert g.bemgpu_load(ctx, ctypes.byref(probs[0])) == 0
        single = g.bemgpu_kernel_launches()
        assert g.bemgpu_assemble(ctx) == 0
        single = g.bemgpu_kernel_launches() - single
        # the batch
        arr = (ctypes.POINTER(api.Problem) * len(probs))(*[ctypes.pointer(p) for p in probs])
        assert g.bemgpu_batch_load(ctx, len(probs), arr) == 0, g.bemgpu_error(ctx)
        n0 = g.bemgpu_kernel_launches()
        assert g.bemgpu_batch_assemble(ctx) == 0, g.bemgpu_error(ctx)
        batched = g.bemgpu_kernel_launches() - n0
        # one launch per kernel for every instance, one diagonal launch per instance
        assert batched == single + len(probs) - 1, (batched, single)
        for b in (1, 0, 2):
            assert g.bemgpu_batch_select(ctx, b) == 0, g.bemgpu_error(ctx)
            assert g.bemgpu_solve(ctx) == 0, g.bemgpu_error(ctx)
            _check(_results(g, ctx, ne), ref[b])
        assert g.bemgpu_status(ctx) == 0
        # a new load ends the batch: the context is a single problem again
        assert g.bemgpu_load(ctx, ctypes.byref(probs[2])) == 0
        assert g.bemgpu_run(ctx) == 0
        _check(_results(g, ctx, ne), ref[2])
    finally:
        g.bemgpu_destroy(ctx)
        for c, p in zip(cases, probs):
            c.free_problem(p)
            c.close()


def test_batch_refuses_mixed_frequencies():
    from bem3_aw_qd2_b200 import api
    g = _lib()
    cases = _cases(wavelengths=[1.0, 1.0, 1.1])
    probs = [c.problem() for c in cases]
    ctx = ctypes.c_void_p()
    assert g.bemgpu_create(0, None, ctypes.byref(ctx)) == 0
    try:
        arr = (ctypes.POINTER(api.Problem) * len(probs))(*[ctypes.pointer(p) for p in probs])
        assert g.bemgpu_batch_load(ctx, len(probs), arr) == -2
        assert b"not the same body" in g.bemgpu_error(ctx)
        assert g.bemgpu_batch_assemble(ctx) == -2
    finally:
        g.bemgpu_destroy(ctx)
        for c, p in zip(cases, probs):
            c.free_problem(p)
            c.close()
