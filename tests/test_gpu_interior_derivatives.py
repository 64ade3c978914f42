"""Interior derivative rows recomputed in blocks (bemgpu_set_interior_derivatives
keep = 0) against the rows kept after the assembly (keep = 1, the default): the
same free-space kernels give the same dG, dH rows, contracted with P and dP by
the same particle-velocity kernel, so every output must agree.

Cases: the 24-quad sphere (quads) and the 80-triangle icosphere (triangles,
padding rows), each with one block of every row and with blocks of 8 rows (a
partial last block); the reference's own 216-quad check case runs in the
default block size.

Tolerance (stated here, used below): P, dP, pv, dpv and the type-0 and type-1
forces within 1e-13 of the kept rows' results relative to each array's
largest entry (the arithmetic is the same; only the launch grouping differs)."""
import ctypes
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-13


def _run(g, prob, ne, keep, rows):
    from bem3_aw_qd2_b200 import api
    ctx = ctypes.c_void_p()
    assert g.bemgpu_create(0, None, ctypes.byref(ctx)) == 0
    try:
        assert g.bemgpu_set_interior_derivatives(ctx, keep, rows) == 0
        assert g.bemgpu_load(ctx, ctypes.byref(prob)) == 0, g.bemgpu_error(ctx)
        assert g.bemgpu_run(ctx) == 0, g.bemgpu_error(ctx)
        out = []
        for d in (0, 1):
            arrs = [np.zeros((ne, 4), np.complex128), np.zeros((ne, 4), np.complex128),
                    np.zeros((ne, 4, 3), np.complex128), np.zeros((ne, 4, 3), np.complex128)]
            assert g.bemgpu_get_solution(ctx, d, *[api._p(a.view(np.float64)) for a in arrs]) == 0
            out += arrs
        for ft in (0, 1):
            F, N, rc = np.zeros(3), np.zeros(3), np.zeros(3)
            assert g.bemgpu_force(ctx, ft, api._p(rc), api._p(F), api._p(N)) == 0
            out += [F, N]
        if not keep:
            # the rows are not kept: nothing to return for dG, dH
            buf = np.zeros(8, np.float64)
            assert g.bemgpu_get_matrix(ctx, 1, 2, api._p(buf)) == -2
        return out
    finally:
        g.bemgpu_destroy(ctx)


@pytest.mark.parametrize("config,rows", [("sphere24", 0), ("sphere24", 8), ("tri80", 0), ("tri80", 8),
                                         ("sphere216", 0)])
def test_recomputed_derivative_rows_match_kept(config, rows):
    from bem3_aw_qd2_b200 import api, meshgen
    h, g = api.libs()
    h.aqd2_set_verbose(0)
    g.bemgpu_load.argtypes = [ctypes.c_void_p, ctypes.POINTER(api.Problem)]
    g.bemgpu_get_matrix.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    case = api.Case.from_files(*meshgen.write_inputs(tempfile.mkdtemp(prefix="bem_dgh_"),
                                                     **meshgen.CONFIGS[config]))
    prob = case.problem()
    ne = meshgen.describe(config)["elements"]
    try:
        ref = _run(g, prob, ne, 1, 0)
        got = _run(g, prob, ne, 0, rows)
    finally:
        case.free_problem(prob)
        case.close()
    for x, y in zip(got, ref):
        assert np.max(np.abs(x - y)) <= TOL * max(np.max(np.abs(y)), 1e-300)
