"""The mixed-precision solve (complex FP32 LU, FP64 refinement) against the
plain FP64 solve of the same assembled system, with the tensor-core
outer-block updates as one TF32 product (mode 2) and as three split products
(mode 3).

Tolerances (stated here, used below):
  surface coefficients P, dP, pv, dpv   1e-10 relative to the array maximum
  force / torque (type 0)               1e-8 relative to |F| (the serving target)
The 216-quad sphere (n = 1728) is one outer block (no tensor-core update runs);
the 1536-quad sphere (n = 12288) has 96 outer blocks on the tensor cores and
panels whose leaves run several rounds of candidate selection.
"""
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel_max(a, b):
    s = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / (s if s > 0 else 1.0))


@pytest.mark.parametrize("config,ne", [("sphere216", 216), ("sphere1536", 1536)])
@pytest.mark.parametrize("mode", [3, 2])
def test_mixed_matches_fp64(config, ne, mode):
    from bem3_aw_qd2_b200 import api, meshgen
    d = tempfile.mkdtemp(prefix="mixed_%s_" % config)
    case = api.Case.from_files(*meshgen.write_inputs(d, **meshgen.CONFIGS[config]))
    try:
        case.solve()
        F64, N64 = case.force(0)
        ref = [case.solution(dd, ne) for dd in (0, 1)]
        case.set_precision(mode)
        case.run_device()
        it, rc, fb = case.solve_stats()
        assert int(np.sum(fb)) == 0, "fell back to FP64"
        assert max(rc) <= 1e-12
        F, N = case.force(0)
        got = [case.solution(dd, ne) for dd in (0, 1)]
        for s64, sm in zip(ref, got):
            for a, b in zip(sm, s64):
                assert rel_max(a, b) <= 1e-10
        s = np.linalg.norm(F64)
        assert np.linalg.norm(F - F64) <= 1e-8 * s
        assert np.linalg.norm(N - N64) <= 1e-8 * s
        assert case.status() == 0
    finally:
        case.close()
