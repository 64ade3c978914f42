"""The request server: each result is the same alone and in the mix, the same
as the drop-in API's solve_bieq_aqd2 + force_FN_aqd2, and repeated
(mesh, media, lattice, frequency, in-plane Bloch wave vector) requests reuse the
resident factorisation.

Tolerances (stated here, used below):
  server alone vs in the mix    1e-12 relative to |F| (the same arithmetic runs;
                                only the order of requests and slots changes)
  server vs drop-in API         1e-12 relative to |F|, force rule 0.  A request
                                that shares a key is solved with the matrices of
                                the key's first request, whose in-plane wave
                                vector equals its own to rounding (sin 20 deg vs
                                sin 160 deg); the 9-point rule's lattice-plane
                                sums react to such rounding (see
                                test_gpu_fields.py), so rule 0 is compared here
"""
import os
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# incidences on the 24-quad sphere: theta 20 and 160 share the in-plane wave
# vector (the reflected direction), as does a different amplitude at theta 20
REQUESTS = [
    dict(theta_deg=20.0, phi_deg=30.0, amp=(1.0, 0.0)),
    dict(theta_deg=160.0, phi_deg=30.0, amp=(1.0, 0.0)),
    dict(theta_deg=35.0, phi_deg=10.0, amp=(1.0, 0.0)),
    dict(theta_deg=20.0, phi_deg=30.0, amp=(0.5, 0.8)),
    dict(theta_deg=50.0, phi_deg=-40.0, amp=(1.0, 0.0)),
]


def key_of(req):
    import math
    th, ph = math.radians(req["theta_deg"]), math.radians(req["phi_deg"])
    kx, ky = math.sin(th) * math.cos(ph), math.sin(th) * math.sin(ph)
    return hash(("sphere24", round(kx, 12), round(ky, 12))) & 0xFFFFFFFFFFFFFFFF


@pytest.fixture(scope="module")
def cases():
    from bem3_aw_qd2_b200 import api, meshgen
    out = []
    for i, r in enumerate(REQUESTS):
        d = tempfile.mkdtemp(prefix="srv%d_" % i)
        cfg = dict(meshgen.CONFIGS["sphere24"])
        cfg.update(theta_deg=r["theta_deg"], phi_deg=r["phi_deg"])
        files = meshgen.write_inputs(d, amp=r["amp"], **cfg)
        out.append(api.Case.from_files(*files))
    return out


def run_server(cases, slots, sequential, precision=0, first_alone=False, force_type=1):
    from bem3_aw_qd2_b200 import api
    srv = api.Server(slots=slots, hbm_budget=8 << 30)
    res = {}
    probs = [c.problem() for c in cases]
    try:
        order = list(range(len(cases)))
        if sequential:
            for i in order:
                srv.submit(probs[i], key_of(REQUESTS[i]), i, precision=precision, force_type=force_type)
                got = []
                while not got:
                    got = srv.poll(timeout_ms=1000)
                for r in got:
                    res[r.id] = r
        else:
            if first_alone:
                srv.submit(probs[0], key_of(REQUESTS[0]), 0, precision=precision, force_type=force_type)
                while 0 not in res:
                    for r in srv.poll(timeout_ms=1000):
                        res[r.id] = r
                order = order[1:]
            for i in order:
                srv.submit(probs[i], key_of(REQUESTS[i]), i, precision=precision, force_type=force_type)
            while len(res) < len(cases):
                for r in srv.poll(timeout_ms=1000):
                    res[r.id] = r
        stats = srv.stats()
    finally:
        srv.close()
        for p in probs:
            cases[0].free_problem(p)
    for r in res.values():
        assert r.status == 0, r.error
    return res, stats


def forces(res):
    return {i: (np.array(r.F[:]), np.array(r.N[:])) for i, r in res.items()}


def test_alone_equals_mix_and_reuse(cases):
    alone, st_a = run_server(cases, slots=1, sequential=True)
    mix, st_m = run_server(cases, slots=3, sequential=False, first_alone=True)
    # one slot, in order: 1 follows 0 (same key) -> reuse; 2 replaces the
    # resident problem, so 3 (0's key again) is assembled afresh
    assert alone[1].reused and not alone[2].reused and not alone[3].reused
    assert st_m["reused"] >= 1 and st_m["completed"] == len(cases)
    fa, fm = forces(alone), forces(mix)
    for i in range(len(cases)):
        s = np.linalg.norm(fa[i][0])
        assert np.linalg.norm(fa[i][0] - fm[i][0]) <= 1e-12 * s
        assert np.linalg.norm(fa[i][1] - fm[i][1]) <= 1e-12 * s


def test_server_matches_dropin(cases):
    res, _ = run_server(cases, slots=2, sequential=False, force_type=0)
    for i, c in enumerate(cases):
        c.solve()
        F, N = c.force(0)
        s = np.linalg.norm(F)
        assert np.linalg.norm(np.array(res[i].F[:]) - F) <= 1e-12 * s
        assert np.linalg.norm(np.array(res[i].N[:]) - N) <= 1e-12 * s


def test_server_mixed_precision(cases):
    """The served mixed form: force within 1e-8 of the served FP64 form."""
    f64, _ = run_server(cases, slots=2, sequential=False, precision=0)
    mx, _ = run_server(cases, slots=2, sequential=False, precision=3)
    for i in range(len(cases)):
        a, b = np.array(f64[i].F[:]), np.array(mx[i].F[:])
        assert np.linalg.norm(a - b) <= 1e-8 * np.linalg.norm(a)


def test_budget_rejects_oversized(cases):
    from bem3_aw_qd2_b200 import api
    srv = api.Server(slots=1, hbm_budget=1 << 20)
    p = cases[0].problem()
    try:
        with pytest.raises(RuntimeError):
            srv.submit(p, 1, 0)
    finally:
        srv.close()
        cases[0].free_problem(p)
