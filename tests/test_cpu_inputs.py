"""CPU checks of the input generators the tests and the bench use: the
icosphere's topology and orientation, the configuration table, and the
serving bench's seeded request stream."""
import collections
import math

import numpy as np

from conftest import ROOT  # noqa: F401


def test_icosphere_closed_outward_on_radius():
    from bem3_aw_qd2_b200 import meshgen
    for level, count in ((1, 80), (3, 1280)):
        nodes, tris = meshgen.icosphere(level, (0.3, 0.3, 0.3))
        assert tris.shape == (count, 3)
        assert np.allclose(np.linalg.norm(nodes, axis=1), 0.3)
        c = nodes.mean(axis=0)
        for t in tris:
            r = nodes[t]
            assert np.dot(np.cross(r[1] - r[0], r[2] - r[0]), r.mean(axis=0) - c) > 0
        # a closed surface: every edge belongs to exactly two triangles, once each way
        edges = collections.Counter()
        for t in tris:
            for a, b in ((t[0], t[1]), (t[1], t[2]), (t[2], t[0])):
                edges[(a, b)] += 1
        assert all(v == 1 for v in edges.values())
        assert all((b, a) in edges for (a, b) in edges)


def test_configurations_describe_their_meshes():
    from bem3_aw_qd2_b200 import meshgen
    for name, cfg in meshgen.CONFIGS.items():
        desc = meshgen.describe(name)
        if cfg.get("ico") is not None:
            _, el = meshgen.icosphere(cfg["ico"], cfg["semi_axes"])
            npe = 3
        else:
            _, el = meshgen.cube_sphere(cfg["n"], cfg["semi_axes"])
            npe = 4
        assert desc["elements"] == len(el)
        assert desc["unknowns"] == 2 * npe * len(el)
        # the reference needs a non-zero in-plane wave vector component on both axes
        th, ph = math.radians(cfg["theta_deg"]), math.radians(cfg["phi_deg"])
        assert math.sin(th) * math.cos(ph) != 0.0 and math.sin(th) * math.sin(ph) != 0.0


def test_stream_requests_seeded_and_keyed():
    import bench
    a = bench.stream_requests(64, np.random.default_rng(2024))
    b = bench.stream_requests(64, np.random.default_rng(2024))
    assert [k for _, k in a] == [k for _, k in b]
    keys = collections.Counter(k for _, k in a)
    assert any(v > 1 for v in keys.values())  # some requests repeat a key
    for r, key in a:
        lat = r["lattice"]
        k = 2 * math.pi / r["wavelength"]
        th, ph = math.radians(r["theta_deg"]), math.radians(r["phi_deg"])
        kx, ky = k * math.sin(th) * math.cos(ph), k * math.sin(th) * math.sin(ph)
        det = lat[0][0] * lat[1][1] - lat[1][0] * lat[0][1]
        g1 = (2 * math.pi * lat[1][1] / det, -2 * math.pi * lat[1][0] / det)
        g2 = (-2 * math.pi * lat[0][1] / det, 2 * math.pi * lat[0][0] / det)
        # no order within 2 % of a Rayleigh anomaly (|k_par + g| = k)
        for i in range(-6, 7):
            for j in range(-6, 7):
                a_n = math.hypot(kx + i * g1[0] + j * g2[0], ky + i * g1[1] + j * g2[1])
                assert abs(a_n - k) >= 0.02 * k * 0.999
    # a repeated key repeats the mesh, lattice and frequency
    first = {}
    for r, key in a:
        sig = (r["n"], tuple(r["semi_axes"]), tuple(map(tuple, r["lattice"])), round(r["wavelength"], 12))
        assert first.setdefault(key, sig) == sig
