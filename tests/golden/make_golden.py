"""Generate the golden fixtures of tests/golden from the reference itself.

Runs the reference's own C code (oracle/_ref, built from the reference
sources by oracle/ref/Makefile) on seeded synthetic inputs and stores its
outputs as compressed .npz files:

  faddeeva.npz   Faddeeva_w(z, 1e-15) on points covering every branch
  qpgf.npz       d3hm_qpgf_d2_v1 / _v1_ew / _v1_fd on random points for a
                 square and an oblique lattice
  sphere24.npz   a full solve of the 24-quad cube-sphere with the
                 216-quad configuration's media, lattice and incidence:
                 coefficient matrices of both domains (the reference's temporary
                 files), P, dP, pv, dpv, force and torque (type 0)

Usage: python tests/golden/make_golden.py  (needs oracle/_ref; about a minute)
"""
import math
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import refwrap  # noqa: E402
from bem3_aw_qd2_b200 import meshgen  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def qp_of(k, theta_deg, phi_deg, d1, d2):
    th, ph = math.radians(theta_deg), math.radians(phi_deg)
    return np.array([k, k * math.sin(th) * math.cos(ph), k * math.sin(th) * math.sin(ph), k * math.cos(th),
                     d1[0], d1[1], d2[0], d2[1]])


def faddeeva_points(rng):
    pts = []
    for x in [0.0, 1e-5, 1e-3, 0.1, 0.5, 1.0, 1.4, 2.5, 5.0, 6.5, 9.0, 12.0, 30.0]:
        for y in [-8.0, -3.0, -1.0, -0.2, 0.0, 1e-8, 0.05, 0.3, 1.0, 2.0, 4.0, 6.9, 7.5, 20.0]:
            pts += [complex(x, y), complex(-x, y)]
    x = rng.uniform(0, 8, 2000)
    y = rng.uniform(-2, 9, 2000)
    pts += list(x + 1j * y)
    return np.array(pts)


def main():
    rng = np.random.default_rng(20241203)
    # Faddeeva
    z = faddeeva_points(rng)
    np.savez_compressed(os.path.join(OUT, "faddeeva.npz"), z=z, w=refwrap.faddeeva_w(z))
    # QPGF on two lattices
    out = {}
    for name, qp in [("square", qp_of(2 * math.pi, 20.0, 30.0, (0.8, 0.0), (0.0, 0.8))),
                     ("oblique", qp_of(2 * math.pi, 35.0, 15.0, (1.0, 0.0), (0.3, 0.9)))]:
        r = np.concatenate([rng.uniform(-0.7, 0.7, (300, 3)),
                            rng.uniform(-0.05, 0.05, (100, 3)),
                            np.column_stack([rng.uniform(-2, 2, (100, 2)), rng.uniform(0.3, 1.0, 100)])])
        out[name + "_qp"] = qp
        out[name + "_r"] = r
        for mode, tag in [(0, "v1"), (1, "ew"), (2, "fd")]:
            G, dG, ret = refwrap.qpgf(qp, r, mode)
            out["%s_%s_G" % (name, tag)] = G
            out["%s_%s_dG" % (name, tag)] = dG
            out["%s_%s_ret" % (name, tag)] = ret
    np.savez_compressed(os.path.join(OUT, "qpgf.npz"), **out)
    # full solve, 24 quads
    tmp = tempfile.mkdtemp(prefix="golden_")
    files = meshgen.write_inputs(tmp, **meshgen.CONFIGS["sphere24"])
    case = refwrap.RefCase(*files)
    mats = case.solve(tmp)
    sol = {}
    for d in range(case.MN + 1):
        P, dP, pv, dpv = case.solution(d)
        sol.update({"P%d" % d: P, "dP%d" % d: dP, "pv%d" % d: pv, "dpv%d" % d: dpv})
    F0, N0 = case.force(0)
    keep = {k: v for k, v in mats.items() if not (k.startswith("dG0") or k.startswith("dH0"))}
    np.savez_compressed(os.path.join(OUT, "sphere24.npz"), F0=F0, N0=N0, **keep, **sol)
    print("fixtures written to", OUT)


if __name__ == "__main__":
    main()
