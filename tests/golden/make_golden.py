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
  qpgf_plane.npz d3hm_qpgf_d2_v1 on points of the lattice plane (z = 0
                 exactly), where the reference's spectral rows stop on an
                 identically zero z-derivative sum
  tri80.npz      a full solve of the 80-triangle icosphere (triangular
                 lattice): matrices of both domains, P, dP, pv, dpv, force
                 and torque (type 0)
  fields24.npz   on the same solved system: force and torque with the
                 9-point rule (type 1), field values (phi_s, p_t, pv_s, pv_t)
                 at points in the home cell, in shifted lattice cells, inside
                 the sphere and next to the boundary with rules 0-3, and
                 boundary values (phi_s_bd, pv_t_bd) on elements of both domains

  sphere216.npz  the 216-quad benchmark configuration solved by the reference
                 (sampled matrix rows, products with a random-phase vector,
                 absolute row sums, P, dP, pv, dpv, forces of both rules)
  sphere54_rot.npz, fields54_rot.npz
                 a full solve, forces, fields and boundary values of a 54-quad
                 sphere turned about a generic axis (no lattice-plane ties)
  shipped_*.npz  the reference's own shipped solved systems (ex.dat,
                 verification/, analysis_sample1/ex1.dat, analysis_sample2/ex2.dat):
                 their input files, the values their example1.log prints and
                 the solutions stored in the .dat files

Usage: python tests/golden/make_golden.py [fields|plane|tri|far|near|sphere216|rot|shipped [dir]]
(needs oracle/_ref; a few minutes; an argument regenerates only that fixture)
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


FIELD_POINTS = [  # (point, rule type)
    ((0.1, 0.2, 0.45), 1), ((0.35, -0.3, -0.1), 1), ((0.0, 0.0, 1.2), 1), ((1.7, -0.9, 0.2), 1),
    ((-0.75, 2.45, -0.5), 1), ((0.05, -0.1, 0.1), 1), ((0.0, 0.0, 0.305), 1), ((0.0, 0.0, 0.295), 1),
    ((0.12, 0.05, 0.42), 0), ((0.12, 0.05, 0.42), 2), ((0.12, 0.05, 0.42), 3), ((-0.02, 0.08, -0.15), 2),
    ((0.31, 0.02, 0.0), 2), ((0.2, 0.3, -0.38), 3),
]
BOUNDARY_POINTS = [  # (domain, element 1-based, zeta, eta, rule type)
    (0, 1, 0.3, -0.5, 1), (0, 7, 0.0, 0.0, 1), (0, 18, -0.7745966692414834, 0.7745966692414834, 1),
    (0, 3, 0.5, 0.25, 2), (0, 11, -0.2, 0.6, 0), (1, 2, 0.3, -0.5, 1), (1, 9, 0.0, 0.0, 2), (1, 20, -0.6, -0.1, 3),
]


def make_plane():
    rng = np.random.default_rng(20241204)
    out = {}
    for name, qp in [("square", qp_of(2 * math.pi, 20.0, 30.0, (0.8, 0.0), (0.0, 0.8))),
                     ("oblique", qp_of(2 * math.pi, 35.0, 15.0, (1.0, 0.0), (0.3, 0.9)))]:
        r = np.column_stack([rng.uniform(-0.9, 0.9, (200, 2)), np.zeros(200)])
        G, dG, ret = refwrap.qpgf(qp, r, 0)
        out.update({name + "_qp": qp, name + "_r": r, name + "_G": G, name + "_dG": dG, name + "_ret": ret})
    # next to the plane (|z| from 1e-19 to 1e-12) on the triangular lattice of
    # the 80-triangle icosphere, whose quadrature points meet such z
    qp = qp_of(2 * math.pi, 20.0, 30.0, (0.8, 0.0), (0.4, 0.69282032302755091741))
    zs = [1e-19, -1e-19, 1e-18, -1e-18, 2.6e-18, -3.5e-18, 5e-18, 7e-18, -7e-18, 1e-17, -1e-17, 3e-17,
          1e-16, -1e-16, 1e-15, 1e-14, 1e-13, 1e-12]
    xy = rng.uniform(-0.6, 0.6, (40, 2))
    r = np.array([(x, y, z) for x, y in xy for z in zs])
    G, dG, ret = refwrap.qpgf(qp, r, 0)
    out.update({"near_qp": qp, "near_r": r, "near_G": G, "near_dG": dG, "near_ret": ret})
    np.savez_compressed(os.path.join(OUT, "qpgf_plane.npz"), **out)


def make_solve(name, out_name):
    tmp = tempfile.mkdtemp(prefix="golden_")
    files = meshgen.write_inputs(tmp, **meshgen.CONFIGS[name])
    case = refwrap.RefCase(*files)
    mats = case.solve(tmp)
    sol = {}
    for d in range(case.MN + 1):
        P, dP, pv, dpv = case.solution(d)
        sol.update({"P%d" % d: P, "dP%d" % d: dP, "pv%d" % d: pv, "dpv%d" % d: dpv})
    F0, N0 = case.force(0)
    keep = {k: v for k, v in mats.items() if not (k.startswith("dG0") or k.startswith("dH0"))}
    np.savez_compressed(os.path.join(OUT, out_name), F0=F0, N0=N0, **keep, **sol)
    return case


TRI_BOUNDARY_POINTS = [  # on triangles: (zeta, eta) inside the reference triangle
    (0, 1, 0.1, -0.2, 1), (0, 7, 0.0, 0.0, 1), (0, 18, -0.3480702390148154917985, -0.6028753385763033130539, 1),
    (0, 33, 0.25, 0.1, 2), (0, 11, -0.2, 0.3, 0), (1, 2, 0.1, -0.2, 1), (1, 49, 0.0, 0.0, 2), (1, 70, -0.3, -0.1, 3),
]


def make_far_pairs(name="sphere216", out_name="far216.npz", n_pairs=400, n_near=80):
    """Reference coefficients G_i, H_i (q0_dcoef_bd_node_t2_cc) of n_pairs
    regular pairs of the mesh, most of them at least 5 element circumradii
    from the nearest lattice image of the target (where the device may use a
    shorter rule), n_near of them nearer."""
    tmp = tempfile.mkdtemp(prefix="golden_")
    cfg = meshgen.CONFIGS[name]
    files = meshgen.write_inputs(tmp, **cfg)
    case = refwrap.RefCase(*files)
    if "ico" in cfg:
        nodes, el = meshgen.icosphere(cfg["ico"], cfg["semi_axes"])
    else:
        nodes, el = meshgen.cube_sphere(cfg["n"], cfg["semi_axes"])
    P = nodes[el]
    cen = P.mean(axis=1)
    rad = np.max(np.linalg.norm(P - cen[:, None, :], axis=2), axis=1)
    d1 = np.array(list(cfg["lattice"][0]) + [0.0])
    d2 = np.array(list(cfg["lattice"][1]) + [0.0])
    rng = np.random.default_rng(20241205)
    ne, nodes_per = len(el), el.shape[1]
    picks = []
    while len(picks) < n_pairs:
        t, s = int(rng.integers(ne)), int(rng.integers(ne))
        if t == s:
            continue
        v = cen[t] - cen[s]
        dmin = min(np.linalg.norm(v + a * d1 + b * d2) for a in (-1, 0, 1) for b in (-1, 0, 1))
        far = dmin >= 5.5 * rad[s]
        if not far and (dmin < 2.0 * rad[s] or sum(1 for x in picks if not x[3]) >= n_near):
            continue
        picks.append((t + 1, int(rng.integers(nodes_per)), s + 1, far))
    G = np.zeros((len(picks), 4), np.complex128)
    H = np.zeros((len(picks), 4), np.complex128)
    for i, (t, tn, s, _) in enumerate(picks):
        cc = case.pair(0, t, tn, s)[0]
        G[i], H[i] = cc[:4], cc[4:8]
    idx = np.array([p[:3] for p in picks], np.int32)
    np.savez_compressed(os.path.join(OUT, out_name), idx=idx, far=np.array([p[3] for p in picks]), G=G, H=H)


def make_tier_pairs(name="sphere1536", out_name="tiers1536.npz", per_band=40):
    """Reference coefficients G_i, H_i (q0_dcoef_bd_node_t2_cc) of regular
    pairs spread over the distance bands of the device's shorter rules:
    (distance from the collocation node's nearest lattice image to the source
    element's centre) / (its circumradius) in 2.2-2.9 (the reference's rule),
    3.1-3.4 (10 points), 3.6-4.8 (9), 5.2-7.8 (8), 8.3-24 (7) and above 26 (6
    points where k R <= 0.2), per_band pairs each.  The node is the bilinear
    map of (+-1/sqrt3, +-1/sqrt3) on its element, as the reference places it."""
    tmp = tempfile.mkdtemp(prefix="golden_")
    cfg = meshgen.CONFIGS[name]
    files = meshgen.write_inputs(tmp, **cfg)
    case = refwrap.RefCase(*files)
    nodes, el = meshgen.cube_sphere(cfg["n"], cfg["semi_axes"])
    P = nodes[el]
    cen = P.mean(axis=1)
    rad = np.max(np.linalg.norm(P - cen[:, None, :], axis=2), axis=1)
    a = 1.0 / np.sqrt(3.0)
    zt, et = (-a, a, a, -a), (-a, -a, a, a)
    d1 = np.array(list(cfg["lattice"][0]) + [0.0])
    d2 = np.array(list(cfg["lattice"][1]) + [0.0])
    bands = [(2.2, 2.9), (3.1, 3.4), (3.6, 4.8), (5.2, 7.8), (8.3, 24.0), (26.0, 1e9)]
    rng = np.random.default_rng(20241209)
    ne = len(el)
    picks, count = [], [0] * len(bands)
    while min(count) < per_band:
        t, s, tn = int(rng.integers(ne)), int(rng.integers(ne)), int(rng.integers(4))
        if t == s:
            continue
        z, e = zt[tn], et[tn]
        N = np.array([(1 - z) * (1 - e), (1 + z) * (1 - e), (1 + z) * (1 + e), (1 - z) * (1 + e)]) / 4
        rt = N @ P[t]
        ratio = min(np.linalg.norm(rt - cen[s] + i * d1 + j * d2) for i in (-1, 0, 1) for j in (-1, 0, 1)) / rad[s]
        for b, (lo, hi) in enumerate(bands):
            if lo <= ratio <= hi and count[b] < per_band:
                count[b] += 1
                picks.append((t + 1, tn, s + 1, b))
    G = np.zeros((len(picks), 4), np.complex128)
    H = np.zeros((len(picks), 4), np.complex128)
    for i, (t, tn, s, _) in enumerate(picks):
        cc = case.pair(0, t, tn, s)[0]
        G[i], H[i] = cc[:4], cc[4:8]
    idx = np.array([p[:3] for p in picks], np.int32)
    np.savez_compressed(os.path.join(OUT, out_name), idx=idx, band=np.array([p[3] for p in picks], np.int8), G=G, H=H)


def make_near_pairs(n_pairs=240):
    """Reference coefficients of node-element pairs of the 216-quad sphere at
    1 to 3 element circumradii (centre distance from the node's nearest
    lattice image): the pairs the reference integrates with its 64 x 64 rule
    (|dF/dt| > 0.5) and the nearest of its 12 x 12 ones."""
    tmp = tempfile.mkdtemp(prefix="golden_")
    cfg = meshgen.CONFIGS["sphere216"]
    files = meshgen.write_inputs(tmp, **cfg)
    case = refwrap.RefCase(*files)
    nodes, el = meshgen.cube_sphere(cfg["n"], cfg["semi_axes"])
    P = nodes[el]
    cen = P.mean(axis=1)
    rad = np.max(np.linalg.norm(P - cen[:, None, :], axis=2), axis=1)
    d1 = np.array(list(cfg["lattice"][0]) + [0.0])
    d2 = np.array(list(cfg["lattice"][1]) + [0.0])
    rng = np.random.default_rng(20241206)
    ne = len(el)
    picks = []
    while len(picks) < n_pairs:
        t, s, tn = int(rng.integers(ne)), int(rng.integers(ne)), int(rng.integers(4))
        if t == s:
            continue
        # the node lies inside element t, near its corner tn
        node = cen[t] + 0.58 * (P[t, tn] - cen[t])
        v = node - cen[s]
        dmin = min(np.linalg.norm(v + a * d1 + b * d2) for a in (-1, 0, 1) for b in (-1, 0, 1))
        if 1.0 * rad[s] <= dmin < 3.0 * rad[s]:
            picks.append((t + 1, tn, s + 1))
    G = np.zeros((len(picks), 4), np.complex128)
    H = np.zeros((len(picks), 4), np.complex128)
    for i, (t, tn, s) in enumerate(picks):
        cc = case.pair(0, t, tn, s)[0]
        G[i], H[i] = cc[:4], cc[4:8]
    np.savez_compressed(os.path.join(OUT, "near216.npz"), idx=np.array(picks, np.int32), G=G, H=H)


def make_fields(case, out_name="fields24.npz", boundary_points=BOUNDARY_POINTS):
    out = {}
    out["F1"], out["N1"] = case.force(1)
    out["F1c"], out["N1c"] = case.force(1, (0.05, -0.02, 0.1))
    pts = np.array([p for p, _ in FIELD_POINTS])
    types = np.array([t for _, t in FIELD_POINTS], np.int32)
    res = {k: [] for k in ["did", "phi_s", "p_t", "pv_s_p", "pv_s_v", "pv_t_p", "pv_t_v"]}
    for p, t in FIELD_POINTS:
        did, phi, _ = case.field("phi_s", p, t)
        res["did"].append(did)
        res["phi_s"].append(phi)
        res["p_t"].append(case.field("p_t", p, t)[1])
        _, a, v = case.field("pv_s", p, t)
        res["pv_s_p"].append(a)
        res["pv_s_v"].append(v)
        _, a, v = case.field("pv_t", p, t)
        res["pv_t_p"].append(a)
        res["pv_t_v"].append(v)
    out["pts"], out["types"] = pts, types
    out.update({k: np.array(v) for k, v in res.items()})
    bd = np.array([b[:4] for b in boundary_points], np.float64)
    btypes = np.array([b[4] for b in boundary_points], np.int32)
    phib, pb, vb = [], [], []
    for did, t, z, e, ty in boundary_points:
        phib.append(case.boundary("phi_s_bd", did, t, z, e, ty)[0])
        a, v = case.boundary("pv_t_bd", did, t, z, e, ty)
        pb.append(a)
        vb.append(v)
    out.update(bd=bd, btypes=btypes, phi_s_bd=np.array(phib), pv_t_bd_p=np.array(pb), pv_t_bd_v=np.array(vb))
    np.savez_compressed(os.path.join(OUT, out_name), **out)


def checksum_weights(n):
    """Fixed weights of the array checksums (the tests rebuild them the same way)."""
    return np.cos(0.7 * np.arange(n) + 0.3)


def make_sphere216():
    """The 216-quad configuration (the benchmark's workload) solved by the
    reference: sampled rows, a random-phase product and the absolute row sums
    of every coefficient matrix, the full P, dP, pv, dpv of both domains and
    the forces of both rules.  Takes several minutes on a few host threads."""
    tmp = tempfile.mkdtemp(prefix="golden_")
    files = meshgen.write_inputs(tmp, **meshgen.CONFIGS["sphere216"])
    case = refwrap.RefCase(*files)
    mats = case.solve(tmp)
    rng = np.random.default_rng(20241207)
    out = {}
    for d in range(case.MN + 1):
        N = 4 * case.dom_ne[d]
        x = np.exp(2j * np.pi * rng.random(N))
        out["x%d" % d] = x
        for name in ("G", "H") + (("dG", "dH") if d > 0 else ()):
            M = mats["%s%d" % (name, d)]
            rows = np.sort(rng.choice(M.shape[0], 6, replace=False))
            out["%s%d_rows" % (name, d)] = rows
            out["%s%d_sample" % (name, d)] = M[rows]
            out["%s%d_Mx" % (name, d)] = M @ x
            out["%s%d_abs" % (name, d)] = np.abs(M).sum(axis=1)
        out["dF%d" % d] = mats["dF%d" % d]
        P, dP, pv, dpv = case.solution(d)
        out.update({"P%d" % d: P, "dP%d" % d: dP, "pv%d" % d: pv, "dpv%d" % d: dpv})
    out["F0"], out["N0"] = case.force(0)
    out["F1"], out["N1"] = case.force(1)
    np.savez_compressed(os.path.join(OUT, "sphere216.npz"), **out)


def make_rot():
    """54 quads turned about a generic axis (no point of one element shares its
    height with another's by symmetry): P, dP, pv, dpv, both force rules and
    the field and boundary values of fields24.npz's point lists (the matrices
    are left out: the 24-quad fixtures cover them)."""
    case = make_solve("sphere54_rot", "sphere54_rot.npz")
    g = dict(np.load(os.path.join(OUT, "sphere54_rot.npz")))
    np.savez_compressed(os.path.join(OUT, "sphere54_rot.npz"),
                        **{k: v for k, v in g.items() if not k.startswith(("G", "H", "dG", "dH", "dF"))})
    make_fields(case, "fields54_rot.npz")


# The solved systems the reference ships: (name, directory, .dat file or None, mesh)
SHIPPED = [("ex", "", "ex.dat", "sphere_m1.msh"), ("veri", "verification", None, "sphere_m1.msh"),
           ("ex1", "analysis_sample1", "ex1.dat", "sphere_m1.msh"), ("ex2", "analysis_sample2", "ex2.dat", "sphere_m3.msh")]


def parse_example1_log(path):
    """p, v (type 0 and 1) at r = (-0.03, 0.01, 0.002) and F, N (type 0 and 1)
    as printed by the reference's example1.c."""
    import re
    cplx = []
    vecs = []
    for line in open(path):
        m = re.match(r"\s*(p|vx|vy|vz)\s*=\s*(\S+)\s*([+-]\S+)\s*I", line)
        if m:
            cplx.append(complex(float(m.group(2)), float(m.group(3))))
        m = re.match(r"\s*[FN] = \(([^)]*)\)", line)
        if m:
            vecs.append([float(v) for v in m.group(1).split(",")])
    assert len(cplx) == 8 and len(vecs) == 4, path
    return {"p_t0": cplx[0], "v_t0": np.array(cplx[1:4]), "p_t1": cplx[4], "v_t1": np.array(cplx[5:8]),
            "F0": np.array(vecs[0]), "N0": np.array(vecs[1]), "F1": np.array(vecs[2]), "N1": np.array(vecs[3])}


def make_shipped(ref_dir):
    """Fixtures of the reference's shipped solved systems: the four input files
    as text (the mesh zlib-compressed), the values its example1.log prints and,
    where the .dat ships, the stored solution: P, dP of every domain in full,
    pv, dpv on 48 seeded elements per domain plus weighted sums over all
    elements (checksum_weights) and the matching sums of absolute values."""
    import zlib
    for name, sub, dat, msh in SHIPPED:
        base = os.path.join(ref_dir, sub)
        out = {"name": name}
        for f in ("pw.txt", "periodicity.txt", "medium.txt"):
            out[f.split(".")[0]] = open(os.path.join(base, f)).read()
        out["mesh_name"] = msh
        out["mesh_z"] = np.frombuffer(zlib.compress(open(os.path.join(base, msh), "rb").read(), 9), np.uint8)
        out.update(parse_example1_log(os.path.join(base, "example1.log")))
        if dat is not None:
            case = refwrap.RefCase.from_dat(os.path.join(base, dat))
            rng = np.random.default_rng(20241208)
            out["MN"] = case.MN
            out["dom_ne"] = np.array(case.dom_ne)
            for d in range(case.MN + 1):
                P, dP, pv, dpv = case.solution(d)
                out["P%d" % d], out["dP%d" % d] = P, dP
                idx = np.sort(rng.choice(case.dom_ne[d], 48, replace=False))
                out["idx%d" % d] = idx
                out["pv%d" % d], out["dpv%d" % d] = pv[idx], dpv[idx]
                w = checksum_weights(pv.size)
                for k, a in (("pv", pv), ("dpv", dpv)):
                    out["%s%d_sum" % (k, d)] = np.dot(w, a.ravel())
                    out["%s%d_abs" % (k, d)] = np.dot(np.abs(w), np.abs(a.ravel()))
        np.savez_compressed(os.path.join(OUT, "shipped_%s.npz" % name), **out)
        print("shipped_%s.npz" % name)


def main():
    rng = np.random.default_rng(20241203)
    if sys.argv[1:] == ["tri"]:
        case = make_solve("tri80", "tri80.npz")
        make_fields(case, "fields_tri80.npz", TRI_BOUNDARY_POINTS)
        print("tri80.npz, fields_tri80.npz written to", OUT)
        return
    if sys.argv[1:] == ["far"]:
        make_far_pairs()
        make_far_pairs("tri320", "far_tri320.npz", 300, 60)
        print("far216.npz, far_tri320.npz written to", OUT)
        return
    if sys.argv[1:] == ["fartri1280"]:
        make_far_pairs("tri1280", "far_tri1280.npz", 300, 60)
        print("far_tri1280.npz written to", OUT)
        return
    if sys.argv[1:] == ["tiers"]:
        make_tier_pairs()
        print("tiers1536.npz written to", OUT)
        return
    if sys.argv[1:] == ["near"]:
        make_near_pairs()
        print("near216.npz written to", OUT)
        return
    if sys.argv[1:] == ["sphere216"]:
        make_sphere216()
        print("sphere216.npz written to", OUT)
        return
    if sys.argv[1:] == ["rot"]:
        make_rot()
        print("sphere54_rot.npz, fields54_rot.npz written to", OUT)
        return
    if sys.argv[1:2] == ["shipped"]:
        make_shipped(sys.argv[2] if len(sys.argv) > 2 else os.environ.get("BEM_REFERENCE_DIR", "/root/reference"))
        return
    if sys.argv[1:] == ["plane"]:
        make_plane()
        print("qpgf_plane.npz written to", OUT)
        return
    if sys.argv[1:] == ["fields"]:
        tmp = tempfile.mkdtemp(prefix="golden_")
        files = meshgen.write_inputs(tmp, **meshgen.CONFIGS["sphere24"])
        case = refwrap.RefCase(*files)
        case.solve(tmp)
        make_fields(case)
        print("fields24.npz written to", OUT)
        return
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
    make_plane()
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
    make_fields(case)
    print("fixtures written to", OUT)


if __name__ == "__main__":
    main()
