"""Synthetic inputs in the reference's file formats.

* cube-sphere / spheroid meshes of bilinear quadrilaterals written as gmsh 2.2
  ASCII with the reference's paired element records (each element twice: once
  with the interior medium as physical tag and an outward normal, once with
  the open-region tag 99 and reversed node order, as read by read_mesh_data,
  bem3_aw_qd2.c:531-828);
* the plane-wave, periodicity and medium text files (aw_pw.c:3-82,
  bem3_aw_qd2.c:424-519).

The host medium is water-like (rho0 = 1000, c0 = 1500) with wavelength 1,
i.e. f = 1500 Hz and k0 = 2 pi, so lengths are in units of the host wavelength.
"""
import math
import os

import numpy as np

RHO0, C0 = 1000.0, 1500.0


def rotation_matrix(axis, deg):
    """Rotation by deg degrees about axis (Rodrigues' formula)."""
    a = np.asarray(axis, dtype=float)
    a = a / np.linalg.norm(a)
    th = math.radians(deg)
    K = np.array([[0.0, -a[2], a[1]], [a[2], 0.0, -a[0]], [-a[1], a[0], 0.0]])
    return np.eye(3) + math.sin(th) * K + (1.0 - math.cos(th)) * (K @ K)


def cube_sphere(n, semi_axes=(0.3, 0.3, 0.3), rot_y_deg=0.0, center=(0.0, 0.0, 0.0), rot=None):
    """Equiangular cube-sphere with 6 n^2 quads mapped to an ellipsoid.

    rot = (axis, degrees): a further rotation after the one about y, e.g. about
    a generic axis so that no mirror plane of the mesh is vertical and no two
    quadrature points of different elements share a height by symmetry.
    Returns (nodes [Nn,3], quads [Ne,4] of 0-based node indices) with every
    quad ordered so that (r1-r0) x (r3-r0) points out of the body."""
    a = np.linspace(-math.pi / 4, math.pi / 4, n + 1)
    t = np.tan(a)
    faces = []
    for axis in range(3):
        for sgn in (1.0, -1.0):
            u, v = np.meshgrid(t, t, indexing="ij")
            p = np.zeros((n + 1, n + 1, 3))
            p[..., axis] = sgn
            p[..., (axis + 1) % 3] = u
            p[..., (axis + 2) % 3] = v
            faces.append(p)
    key_to_id, nodes, quads = {}, [], []

    def node_id(x):
        x = x / np.linalg.norm(x)
        k = tuple(np.round(x, 12))
        if k not in key_to_id:
            key_to_id[k] = len(nodes)
            nodes.append(x)
        return key_to_id[k]

    for p in faces:
        ids = [[node_id(p[i, j]) for j in range(n + 1)] for i in range(n + 1)]
        for i in range(n):
            for j in range(n):
                quads.append([ids[i][j], ids[i + 1][j], ids[i + 1][j + 1], ids[i][j + 1]])
    nodes = np.array(nodes) * np.array(semi_axes, dtype=float)
    if rot_y_deg:
        th = math.radians(rot_y_deg)
        R = np.array([[math.cos(th), 0.0, math.sin(th)], [0.0, 1.0, 0.0], [-math.sin(th), 0.0, math.cos(th)]])
        nodes = nodes @ R.T
    if rot is not None:
        nodes = nodes @ rotation_matrix(*rot).T
    nodes = nodes + np.array(center, dtype=float)
    quads = np.array(quads, dtype=np.int64)
    c = nodes.mean(axis=0)
    for q in quads:
        r = nodes[q]
        nrm = np.cross(r[1] - r[0], r[3] - r[0])
        if np.dot(nrm, r.mean(axis=0) - c) < 0:
            q[[1, 3]] = q[[3, 1]]
    return nodes, quads


def icosphere(level, semi_axes=(0.3, 0.3, 0.3), rot_y_deg=0.0, center=(0.0, 0.0, 0.0)):
    """Icosahedron subdivided `level` times (20 4^level triangles), projected to
    the unit sphere and mapped to an ellipsoid.  Returns (nodes [Nn,3],
    triangles [Ne,3] of 0-based node indices) with (r1-r0) x (r2-r0) pointing
    out of the body."""
    g = (1.0 + math.sqrt(5.0)) / 2.0
    verts = [(-1, g, 0), (1, g, 0), (-1, -g, 0), (1, -g, 0), (0, -1, g), (0, 1, g), (0, -1, -g), (0, 1, -g),
             (g, 0, -1), (g, 0, 1), (-g, 0, -1), (-g, 0, 1)]
    verts = [np.array(v, float) / np.linalg.norm(v) for v in verts]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6),
             (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10),
             (8, 6, 7), (9, 8, 1)]
    for _ in range(level):
        mid = {}

        def midpoint(a, b):
            key = (min(a, b), max(a, b))
            if key not in mid:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                mid[key] = len(verts) - 1
            return mid[key]
        nf = []
        for a, b, c in faces:
            ab, bc, ca = midpoint(a, b), midpoint(b, c), midpoint(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    nodes = np.array(verts) * np.array(semi_axes)
    th = math.radians(rot_y_deg)
    R = np.array([[math.cos(th), 0, math.sin(th)], [0, 1, 0], [-math.sin(th), 0, math.cos(th)]])
    nodes = nodes @ R.T + np.array(center)
    tris = np.array(faces, dtype=int)
    c = nodes.mean(axis=0)
    for t in tris:
        r = nodes[t]
        if np.dot(np.cross(r[1] - r[0], r[2] - r[0]), r.mean(axis=0) - c) < 0:
            t[[1, 2]] = t[[2, 1]]
    return nodes, tris


def write_msh(path, nodes, elems, inner_tag=1, open_tag=99):
    """gmsh 2.2 ASCII: every element twice (the body side, then the open side
    with the reversed orientation); quads are type 3, triangles type 2."""
    lines = ["$MeshFormat", "2.2 0 8", "$EndMeshFormat", "$Nodes", str(len(nodes))]
    for i, x in enumerate(nodes):
        lines.append("%d %.17g %.17g %.17g" % (i + 1, x[0], x[1], x[2]))
    lines += ["$EndNodes", "$Elements", str(2 * len(elems))]
    for e, q in enumerate(elems):
        v = [int(x) + 1 for x in q]
        et = 3 if len(v) == 4 else 2
        rev = [v[0]] + v[:0:-1]
        lines.append("%d %d 2 %d %d %s" % (2 * e + 1, et, inner_tag, 1, " ".join(map(str, v))))
        lines.append("%d %d 2 %d %d %s" % (2 * e + 2, et, open_tag, 1, " ".join(map(str, rev))))
    lines.append("$EndElements")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def write_inputs(dirname, *, n=6, semi_axes=(0.3, 0.3, 0.3), rot_y_deg=0.0, lattice=((0.8, 0.0), (0.0, 0.8)),
                 theta_deg=20.0, phi_deg=30.0, rho_in=1.2 * RHO0, c_in=1.5 * C0, wavelength=1.0, amp=(1.0, 0.0),
                 ico=None, rot=None, center=(0.0, 0.0, 0.0)):
    """Write pw.txt, periodicity.txt, medium.txt and body.msh; returns the 4 paths.
    ico: icosphere subdivision level (triangles) instead of the cube-sphere;
    rot, center: see cube_sphere (quads only)."""
    os.makedirs(dirname, exist_ok=True)
    f = C0 / wavelength
    pw = os.path.join(dirname, "pw.txt")
    with open(pw, "w") as fp:
        fp.write("## plane wave\n# rho0[kg/m^3] c0[m/s] f[Hz]\n%.17g %.17g %.17g\n" % (RHO0, C0, f))
        fp.write("# real(p) imag(p) tx ty tz theta psi\n%.17g %.17g 0.0 0.0 0.0 %.17g %.17g\n"
                 % (amp[0], amp[1], math.radians(theta_deg), math.radians(phi_deg)))
    per = os.path.join(dirname, "periodicity.txt")
    with open(per, "w") as fp:
        fp.write("## periodicity\n# ps d1x d1y d2x d2y\n1 %.17g %.17g %.17g %.17g\n"
                 % (lattice[0][0], lattice[0][1], lattice[1][0], lattice[1][1]))
    med = os.path.join(dirname, "medium.txt")
    with open(med, "w") as fp:
        fp.write("## medium\n# number of medium\n1\n# rho0 c0\n%.17g %.17g\n" % (rho_in, c_in))
    msh = os.path.join(dirname, "body.msh")
    if ico is not None:
        nodes, elems = icosphere(ico, semi_axes, rot_y_deg)
    else:
        nodes, elems = cube_sphere(n, semi_axes, rot_y_deg, center, rot)
    write_msh(msh, nodes, elems)
    return pw, per, med, msh


# The configurations of the benchmark: names, sizes and parameters.
CONFIGS = {
    # one sphere r = 0.3, 216 quads, square lattice 0.8, theta 20 deg, phi 30 deg
    "sphere216": dict(n=6, semi_axes=(0.3, 0.3, 0.3), lattice=((0.8, 0.0), (0.0, 0.8)), theta_deg=20.0, phi_deg=30.0),
    # triangles: icosphere r = 0.3 with 80 triangles (fixtures) and 1280 triangles, triangular lattice 0.8
    "tri80": dict(ico=1, semi_axes=(0.3, 0.3, 0.3), lattice=((0.8, 0.0), (0.4, 0.69282032302755091741)),
                  theta_deg=20.0, phi_deg=30.0),
    # near-normal incidence (the reference rejects kx = 0 or ky = 0)
    "tri320": dict(ico=2, semi_axes=(0.3, 0.3, 0.3), lattice=((0.8, 0.0), (0.4, 0.69282032302755091741)),
                   theta_deg=20.0, phi_deg=30.0),
    "tri1280": dict(ico=3, semi_axes=(0.3, 0.3, 0.3), lattice=((0.8, 0.0), (0.4, 0.69282032302755091741)),
                    theta_deg=1e-6, phi_deg=45.0),
    # small case for fixtures and smoke tests: 24 quads, same physics
    "sphere24": dict(n=2, semi_axes=(0.3, 0.3, 0.3), lattice=((0.8, 0.0), (0.0, 0.8)), theta_deg=20.0, phi_deg=30.0),
    # 54 quads turned about a generic axis and moved off the lattice plane: no
    # quadrature point shares its height with another element's point by
    # symmetry, so the reference's lattice sums never stop on an exactly zero
    # derivative row there
    "sphere54_rot": dict(n=3, semi_axes=(0.3, 0.3, 0.3), rot=((1.0, 2.0, 3.0), 37.0), center=(0.0, 0.0, 0.013),
                         lattice=((0.8, 0.0), (0.0, 0.8)), theta_deg=20.0, phi_deg=30.0),
    # 1536 quads (the batched-sweep mesh), one incidence
    "sphere1536": dict(n=16, semi_axes=(0.3, 0.3, 0.3), lattice=((0.8, 0.0), (0.0, 0.8)), theta_deg=20.0, phi_deg=30.0),
    # prolate spheroid 0.2/0.2/0.4 rotated 30 deg about y, 6144 quads, oblique lattice
    "spheroid6144": dict(n=32, semi_axes=(0.2, 0.2, 0.4), rot_y_deg=30.0, lattice=((1.0, 0.0), (0.3, 0.9)),
                         theta_deg=35.0, phi_deg=15.0),
}


def describe(name):
    """Element count and kind, unknowns and parameters of a configuration."""
    c = CONFIGS[name]
    if c.get("ico") is not None:
        ne, npe, kind = 20 * 4 ** c["ico"], 3, "linear triangles (icosphere)"
    else:
        ne, npe, kind = 6 * c["n"] ** 2, 4, "bilinear quads (cube-sphere)"
    return {"elements": ne, "element_kind": kind, "unknowns": 2 * npe * ne, "semi_axes": list(c["semi_axes"]),
            "lattice": [list(v) for v in c["lattice"]], "theta_deg": c["theta_deg"], "phi_deg": c["phi_deg"]}
