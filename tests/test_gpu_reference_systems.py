"""The default device path (far-pair rule on, Ewald parameter by rule and by
the autotuner) against systems the reference itself solved:

* the solved systems the reference ships (its ex.dat with sphere_m1.msh on a
  square lattice, analysis_sample1/ex1.dat on a triangular lattice,
  analysis_sample2/ex2.dat with three media, and the verification/ inputs whose
  .dat is not shipped): the device solves the shipped input files and must give
  the P, dP, pv, dpv stored in the .dat files and the values the reference's
  example1.log prints (field at a point, force and torque with both rules);
* the 216-quad benchmark configuration solved by the reference here
  (tests/golden/sphere216.npz: sampled matrix rows, products with a
  random-phase vector, P, dP, pv, dpv, forces);
* a 54-quad sphere turned about a generic axis (sphere54_rot.npz,
  fields54_rot.npz), where no lattice-plane ties occur, at 1e-9 for the
  9-point force and the boundary values too;
* the reference's own driver programs (aw_d3qd2_bv_solver.c, example1.c)
  compiled unchanged against this library.

Tolerances (stated here, used below):
  matrix entries               1e-10 of the row maximum (sampled rows); the
                               product with a unit-modulus vector 1e-10 of the
                               row's absolute sum
  P, dP, pv, dpv               1e-9 of the array maximum; weighted sums over all
                               elements 1e-9 of the weighted absolute sum
  field values, type-0 force   1e-9 relative
  torque                       1e-9 of |F| times the body's radius (the torque
                               is a small difference of large moments: its own
                               relative error means nothing)
  9-point force on the mirror-symmetric meshes (the cube-spheres, and the
                               shipped gmsh spheres, whose 9-point targets share
                               heights with other elements' points)
                               TOL_RULE = 1e-7: the reference's own lattice-plane
                               rounding noise (test_gpu_fields.py); measured on
                               the shipped systems 3e-11 (ex), 9e-8 (verification),
                               7e-12 (ex1)
"""
import os
import re
import subprocess
import tempfile
import zlib

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu
GOLD = os.path.join(ROOT, "tests", "golden")
LIB = os.path.join(ROOT, "bem3_aw_qd2_b200", "lib")
TOL = 1e-9
TOL_MAT = 1e-10
TOL_RULE = 1e-7
R_FIELD = (-0.03, 0.01, 0.002)  # example1.c's field point


def rel_max(a, b):
    s = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / (s if s > 0 else 1.0))


def checksum_weights(n):
    return np.cos(0.7 * np.arange(n) + 0.3)


def write_shipped_inputs(g, d):
    """The shipped input files of one fixture, written to directory d."""
    names = []
    for key in ("pw", "periodicity", "medium"):
        path = os.path.join(d, key + ".txt")
        with open(path, "w") as f:
            f.write(str(g[key]))
        names.append(path)
    path = os.path.join(d, str(g["mesh_name"]))
    with open(path, "wb") as f:
        f.write(zlib.decompress(g["mesh_z"].tobytes()))
    names.append(path)
    return names


def parse_example1(text):
    """p, v (type 0, 1) and F, N (type 0, 1) from example1.c's output."""
    cplx, vecs = [], []
    for line in text.splitlines():
        m = re.match(r"\s*(p|vx|vy|vz)\s*=\s*(\S+)\s*([+-]\S+)\s*I", line)
        if m:
            cplx.append(complex(float(m.group(2)), float(m.group(3))))
        m = re.match(r"\s*[FN] = \(([^)]*)\)", line)
        if m:
            vecs.append([float(v) for v in m.group(1).split(",")])
    assert len(cplx) == 8 and len(vecs) == 4, text[-2000:]
    return {"p_t0": cplx[0], "v_t0": np.array(cplx[1:4]), "p_t1": cplx[4], "v_t1": np.array(cplx[5:8]),
            "F0": np.array(vecs[0]), "N0": np.array(vecs[1]), "F1": np.array(vecs[2]), "N1": np.array(vecs[3])}


def check_log_values(got, g, radius, tol_force1=TOL_RULE, tol_print=0.0):
    """got: dict as parse_example1 returns; g: the fixture; radius: the body's
    size (torque scale).  tol_print adds the rounding of 15 printed digits when
    got comes from printed text."""
    t = TOL + tol_print
    for k in ("p_t0", "p_t1"):
        assert abs(got[k] - g[k]) <= t * abs(g[k]), (k, got[k], g[k])
    for k in ("v_t0", "v_t1"):
        assert np.linalg.norm(got[k] - g[k]) <= t * np.linalg.norm(g[k]), (k, got[k], g[k])
    for ty, tf in (("0", t), ("1", tol_force1 + tol_print)):
        F, Fr, N, Nr = got["F" + ty], g["F" + ty], got["N" + ty], g["N" + ty]
        assert np.linalg.norm(F - Fr) <= tf * np.linalg.norm(Fr), ("F" + ty, F, Fr)
        assert np.linalg.norm(N - Nr) <= tf * np.linalg.norm(Fr) * radius, ("N" + ty, N, Nr)


def mesh_radius(g):
    """Largest distance of a mesh node from the origin (the torque centre)."""
    text = zlib.decompress(g["mesh_z"].tobytes()).decode().split("\n")
    i = text.index("$Nodes")
    pts = np.array([[float(x) for x in line.split()[1:4]] for line in text[i + 2:i + 2 + int(text[i + 1])]])
    return float(np.max(np.linalg.norm(pts, axis=1)))


def case_log_values(case):
    out = {}
    for ty in (0, 1):
        _, p, v = case.field("pv_t", R_FIELD, ty)
        out["p_t%d" % ty], out["v_t%d" % ty] = p, v
        out["F%d" % ty], out["N%d" % ty] = case.force(ty)
    return out


SHIPPED = ["ex", "veri", "ex1", "ex2"]


@pytest.fixture(scope="module", params=SHIPPED)
def shipped(request):
    from bem3_aw_qd2_b200 import api
    g = np.load(os.path.join(GOLD, "shipped_%s.npz" % request.param))
    d = tempfile.mkdtemp(prefix="bem_shipped_")
    case = api.Case.from_files(*write_shipped_inputs(g, d))
    case.solve()
    yield request.param, case, g
    case.close()


def test_shipped_solution_matches_dat(shipped):
    """P, dP in full and pv, dpv (48 elements per domain and weighted sums over
    all) against the arrays the reference stored in its .dat file."""
    name, case, g = shipped
    if "P0" not in g:
        pytest.skip("the reference ships no .dat for %s" % name)
    assert case.status() == 0
    for d in range(int(g["MN"]) + 1):
        ne = int(g["dom_ne"][d])
        P, dP, pv, dpv = case.solution(d, ne)
        assert rel_max(P, g["P%d" % d]) < TOL, (d, rel_max(P, g["P%d" % d]))
        assert rel_max(dP, g["dP%d" % d]) < TOL, (d, rel_max(dP, g["dP%d" % d]))
        idx = g["idx%d" % d]
        for k, a in (("pv", pv), ("dpv", dpv)):
            ref = g["%s%d" % (k, d)]
            assert np.max(np.abs(a[idx] - ref)) <= TOL * np.max(np.abs(ref)), (k, d)
            s = np.dot(checksum_weights(a.size), a.ravel())
            assert abs(s - g["%s%d_sum" % (k, d)]) <= TOL * float(g["%s%d_abs" % (k, d)]), (k, d)


def test_shipped_example1_values(shipped):
    """Field at example1.c's point and force / torque of both rules against
    the reference's example1.log of the same system."""
    name, case, g = shipped
    check_log_values(case_log_values(case), g, mesh_radius(g))


# ---- the 216-quad benchmark configuration, solved by the reference


@pytest.fixture(scope="module")
def sphere216():
    from bem3_aw_qd2_b200 import api, meshgen
    path = os.path.join(GOLD, "sphere216.npz")
    if not os.path.exists(path):
        pytest.skip("sphere216.npz not generated")
    d = tempfile.mkdtemp(prefix="bem216_")
    case = api.Case.from_files(*meshgen.write_inputs(d, **meshgen.CONFIGS["sphere216"]))
    case.solve()
    yield case, np.load(path)
    case.close()


def _check_sphere216(case, g):
    for d in (0, 1):
        N = 864
        for name in ("G", "H") + (("dG", "dH") if d else ()):
            M = case.matrix(d, name, N)
            rows = g["%s%d_rows" % (name, d)]
            ref = g["%s%d_sample" % (name, d)]
            scale = np.max(np.abs(ref), axis=1, keepdims=True)
            assert np.max(np.abs(M[rows] - ref) / scale) < TOL_MAT, (name, d)
            Mx = M @ g["x%d" % d]
            assert np.all(np.abs(Mx - g["%s%d_Mx" % (name, d)]) <= TOL_MAT * g["%s%d_abs" % (name, d)]), (name, d)
        dF = case.matrix(d, "dF", N)
        ref = g["dF%d" % d]
        assert np.max(np.abs(dF[:, 0] - ref[:, 0])) < TOL_MAT * np.max(np.abs(ref[:, 0]))
        assert np.max(np.abs(dF[:, 1:] - ref[:, 1:])) < 1e-11
        P, dP, pv, dpv = case.solution(d, 216)
        for k, a in (("P", P), ("dP", dP), ("pv", pv), ("dpv", dpv)):
            assert rel_max(a, g["%s%d" % (k, d)]) < TOL, (k, d, rel_max(a, g["%s%d" % (k, d)]))
    F, N = case.force(0)
    assert np.linalg.norm(F - g["F0"]) <= TOL * np.linalg.norm(g["F0"])
    assert np.linalg.norm(N - g["N0"]) <= TOL * np.linalg.norm(g["F0"]) * 0.3
    F, N = case.force(1)
    assert np.linalg.norm(F - g["F1"]) <= TOL_RULE * np.linalg.norm(g["F1"])
    assert np.linalg.norm(N - g["N1"]) <= TOL_RULE * np.linalg.norm(g["F1"]) * 0.3
    assert case.status() == 0


def test_sphere216_default_path(sphere216):
    """The benchmark's own path (far-pair rule, Ewald parameter by rule)."""
    case, g = sphere216
    _check_sphere216(case, g)


def test_sphere216_autotuned_ewald(sphere216):
    """The same with the autotuner's Ewald parameter (as bench.py runs it)."""
    case, g = sphere216
    scale = case.autotune()
    assert 0.25 <= scale <= 4.0
    case.run_device()
    _check_sphere216(case, g)
    case.set_ewald_scale(0.0)


# ---- a mesh without lattice-plane ties: the 9-point rule at 1e-9


@pytest.fixture(scope="module")
def rotated():
    from bem3_aw_qd2_b200 import api, meshgen
    d = tempfile.mkdtemp(prefix="bem54r_")
    case = api.Case.from_files(*meshgen.write_inputs(d, **meshgen.CONFIGS["sphere54_rot"]))
    case.solve()
    yield case, np.load(os.path.join(GOLD, "sphere54_rot.npz")), np.load(os.path.join(GOLD, "fields54_rot.npz"))
    case.close()


def test_rotated_solution_and_forces(rotated):
    case, g, f = rotated
    assert case.status() == 0
    for d in (0, 1):
        for k, a in zip(("P", "dP", "pv", "dpv"), case.solution(d, 54)):
            assert rel_max(a, g["%s%d" % (k, d)]) < TOL, (k, d)
    for ty, Fr, Nr in ((0, g["F0"], g["N0"]), (1, f["F1"], f["N1"])):
        F, N = case.force(ty)
        assert np.linalg.norm(F - Fr) <= TOL * np.linalg.norm(Fr), (ty, F, Fr)
        assert np.linalg.norm(N - Nr) <= TOL * np.linalg.norm(Nr), (ty, N, Nr)
    F, N = case.force(1, (0.05, -0.02, 0.1))
    assert np.linalg.norm(F - f["F1c"]) <= TOL * np.linalg.norm(f["F1c"])
    assert np.linalg.norm(N - f["N1c"]) <= TOL * np.linalg.norm(f["N1c"])


def test_rotated_boundary_and_field_values(rotated):
    """Every boundary value at 1e-9, the 9-point rule positions included."""
    case, _, f = rotated
    dom = f["bd"][:, 0].astype(int)
    phi, p, v = [], [], []
    for (did, t, z, e), ty in zip(f["bd"], f["btypes"]):
        phi.append(case.boundary("phi_s_bd", int(did), int(t), float(z), float(e), int(ty))[0])
        a, b = case.boundary("pv_t_bd", int(did), int(t), float(z), float(e), int(ty))
        p.append(a)
        v.append(b)
    for d in (0, 1):
        m = dom == d
        for got, key in ((np.array(phi), "phi_s_bd"), (np.array(p), "pv_t_bd_p"), (np.array(v), "pv_t_bd_v")):
            ref = f[key]
            err = np.abs(got - ref).reshape(len(ref), -1).max(axis=1)
            assert np.all(err[m] <= TOL * np.max(np.abs(ref[m]))), (key, d)
    for i, (pt, ty) in enumerate(zip(f["pts"], f["types"])):
        did, a, vv = case.field("pv_t", pt, int(ty))
        assert did == f["did"][i]
        assert abs(a - f["pv_t_p"][i]) <= TOL * np.max(np.abs(f["pv_t_p"]))
        assert np.max(np.abs(vv - f["pv_t_v"][i])) <= TOL * np.max(np.abs(f["pv_t_v"]))


# ---- the reference's driver programs, compiled unchanged against this library


def _run(cmd, cwd):
    r = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    return r.stdout


def test_reference_drivers_on_shipped_inputs():
    """aw_d3qd2_bv_solver (reference source, this library) solves the shipped
    ex.dat inputs on the GPU and writes a .dat; example1 (reference source,
    this library) reads it and prints the values of the reference's
    example1.log to the printed digits plus the 1e-9 tolerance."""
    solver, ex1 = os.path.join(LIB, "aw_d3qd2_bv_solver"), os.path.join(LIB, "example1.out")
    if not (os.path.exists(solver) and os.path.exists(ex1)):
        pytest.skip("driver programs not built (the reference sources were absent at build time)")
    g = np.load(os.path.join(GOLD, "shipped_ex.npz"))
    d = tempfile.mkdtemp(prefix="bem_drivers_")
    files = [os.path.basename(p) for p in write_shipped_inputs(g, d)]
    _run([solver] + files + ["out.dat"], d)
    got = parse_example1(_run([ex1, "out.dat"], d))
    check_log_values(got, g, mesh_radius(g), tol_print=1e-14)


def test_dat_from_library_read_by_reference():
    """The .dat written by the library (through the reference's own solver
    driver) is read by the reference's own example1 build (oracle/_ref) with
    the same printed results as the library's example1."""
    from bem3_aw_qd2_b200 import meshgen
    solver, ex1 = os.path.join(LIB, "aw_d3qd2_bv_solver"), os.path.join(LIB, "example1.out")
    ref_ex1 = os.path.join(ROOT, "oracle", "_ref", "example1.out")
    if not (os.path.exists(solver) and os.path.exists(ex1) and os.path.exists(ref_ex1)):
        pytest.skip("driver programs or oracle/_ref not built")
    d = tempfile.mkdtemp(prefix="bem_drivers24_")
    files = [os.path.basename(p) for p in meshgen.write_inputs(d, **meshgen.CONFIGS["sphere24"])]
    _run([solver] + files + ["s24.dat"], d)
    ours = parse_example1(_run([ex1, "s24.dat"], d))
    env_out = subprocess.run([ref_ex1, "s24.dat"], cwd=d, capture_output=True, text=True, timeout=900,
                             env=dict(os.environ, OMP_NUM_THREADS=str(min(16, os.cpu_count() or 1))))
    assert env_out.returncode == 0, env_out.stderr[-2000:]
    theirs = parse_example1(env_out.stdout)
    # the reference's 9-point force on this mirror-symmetric mesh carries its
    # lattice-plane rounding noise (TOL_RULE)
    check_log_values(ours, theirs, 0.3, tol_print=1e-14)
