"""bemgpu_assemble_domain_static: the assembly entry point that allocates
nothing, for callers that cannot allocate device memory (their device memory
belongs to another allocator's fixed pool, or they reach the library through a
foreign-function interface that can pass device buffers but not manage CUDA
allocations).

It is called through the C ABI with caller-owned device buffers (torch
tensors) and must give the same matrices as the regular context path
(bemgpu_assemble + bemgpu_get_matrix), within the parity tolerance of the
other tests (1e-10 relative to the row maximum), on two calls in a row: the
second call finds the first call's scratch contents in the shared array.

This file is collected last on purpose and builds its case itself, so it
passes both alone in a fresh process and after the other tests.
"""
import ctypes
import os
import struct
import tempfile

import numpy as np
import pytest

from conftest import ROOT  # noqa: F401

pytestmark = pytest.mark.gpu


def parse_dat(path):
    """Element tables and domain lists from a .dat file (bem3_aw_qd2.c:185-224 layout)."""
    b = open(path, "rb").read()
    qp = np.frombuffer(b, np.float64, 8, 744)  # AQD2.bd.qd: k, kx, ky, kz, d1, d2
    MN = struct.unpack_from("i", b, 440)[0]
    Nn, Ne = struct.unpack_from("ii", b, 808)
    o = 2720
    k0 = np.frombuffer(b, np.float64, MN + 1, o + 2 * 8 * (MN + 1))
    o += 4 * 8 * (MN + 1) + 2 * 16 * (MN + 1) + 240
    rn = np.frombuffer(b, np.float64, 3 * (Nn + 1), o).reshape(-1, 3); o += 24 * (Nn + 1)
    ed = np.frombuffer(b, np.int32, 4 * (Ne + 1), o).reshape(-1, 4); o += 16 * (Ne + 1)
    o += 16 * (Ne + 1) + 3 * 4 * (Ne + 1)  # eni, md, sd, gd
    ren = np.frombuffer(b, np.float64, 12 * (Ne + 1), o).reshape(-1, 12); o += 96 * (Ne + 1)
    o += 96 * (Ne + 1) + 2 * 64 * (Ne + 1)  # wen, Pi, dPi
    sids = []
    for _ in range(MN + 1):
        ne = struct.unpack_from("i", b, o)[0]; o += 4
        sids.append(np.frombuffer(b, np.int32, ne + 1, o)[1:].copy()); o += 4 * (ne + 1)
        o += 2 * 64 * (ne + 1) + 2 * 192 * (ne + 1)
    # bilinear element constants (init_elem_const, bem3_aw_qd2.c:941-972)
    rc = np.stack([rn[ed[1:, j]] for j in range(4)], axis=2)  # [Ne][3][4]
    cr = np.stack([0.25 * (rc[..., 0] + rc[..., 1] + rc[..., 2] + rc[..., 3]),
                   0.25 * (-rc[..., 0] + rc[..., 1] + rc[..., 2] - rc[..., 3]),
                   0.25 * (-rc[..., 0] - rc[..., 1] + rc[..., 2] + rc[..., 3]),
                   0.25 * (rc[..., 0] - rc[..., 1] + rc[..., 2] - rc[..., 3])], axis=2)
    cw = np.zeros((Ne, 3, 3))
    for k, (a, c) in enumerate([(1, 2), (2, 0), (0, 1)]):
        A, B = rc[:, a], rc[:, c]
        cw[:, k, 0] = 0.125 * ((A[:, 0] - A[:, 2]) * (B[:, 1] - B[:, 3]) - (A[:, 1] - A[:, 3]) * (B[:, 0] - B[:, 2]))
        cw[:, k, 1] = 0.125 * ((A[:, 2] - A[:, 3]) * (B[:, 0] - B[:, 1]) - (A[:, 0] - A[:, 1]) * (B[:, 2] - B[:, 3]))
        cw[:, k, 2] = 0.125 * ((A[:, 1] - A[:, 2]) * (B[:, 0] - B[:, 3]) - (A[:, 0] - A[:, 3]) * (B[:, 1] - B[:, 2]))
    bdc = np.einsum("ed,ed->e", cr[:, :, 1], cw[:, :, 2])
    plane = np.abs(bdc / (np.linalg.norm(cr[:, :, 1], axis=1) * np.linalg.norm(cw[:, :, 2], axis=1))) < 1e-15
    return dict(qp=qp.copy(), k0=k0.copy(), cr=cr.reshape(Ne, 12), cw=cw.reshape(Ne, 9), ren=ren[1:].copy(),
                plane=plane.astype(np.uint8), sids=sids)


def rel_rows(a, b):
    s = np.max(np.abs(b), axis=1, keepdims=True)
    s[s == 0] = 1.0
    return float(np.max(np.abs(a - b) / s))


def _entry():
    from bem3_aw_qd2_b200 import api
    _, g = api.libs()
    fn = g.bemgpu_assemble_domain_static
    vp = ctypes.c_void_p
    fn.argtypes = [vp, vp, vp, vp, vp, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_double,
                   vp, vp, vp, vp, vp, vp]
    fn.restype = ctypes.c_int
    return fn


def _static_matrices(fn, t, dom, stream, dev, outs=None):
    """One call of the entry point for domain dom of the parsed case t into
    caller-owned torch buffers (made once and passed back in as outs)."""
    import torch
    sid = torch.tensor(t["sids"][dom], dtype=torch.int32, device=dev)
    ne = len(t["sids"][dom])
    N = 4 * ne
    if outs is None:
        outs = dict(G=torch.empty((N, N), dtype=torch.complex128, device=dev),
                    H=torch.empty((N, N), dtype=torch.complex128, device=dev),
                    dF=torch.empty((N, 3), dtype=torch.float64, device=dev),
                    dG=torch.empty((2 * N, N), dtype=torch.complex128, device=dev) if dom else None,
                    dH=torch.empty((2 * N, N), dtype=torch.complex128, device=dev) if dom else None,
                    sid=sid)
    for k in ("G", "H", "dF", "dG", "dH"):
        if outs[k] is not None:
            outs[k].fill_(float("nan"))
    torch.cuda.synchronize()
    qp = np.ascontiguousarray(t["qp"])
    rc = fn(t["cr_d"].data_ptr(), t["cw_d"].data_ptr(), t["ren_d"].data_ptr(), t["plane_d"].data_ptr(),
            outs["sid"].data_ptr(), ne, qp.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 1 if dom == 0 else 0,
            float(t["k0"][dom]), outs["G"].data_ptr(), outs["H"].data_ptr(),
            outs["dG"].data_ptr() if outs["dG"] is not None else None,
            outs["dH"].data_ptr() if outs["dH"] is not None else None, outs["dF"].data_ptr(), stream.cuda_stream)
    assert rc == 0, "domain %d returned %d" % (dom, rc)
    torch.cuda.synchronize()
    return outs


def _case_tables(config):
    import torch
    from bem3_aw_qd2_b200 import api, meshgen
    h, _ = api.libs()
    h.aqd2_set_verbose(0)
    d = tempfile.mkdtemp(prefix="bem_static_")
    case = api.Case.from_files(*meshgen.write_inputs(d, **meshgen.CONFIGS[config]))
    case.solve()
    datp = os.path.join(d, "case.dat")
    case.dat_write(datp)
    t = parse_dat(datp)
    dev = torch.device("cuda:0")
    for k in ("cr", "cw", "ren", "plane"):
        t[k + "_d"] = torch.tensor(t[k], device=dev)
    return case, t, dev


def test_static_assembly_matches_context_path_twice():
    """24 quads: the same matrices as the context path and as the reference's
    own (tests/golden/sphere24.npz), on two calls in a row."""
    import torch
    case, t, dev = _case_tables("sphere24")
    gold = np.load(os.path.join(ROOT, "tests", "golden", "sphere24.npz"))
    fn = _entry()
    stream = torch.cuda.Stream(device=dev)
    for call in range(2):
        for dom in (0, 1):
            N = 4 * len(t["sids"][dom])
            o = _static_matrices(fn, t, dom, stream, dev)
            for k in ("G", "H") + (("dG", "dH") if dom else ()):
                got = o[k].cpu().numpy()
                assert rel_rows(got, case.matrix(dom, k, N)) < 1e-10, (call, dom, k)
                assert rel_rows(got, gold["%s%d" % (k, dom)]) < 1e-10, (call, dom, k)
            dF = o["dF"].cpu().numpy()
            assert np.max(np.abs(dF - case.matrix(dom, "dF", N))) < 1e-10
            ref = gold["dF%d" % dom]
            assert np.max(np.abs(dF[:, 0] - ref[:, 0])) < 1e-10 * np.max(np.abs(ref[:, 0]))
            assert np.max(np.abs(dF[:, 1:] - ref[:, 1:])) < 1e-11
    case.close()


def test_static_assembly_with_far_pairs_allocates_nothing():
    """216 quads, where most regular pairs are far: the entry point keeps the
    reference's 12 x 12 rule on every pair, so it is compared with a context
    set to that rule (bemgpu_set_far_rule(ctx, 0)).  The second call runs with
    the device's free memory unchanged: nothing is allocated."""
    import torch
    case, t, dev = _case_tables("sphere216")
    case.set_far_rule(0)
    case.run_device()
    fn = _entry()
    stream = torch.cuda.Stream(device=dev)
    outs = {dom: _static_matrices(fn, t, dom, stream, dev) for dom in (0, 1)}  # warm: loads the kernels
    free_before = torch.cuda.mem_get_info(dev)[0]
    for dom in (0, 1):
        _static_matrices(fn, t, dom, stream, dev, outs[dom])
    free_after = torch.cuda.mem_get_info(dev)[0]
    assert free_after == free_before, (free_before, free_after)
    for dom in (0, 1):
        N = 4 * len(t["sids"][dom])
        for k in ("G", "H") + (("dG", "dH") if dom else ()):
            assert rel_rows(outs[dom][k].cpu().numpy(), case.matrix(dom, k, N)) < 1e-10, (dom, k)
        assert np.max(np.abs(outs[dom]["dF"].cpu().numpy() - case.matrix(dom, "dF", N))) < 1e-10
    case.close()


def test_static_assembly_rejects_bad_arguments():
    """Sizes beyond the limit and missing pointers are error returns (-2),
    checked on the host before any device work."""
    import torch
    fn = _entry()
    qp = np.zeros(8)
    qpp = qp.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    rc = fn(None, None, None, None, None, 1537, qpp, 1, 1.0, None, None, None, None, None, None)
    assert rc == -2
    rc = fn(None, None, None, None, None, 4, qpp, 1, 1.0, None, None, None, None, None, None)
    assert rc == -2
    dev = torch.device("cuda:0")
    ne, N = 1, 4
    buf = {k: torch.zeros(n, dtype=torch.float64, device=dev) for k, n in
           (("cr", 12), ("cw", 9), ("ren", 12), ("G", 2 * N * N), ("H", 2 * N * N), ("dF", 3 * N))}
    plane = torch.zeros(1, dtype=torch.uint8, device=dev)
    sid = torch.ones(1, dtype=torch.int32, device=dev)
    args = [buf["cr"].data_ptr(), buf["cw"].data_ptr(), buf["ren"].data_ptr(), plane.data_ptr(), sid.data_ptr(), ne,
            qpp]
    # an interior domain (periodic = 0) without its dG / dH outputs
    rc = fn(*args, 0, 1.0, buf["G"].data_ptr(), buf["H"].data_ptr(), None, None, buf["dF"].data_ptr(), None)
    assert rc == -2
    # a periodic domain without H
    rc = fn(*args, 1, 1.0, buf["G"].data_ptr(), None, None, None, buf["dF"].data_ptr(), None)
    assert rc == -2
