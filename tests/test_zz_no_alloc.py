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


def test_static_assembly_matches_context_path_twice():
    import torch
    from bem3_aw_qd2_b200 import api, meshgen
    h, _ = api.libs()
    h.aqd2_set_verbose(0)
    d = tempfile.mkdtemp(prefix="bem_static_")
    files = meshgen.write_inputs(d, **meshgen.CONFIGS["sphere24"])
    case = api.Case.from_files(*files)
    case.solve()
    datp = os.path.join(d, "case.dat")
    case.dat_write(datp)
    t = parse_dat(datp)
    dev = torch.device("cuda:0")
    cr = torch.tensor(t["cr"], device=dev)
    cw = torch.tensor(t["cw"], device=dev)
    ren = torch.tensor(t["ren"], device=dev)
    plane = torch.tensor(t["plane"], device=dev)
    fn = _entry()
    stream = torch.cuda.Stream(device=dev)
    qp = np.ascontiguousarray(t["qp"])
    for call in range(2):
        for dom in (0, 1):
            sid = torch.tensor(t["sids"][dom], dtype=torch.int32, device=dev)
            ne = len(t["sids"][dom])
            N = 4 * ne
            G = torch.full((N, N), float("nan"), dtype=torch.complex128, device=dev)
            H = torch.full((N, N), float("nan"), dtype=torch.complex128, device=dev)
            dF = torch.full((N, 3), float("nan"), dtype=torch.float64, device=dev)
            dG = torch.zeros((2 * N, N), dtype=torch.complex128, device=dev) if dom else None
            dH = torch.zeros((2 * N, N), dtype=torch.complex128, device=dev) if dom else None
            torch.cuda.synchronize()
            rc = fn(cr.data_ptr(), cw.data_ptr(), ren.data_ptr(), plane.data_ptr(), sid.data_ptr(), ne,
                    qp.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 1 if dom == 0 else 0, float(t["k0"][dom]),
                    G.data_ptr(), H.data_ptr(), dG.data_ptr() if dG is not None else None,
                    dH.data_ptr() if dH is not None else None, dF.data_ptr(), stream.cuda_stream)
            assert rc == 0, "call %d domain %d returned %d" % (call, dom, rc)
            torch.cuda.synchronize()
            assert rel_rows(G.cpu().numpy(), case.matrix(dom, "G", N)) < 1e-10
            assert rel_rows(H.cpu().numpy(), case.matrix(dom, "H", N)) < 1e-10
            assert np.max(np.abs(dF.cpu().numpy() - case.matrix(dom, "dF", N))) < 1e-10
            if dom:
                assert rel_rows(dG.cpu().numpy(), case.matrix(dom, "dG", N)) < 1e-10
                assert rel_rows(dH.cpu().numpy(), case.matrix(dom, "dH", N)) < 1e-10


def test_static_assembly_rejects_oversized_domain():
    fn = _entry()
    qp = np.zeros(8)
    rc = fn(None, None, None, None, None, 1537, qp.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 1, 1.0,
            None, None, None, None, None, None)
    assert rc == -2
