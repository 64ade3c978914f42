"""The device dense complex solve (bem_lu.cu through bemgpu_zgesv: tournament-
pivoting LU on a thread-block cluster, DMMA trailing updates, flag-ordered
triangular solves) against numpy's LAPACK solve.

Sizes cover: a single short panel (n < 32), panels whose rows fit one CTA
(n <= 256), panels spread over the cluster's 8 CTAs, panels whose CTAs run
several tournament rounds (n > 2048), a last panel narrower than 32, one
outer block of 128 columns and the sizes on either side of it (127, 129),
several outer blocks with a partial last one (300, 700, 2500), and the
216-quad benchmark's global size (n = 1728).

The complex FP32 factorisation of the mixed-precision solves is checked the
same way with each trailing-update arithmetic: FP32 CUDA cores, one TF32
product on the tensor cores (tcgen05) and three split TF32 products.

Tolerances (stated here, used below): FP64, the relative residual
||A x - b|| / (||A|| ||x||) below 1e-13, and the solution within 1e-10 of
numpy's relative to its norm (the matrices are well conditioned); complex
FP32, that residual below 2e-6 (FP32 updates and three split TF32 products;
measured 1-3e-8) or 1e-4 (one TF32 product; measured 5e-6)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIZES = [1, 7, 31, 32, 33, 100, 127, 128, 129, 255, 256, 257, 300, 700, 1728, 2500]


def zgesv(A, B):
    from bem3_aw_qd2_b200 import api
    _, g = api.libs()
    g.bemgpu_zgesv.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    A = np.ascontiguousarray(A, dtype=np.complex128)
    X = np.asfortranarray(B, dtype=np.complex128).copy(order="F")
    n, nrhs = X.shape
    rc = g.bemgpu_zgesv(0, n, nrhs, A.ctypes.data, X.ctypes.data)
    return rc, X


def random_system(n, nrhs, seed, permuted=False):
    rng = np.random.default_rng(seed)
    A = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / np.sqrt(n)
    A += np.eye(n) * (1.5 + 0.5j)
    if permuted:
        # a row permutation of a diagonally heavy matrix: every panel must move rows
        A = A[rng.permutation(n)]
    B = rng.standard_normal((n, nrhs)) + 1j * rng.standard_normal((n, nrhs))
    return A, B


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("nrhs", [1, 3])
def test_zgesv_matches_lapack(n, nrhs):
    A, B = random_system(n, nrhs, seed=1000 + n + nrhs)
    rc, X = zgesv(A, B)
    assert rc == 0
    ref = np.linalg.solve(A, B)
    res = np.linalg.norm(A @ X - B) / (np.linalg.norm(A) * np.linalg.norm(X))
    assert res < 1e-13, res
    assert np.linalg.norm(X - ref) / np.linalg.norm(ref) < 1e-10


@pytest.mark.parametrize("n", [40, 300, 1728, 2100])
def test_zgesv_row_moves(n):
    """Rows out of order: the pivots come from far below the panel."""
    A, B = random_system(n, 2, seed=77 + n, permuted=True)
    rc, X = zgesv(A, B)
    assert rc == 0
    ref = np.linalg.solve(A, B)
    assert np.linalg.norm(X - ref) / np.linalg.norm(ref) < 1e-10


def test_zgesv_reports_singular_matrix():
    n = 64
    A, B = random_system(n, 1, seed=5)
    A[:, 10] = 0.0  # a zero column: no pivot for column 10
    rc, _ = zgesv(A, B)
    assert rc == -3


@pytest.mark.parametrize("n", [100, 129, 300, 700, 1728, 2500])
@pytest.mark.parametrize("mode", ["fp32", "tf32", "tf32x3"])
def test_complex_fp32_lu(n, mode):
    """The mixed-precision solves' FP32 LU (bem_lu_factor_c / bem_lu_solve_c),
    its outer-block updates on the CUDA cores or on the tensor cores."""
    import torch
    from bem3_aw_qd2_b200 import api
    _, g = api.libs()
    vp = ctypes.c_void_p
    g.bem_lu_init.argtypes = [vp, ctypes.c_int]
    g.bem_lu_free.argtypes = [vp]
    g.bem_lu_factor_c.argtypes = [vp, vp, ctypes.c_int, vp]
    g.bem_lu_solve_c.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, vp, vp]
    g.bem_lu_status.argtypes = [vp, vp]
    g.bem_lu_status.restype = ctypes.c_uint
    g.bem_lu_attach_tc.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    g.bem_lu_detach_tc.argtypes = [vp]
    A, B = random_system(n, 2, seed=500 + n, permuted=True)
    w = ctypes.create_string_buffer(4096)
    wp = ctypes.addressof(w)
    assert g.bem_lu_init(wp, 0) == 0
    try:
        if mode != "fp32":
            assert g.bem_lu_attach_tc(wp, n, 1 if mode == "tf32" else 3) == 0
        st = torch.cuda.Stream()
        Ad = torch.from_numpy(A.astype(np.complex64)).cuda()
        Bd = torch.from_numpy(np.ascontiguousarray(B.T).astype(np.complex64)).cuda()  # column-major n x 2
        torch.cuda.synchronize()
        assert g.bem_lu_factor_c(wp, Ad.data_ptr(), n, st.cuda_stream) == 0
        assert g.bem_lu_solve_c(wp, Ad.data_ptr(), n, 2, Bd.data_ptr(), st.cuda_stream) == 0
        assert g.bem_lu_status(wp, st.cuda_stream) == 0
        X = Bd.cpu().numpy().T.astype(np.complex128)
    finally:
        g.bem_lu_detach_tc(wp)
        g.bem_lu_free(wp)
    res = np.linalg.norm(A @ X - B) / (np.linalg.norm(A) * np.linalg.norm(X))
    assert res < (1e-4 if mode == "tf32" else 2e-6), res
