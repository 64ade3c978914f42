"""The device dense complex solve (bem_lu.cu through bemgpu_zgesv: tournament-
pivoting LU on a thread-block cluster, DMMA trailing updates, flag-ordered
triangular solves) against numpy's LAPACK solve.

Sizes cover: a single short panel (n < 32), panels whose rows fit one CTA
(n <= 256), panels spread over the cluster's 8 CTAs, panels whose CTAs run
several tournament rounds (n > 2048), a last panel narrower than 32, and the
216-quad benchmark's global size (n = 1728).

Tolerances (stated here, used below): the relative residual
||A x - b|| / (||A|| ||x||) below 1e-13, and the solution within 1e-10 of
numpy's relative to its norm (the matrices are well conditioned)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIZES = [1, 7, 31, 32, 33, 100, 255, 256, 257, 700, 1728, 2500]


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
