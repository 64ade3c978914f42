"""Test infrastructure: ctypes access to the reference build in oracle/_ref.

oracle/_ref/libbem3ref.so is the reference's own C sources compiled unchanged
(recipe: oracle/ref/Makefile) plus oracle/ref/ref_hooks.c, which only exposes
the reference's functions and temporary files.  Used by tests/, by the
fixture generator in tests/golden/ and by the CPU-baseline leg of bench.py;
never by the product path.
"""
import ctypes
import os
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "_ref", "libbem3ref.so")

_lib = None


def available():
    return os.path.exists(LIBPATH)


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(LIBPATH)
        d = ctypes.POINTER(ctypes.c_double)
        i = ctypes.POINTER(ctypes.c_int)
        L.ref_sizeof_aqd2.restype = ctypes.c_size_t
        L.ref_faddeeva_w.argtypes = [d, ctypes.c_int, ctypes.c_double, d]
        L.ref_qpgf.argtypes = [ctypes.c_int, d, d, ctypes.c_int, ctypes.c_double, d, d, i]
        L.ref_load.argtypes = [ctypes.c_void_p] + [ctypes.c_char_p] * 4
        L.ref_solve_keep_files.argtypes = [ctypes.c_void_p]
        L.ref_assemble_domain_files.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ref_assemble_rows.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.ref_assemble_rows.restype = ctypes.c_double
        L.ref_assemble_list.argtypes = [ctypes.c_void_p, ctypes.c_int, i, ctypes.c_int]
        L.ref_assemble_list.restype = ctypes.c_double
        L.ref_pair_coef.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, d]
        L.ref_domain_ne.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ref_get_solution.argtypes = [ctypes.c_void_p, ctypes.c_int, d, d, d, d]
        L.force_FN_aqd2.argtypes = [d, d, d, ctypes.c_int, ctypes.c_void_p]
        L.finalize_aqd2.argtypes = [ctypes.c_void_p]
        L.dat_read_aqd2.argtypes = [ctypes.c_char_p, ctypes.c_void_p]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def faddeeva_w(z, relerr=1e-15):
    z = np.ascontiguousarray(np.asarray(z, dtype=np.complex128))
    out = np.zeros_like(z)
    lib().ref_faddeeva_w(_p(z.view(np.float64)), z.size, relerr, _p(out.view(np.float64)))
    return out


def qpgf(qp, r, mode=0, eps=1e-15):
    """mode 0: d3hm_qpgf_d2_v1, 1: Ewald, 2: spectral, 3: G only, 4: grad only."""
    qp = np.ascontiguousarray(qp, dtype=np.float64)
    r = np.ascontiguousarray(r, dtype=np.float64).reshape(-1, 3)
    n = len(r)
    G = np.zeros(n, np.complex128)
    dG = np.zeros((n, 3), np.complex128)
    ret = np.zeros(n, np.int32)
    lib().ref_qpgf(mode, _p(qp), _p(r), n, eps, _p(G.view(np.float64)), _p(dG.view(np.float64)),
                   ret.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
    return G, dG, ret


class RefCase:
    """The reference solver on one set of input files."""

    def __init__(self, pw, per, med, msh):
        L = lib()
        self.buf = ctypes.create_string_buffer(L.ref_sizeof_aqd2())
        self.qd = ctypes.cast(self.buf, ctypes.c_void_p)
        L.ref_load(self.qd, pw.encode(), per.encode(), med.encode(), msh.encode())
        self.MN = L.ref_mn(self.qd)
        self.dom_ne = [L.ref_domain_ne(self.qd, d) for d in range(self.MN + 1)]

    @classmethod
    def from_dat(cls, path):
        """dat_read_aqd2 (bem3_aw_qd2.c:226) of a solved system, e.g. one the
        reference ships with its results."""
        L = lib()
        c = cls.__new__(cls)
        c.buf = ctypes.create_string_buffer(L.ref_sizeof_aqd2())
        c.qd = ctypes.cast(c.buf, ctypes.c_void_p)
        L.dat_read_aqd2(path.encode(), c.qd)
        c.MN = L.ref_mn(c.qd)
        c.dom_ne = [L.ref_domain_ne(c.qd, d) for d in range(c.MN + 1)]
        return c

    def solve(self, workdir=None):
        """Full solve; returns the coefficient matrices read from the temp files."""
        workdir = workdir or tempfile.mkdtemp(prefix="bemref_")
        cwd = os.getcwd()
        os.chdir(workdir)
        try:
            lib().ref_solve_keep_files(self.qd)
            mats = {}
            for d in range(self.MN + 1):
                N = 4 * self.dom_ne[d]
                mats["G%d" % d] = np.fromfile("tmpG_%05d.dat" % d, np.complex128).reshape(N, N)
                mats["H%d" % d] = np.fromfile("tmpH_%05d.dat" % d, np.complex128).reshape(N, N)
                mats["dG%d" % d] = np.fromfile("tmpdG_%05d.dat" % d, np.complex128).reshape(2 * N, N)
                mats["dH%d" % d] = np.fromfile("tmpdH_%05d.dat" % d, np.complex128).reshape(2 * N, N)
                mats["dF%d" % d] = np.fromfile("tmpdF_%05d.dat" % d, np.float64).reshape(N, 3)
            return mats
        finally:
            os.chdir(cwd)

    def solution(self, d):
        n = self.dom_ne[d]
        P = np.zeros((n, 4), np.complex128)
        dP = np.zeros((n, 4), np.complex128)
        pv = np.zeros((n, 4, 3), np.complex128)
        dpv = np.zeros((n, 4, 3), np.complex128)
        lib().ref_get_solution(self.qd, d, _p(P.view(np.float64)), _p(dP.view(np.float64)), _p(pv.view(np.float64)),
                               _p(dpv.view(np.float64)))
        return P, dP, pv, dpv

    def force(self, type_=0, rc=(0.0, 0.0, 0.0)):
        F = np.zeros(3)
        N = np.zeros(3)
        rc = np.ascontiguousarray(rc, dtype=np.float64)
        lib().force_FN_aqd2(_p(F), _p(N), _p(rc), type_, self.qd)
        return F, N

    def field(self, fn, rt, type_):
        """Reference field function fn ("pv_t", "pv_s", "phi_s", "p_t", ...) at point rt.
        Returns (domain id, p or phi, pv or None)."""
        L = lib()
        rt = np.ascontiguousarray(rt, dtype=np.float64)
        a = np.zeros(2)
        v = np.zeros(6)
        f = getattr(L, fn + "_aqd2")
        f.restype = ctypes.c_int
        if fn.startswith("pv"):
            did = f(_p(a), _p(v), _p(rt), type_, self.qd)
            return did, complex(a[0], a[1]), v.view(np.complex128).copy()
        did = f(_p(a), _p(rt), type_, self.qd)
        return did, complex(a[0], a[1]), None

    def boundary(self, fn, did, t, zeta, eta, type_):
        """Reference boundary function fn ("pv_t_bd", "phi_s_bd", ...) at (zeta, eta) of
        element t (1-based) of domain did.  Returns (p or phi, pv or None)."""
        L = lib()
        a = np.zeros(2)
        v = np.zeros(6)
        f = getattr(L, fn + "_aqd2")
        f.restype = None
        if fn.startswith("pv"):
            f(_p(a), _p(v), did, t, ctypes.c_double(zeta), ctypes.c_double(eta), type_, self.qd)
            return complex(a[0], a[1]), v.view(np.complex128).copy()
        f(_p(a), did, t, ctypes.c_double(zeta), ctypes.c_double(eta), type_, self.qd)
        return complex(a[0], a[1]), None

    def assemble_rows(self, did, t0, t1):
        """Time the reference's own assembly loop on collocation elements [t0, t1) (1-based)."""
        return lib().ref_assemble_rows(self.qd, did, t0, t1)

    def assemble_list(self, did, rows):
        """The reference's assembly loop on the listed collocation elements (1-based)."""
        rows = np.ascontiguousarray(rows, dtype=np.int32)
        return lib().ref_assemble_list(self.qd, did, rows.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), len(rows))

    def pair(self, did, t, tn, s):
        out = np.zeros(54)
        lib().ref_pair_coef(self.qd, did, t, tn, s, _p(out))
        return out.view(np.complex128).reshape(3, 9)
