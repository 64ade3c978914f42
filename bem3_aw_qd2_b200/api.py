"""Python mirror of the reference's bem3_aw_qd2.h API over the native library.

    case = Case.from_files(pw, periodicity, medium, mesh)   # read_aqd2 + initialize_aqd2
    case.solve()                                             # solve_bieq_aqd2 (on the GPU)
    F, N = case.force(type=0)                                # force_FN_aqd2
    case.dat_write("out.dat")                                # dat_write_aqd2

Everything below the ctypes calls runs in lib/libbem3_aw_qd2.so (C host
code) and lib/libbemgpu.so (CUDA kernels + C ABI, include/bemgpu.h).  There
is no Python or CPU implementation of the compute: if the native library is
missing, importing this module fails.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBDIR = os.path.join(HERE, "lib")
_host = None
_gpu = None

_d = ctypes.POINTER(ctypes.c_double)
_i = ctypes.POINTER(ctypes.c_int)


def libs():
    """Load lib/libbemgpu.so and lib/libbem3_aw_qd2.so (raises if absent)."""
    global _host, _gpu
    if _host is None:
        gpath = os.path.join(LIBDIR, "libbemgpu.so")
        hpath = os.path.join(LIBDIR, "libbem3_aw_qd2.so")
        if not (os.path.exists(gpath) and os.path.exists(hpath)):
            raise RuntimeError("native library not built: run bem3_aw_qd2_b200/build.py (%s)" % LIBDIR)
        g = ctypes.CDLL(gpath)
        h = ctypes.CDLL(hpath)
        vp = ctypes.c_void_p
        g.bemgpu_create.argtypes = [ctypes.c_int, vp, ctypes.POINTER(vp)]
        g.bemgpu_destroy.argtypes = [vp]
        g.bemgpu_error.argtypes = [vp]
        g.bemgpu_error.restype = ctypes.c_char_p
        g.bemgpu_status.argtypes = [vp]
        g.bemgpu_status.restype = ctypes.c_uint
        for name in ("bemgpu_assemble", "bemgpu_solve", "bemgpu_run", "bemgpu_sync"):
            getattr(g, name).argtypes = [vp]
        g.bemgpu_get_solution.argtypes = [vp, ctypes.c_int, _d, _d, _d, _d]
        g.bemgpu_get_matrix.argtypes = [vp, ctypes.c_int, ctypes.c_int, _d]
        g.bemgpu_force.argtypes = [vp, ctypes.c_int, _d, _d, _d]
        g.bemgpu_faddeeva_w.argtypes = [_d, ctypes.c_int, _d]
        g.bemgpu_qpgf.argtypes = [_d, _d, ctypes.c_int, _d, _d, _i]
        g.bemgpu_stream.argtypes = [vp]
        g.bemgpu_stream.restype = vp
        g.bemgpu_set_profiling.argtypes = [vp, ctypes.c_int]
        g.bemgpu_phase_times.argtypes = [vp, _d, ctypes.c_int]
        g.bemgpu_work_counters.argtypes = [vp, ctypes.POINTER(ctypes.c_ulonglong), ctypes.c_int]
        g.bemgpu_set_precision.argtypes = [vp, ctypes.c_int]
        g.bemgpu_get_precision.argtypes = [vp]
        g.bemgpu_set_ewald_scale.argtypes = [vp, ctypes.c_double]
        g.bemgpu_set_far_rule.argtypes = [vp, ctypes.c_int]
        g.bemgpu_rule_pairs.argtypes = [vp, ctypes.POINTER(ctypes.c_ulonglong)]
        g.bemgpu_autotune.argtypes = [vp, _d]
        g.bemgpu_solve_stats.argtypes = [vp, _i, _d, _i, ctypes.c_int]
        g.bemgpu_set_interior_reuse.argtypes = [vp, ctypes.c_int]
        g.bemgpu_set_interior_derivatives.argtypes = [vp, ctypes.c_int, ctypes.c_int]
        g.bemgpu_interior_reuses.argtypes = [vp]
        g.bemgpu_interior_reuses.restype = ctypes.c_longlong
        g.bemgpu_kernel_launches.argtypes = []
        g.bemgpu_kernel_launches.restype = ctypes.c_ulonglong
        h.read_aqd2.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_char_p), vp]
        for name in ("print_aqd2", "initialize_aqd2", "finalize_aqd2", "solve_bieq_aqd2"):
            getattr(h, name).argtypes = [vp]
        h.dat_write_aqd2.argtypes = [ctypes.c_char_p, vp]
        h.dat_read_aqd2.argtypes = [ctypes.c_char_p, vp]
        h.force_FN_aqd2.argtypes = [_d, _d, _d, ctypes.c_int, vp]
        h.aqd2_device_context.argtypes = [vp]
        h.aqd2_device_context.restype = vp
        h.aqd2_last_timing.argtypes = [_d]
        h.aqd2_set_device.argtypes = [ctypes.c_int]
        h.aqd2_set_interior_derivatives.argtypes = [ctypes.c_int]
        h.aqd2_set_verbose.argtypes = [ctypes.c_int]
        h.aqd2_problem_build.argtypes = [vp, ctypes.POINTER(Problem)]
        h.aqd2_problem_free.argtypes = [ctypes.POINTER(Problem)]
        g.bemgpu_server_create.argtypes = [ctypes.c_int, ctypes.c_size_t, ctypes.c_int, ctypes.POINTER(vp)]
        g.bemgpu_server_submit.argtypes = [vp, ctypes.POINTER(Problem), ctypes.c_ulonglong, ctypes.c_int, ctypes.c_int,
                                           _d, ctypes.c_longlong]
        g.bemgpu_server_poll.argtypes = [vp, ctypes.POINTER(Result), ctypes.c_int, ctypes.c_int]
        g.bemgpu_server_stats.argtypes = [vp, _d]
        g.bemgpu_server_destroy.argtypes = [vp]
        _host, _gpu = h, g
    return _host, _gpu


class Problem(ctypes.Structure):
    """bemgpu_problem (include/bemgpu.h)."""
    _fields_ = [("Ne", ctypes.c_int), ("NN", ctypes.c_int), ("MN", ctypes.c_int), ("ps", ctypes.c_int),
                ("qp", ctypes.c_double * 8)] + \
               [(n, ctypes.c_void_p) for n in ("cr", "cw", "ren", "wen", "npe", "eni", "md", "sd", "dom_ne", "sid",
                                              "k0", "k2", "rho0", "c0", "Pi", "dPi", "p_inc", "v_inc", "xl", "wl",
                                              "xh", "wh", "plane")] + \
               [("pw", ctypes.c_double * 16)]


class Result(ctypes.Structure):
    """bemgpu_result (include/bemgpu.h)."""
    _fields_ = [("id", ctypes.c_longlong), ("status", ctypes.c_int), ("reused", ctypes.c_int),
                ("precision", ctypes.c_int), ("F", ctypes.c_double * 3), ("N", ctypes.c_double * 3), ("queue_ms", ctypes.c_double),
                ("service_ms", ctypes.c_double), ("error", ctypes.c_char * 160)]


def _p(a):
    return a.ctypes.data_as(_d)


AQD2_SIZE = 2720  # sizeof(AQD2) on x86-64, fixed by the .dat format


class Case:
    """One AQD2 object (the reference's solver state) and its device context."""

    def __init__(self):
        libs()
        self.buf = ctypes.create_string_buffer(AQD2_SIZE)
        self.qd = ctypes.cast(self.buf, ctypes.c_void_p)
        self._alive = False

    @classmethod
    def from_files(cls, pw, per, med, msh, rotation=None):
        """read_aqd2 + initialize_aqd2; rotation = (rvx, rvy, rvz, theta, tx, ty, tz) or None."""
        h, _ = libs()
        c = cls()
        args = ["bem3_aw_qd2", pw, per, med, msh, "unused.dat"]
        if rotation is not None:
            args += ["%.17g" % v for v in rotation]
        argv = (ctypes.c_char_p * len(args))(*[a.encode() for a in args])
        h.read_aqd2(len(args), argv, c.qd)
        h.initialize_aqd2(c.qd)
        c._alive = True
        return c

    @classmethod
    def from_dat(cls, path):
        h, _ = libs()
        c = cls()
        h.dat_read_aqd2(path.encode(), c.qd)
        c._alive = True
        return c

    def solve(self):
        """solve_bieq_aqd2: upload, assemble, solve, download (host buffers in and out)."""
        libs()[0].solve_bieq_aqd2(self.qd)

    def timing(self):
        t = np.zeros(4)
        libs()[0].aqd2_last_timing(_p(t))
        return t

    def force(self, type=0, rc=(0.0, 0.0, 0.0)):
        F = np.zeros(3)
        N = np.zeros(3)
        rc = np.ascontiguousarray(rc, dtype=np.float64)
        libs()[0].force_FN_aqd2(_p(F), _p(N), _p(rc), type, self.qd)
        return F, N

    def field(self, fn, rt, type=1):
        """Field function fn of the reference API ("phi_s", "phi_t", "p_s", "p_t", "pv_s",
        "pv_t", ...) at point rt.  Returns (domain id, phi or p, pv or None)."""
        h = libs()[0]
        rt = np.ascontiguousarray(rt, dtype=np.float64)
        a = np.zeros(2)
        v = np.zeros(6)
        f = getattr(h, fn + "_aqd2")
        f.restype = ctypes.c_int
        if fn.startswith("pv"):
            f.argtypes = [_d, _d, _d, ctypes.c_int, ctypes.c_void_p]
            did = f(_p(a), _p(v), _p(rt), type, self.qd)
            return did, complex(a[0], a[1]), v.view(np.complex128).copy()
        f.argtypes = [_d, _d, ctypes.c_int, ctypes.c_void_p]
        did = f(_p(a), _p(rt), type, self.qd)
        return did, complex(a[0], a[1]), None

    def boundary(self, fn, did, t, zeta, eta, type=1):
        """Boundary function fn ("phi_s_bd", "pv_t_bd", ...) at (zeta, eta) of element t
        (1-based) of domain did.  Returns (phi or p, pv or None)."""
        h = libs()[0]
        a = np.zeros(2)
        v = np.zeros(6)
        f = getattr(h, fn + "_aqd2")
        f.restype = None
        ints = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_void_p]
        if fn.startswith("pv"):
            f.argtypes = [_d, _d] + ints
            f(_p(a), _p(v), did, t, zeta, eta, type, self.qd)
            return complex(a[0], a[1]), v.view(np.complex128).copy()
        f.argtypes = [_d] + ints
        f(_p(a), did, t, zeta, eta, type, self.qd)
        return complex(a[0], a[1]), None

    def problem(self):
        """The initialised problem as a bemgpu_problem with library-owned host arrays
        (aqd2_problem_build); release with free_problem."""
        pr = Problem()
        libs()[0].aqd2_problem_build(self.qd, ctypes.byref(pr))
        return pr

    @staticmethod
    def free_problem(pr):
        libs()[0].aqd2_problem_free(ctypes.byref(pr))

    def dat_write(self, path):
        libs()[0].dat_write_aqd2(path.encode(), self.qd)

    # ---- device context access (tests, benchmarks)
    @property
    def ctx(self):
        c = libs()[0].aqd2_device_context(self.qd)
        if not c:
            raise RuntimeError("no device context: call solve() first")
        return c

    def _check(self, rc, what):
        if rc != 0:
            raise RuntimeError("%s failed (%d): %s" % (what, rc, libs()[1].bemgpu_error(self.ctx).decode()))

    def run_device(self):
        """bemgpu_run on the resident problem (inputs already on the device)."""
        self._check(libs()[1].bemgpu_run(self.ctx), "bemgpu_run")

    def set_precision(self, mode):
        """0 FP64 LU; 1 FP32, 2 TF32, 3 TF32x3 (three split TF32 products), 4 as 2 with FP64 refinement."""
        self._check(libs()[1].bemgpu_set_precision(self.ctx, int(mode)), "set_precision")

    def autotune(self):
        """Pick the Ewald parameter for the loaded problem (bemgpu_autotune); returns the scale."""
        out = np.zeros(1)
        self._check(libs()[1].bemgpu_autotune(self.ctx, _p(out)), "autotune")
        return float(out[0])

    def set_ewald_scale(self, scale):
        self._check(libs()[1].bemgpu_set_ewald_scale(self.ctx, float(scale)), "set_ewald_scale")

    def set_far_rule(self, on):
        """1 (default): shorter rules (10 down to 6 points a side) for regular pairs of
        the periodic domain far enough from every lattice image; 0: 12 x 12 everywhere."""
        self._check(libs()[1].bemgpu_set_far_rule(self.ctx, int(bool(on))), "set_far_rule")

    def rule_pairs(self):
        """Regular pairs of the periodic domain in the last assembly: on the
        reference's 12 x 12 rule, then on the 10, 9, 8, 7 and 6-point rules
        (None when the assembly kept no pair lists)."""
        out = (ctypes.c_ulonglong * 6)()
        if libs()[1].bemgpu_rule_pairs(self.ctx, out) != 0:
            return None
        return list(out)

    def precision(self):
        """The precision mode in effect (see bemgpu.h)."""
        return libs()[1].bemgpu_get_precision(self.ctx)

    def solve_stats(self):
        """(iterations, final relative correction, fell back to FP64) per dense system of the last solve."""
        it = np.zeros(16, np.int32)
        rc = np.zeros(16)
        fb = np.zeros(16, np.int32)
        k = libs()[1].bemgpu_solve_stats(self.ctx, it.ctypes.data_as(_i), _p(rc), fb.ctypes.data_as(_i), 16)
        return it[:k], rc[:k], fb[:k]

    def sync(self):
        self._check(libs()[1].bemgpu_sync(self.ctx), "bemgpu_sync")

    def status(self):
        return libs()[1].bemgpu_status(self.ctx)

    def matrix(self, d, which, N):
        """which: 'G', 'H', 'dG', 'dH', 'dF'; N = 4 * elements of domain d."""
        w = {"G": 0, "H": 1, "dG": 2, "dH": 3, "dF": 4}[which]
        if w == 4:
            out = np.zeros((N, 3))
        elif w >= 2:
            out = np.zeros((2 * N, N), np.complex128)
        else:
            out = np.zeros((N, N), np.complex128)
        self._check(libs()[1].bemgpu_get_matrix(self.ctx, d, w, _p(out.view(np.float64) if out.dtype == np.complex128 else out)),
                    "get_matrix")
        return out

    def solution(self, d, ne):
        P = np.zeros((ne, 4), np.complex128)
        dP = np.zeros((ne, 4), np.complex128)
        pv = np.zeros((ne, 4, 3), np.complex128)
        dpv = np.zeros((ne, 4, 3), np.complex128)
        self._check(libs()[1].bemgpu_get_solution(self.ctx, d, _p(P.view(np.float64)), _p(dP.view(np.float64)),
                                                  _p(pv.view(np.float64)), _p(dpv.view(np.float64))), "get_solution")
        return P, dP, pv, dpv

    def close(self):
        if self._alive:
            libs()[0].finalize_aqd2(self.qd)
            self._alive = False

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def faddeeva_w(z):
    """Device Faddeeva function at the complex points z (numpy array)."""
    z = np.ascontiguousarray(np.asarray(z, dtype=np.complex128))
    w = np.zeros_like(z)
    rc = libs()[1].bemgpu_faddeeva_w(_p(z.view(np.float64)), z.size, _p(w.view(np.float64)))
    if rc != 0:
        raise RuntimeError("bemgpu_faddeeva_w failed")
    return w


def qpgf(qp, r):
    """Device quasi-periodic Green's function and gradient at points r[n,3]."""
    qp = np.ascontiguousarray(qp, dtype=np.float64)
    r = np.ascontiguousarray(r, dtype=np.float64).reshape(-1, 3)
    n = len(r)
    G = np.zeros(n, np.complex128)
    dG = np.zeros((n, 3), np.complex128)
    ret = np.zeros(n, np.int32)
    rc = libs()[1].bemgpu_qpgf(_p(qp), _p(r), n, _p(G.view(np.float64)), _p(dG.view(np.float64)),
                               ret.ctypes.data_as(_i))
    if rc != 0:
        raise RuntimeError("bemgpu_qpgf failed")
    return G, dG, ret


class Server:
    """The request server of the C ABI (bemgpu_server_*): continuous batching,
    factorisation reuse by key, admission by a device-memory budget."""

    def __init__(self, device=0, hbm_budget=64 << 30, slots=4):
        _, g = libs()
        self.g = g
        self.h = ctypes.c_void_p()
        if g.bemgpu_server_create(device, hbm_budget, slots, ctypes.byref(self.h)) != 0:
            raise RuntimeError("bemgpu_server_create failed")

    def submit(self, problem, key, rid, precision=0, force_type=0, rc=(0.0, 0.0, 0.0)):
        rc = np.ascontiguousarray(rc, dtype=np.float64)
        r = self.g.bemgpu_server_submit(self.h, ctypes.byref(problem), key & 0xFFFFFFFFFFFFFFFF, precision, force_type,
                                        _p(rc), rid)
        if r != 0:
            raise RuntimeError("request %d not admissible (%d)" % (rid, r))

    def poll(self, max_results=64, timeout_ms=100):
        buf = (Result * max_results)()
        k = self.g.bemgpu_server_poll(self.h, buf, max_results, timeout_ms)
        return [buf[i] for i in range(k)]

    def stats(self):
        out = np.zeros(8)
        self.g.bemgpu_server_stats(self.h, _p(out))
        keys = ["submitted", "completed", "reused", "running", "queued", "bytes_resident", "bytes_peak", "evictions"]
        return dict(zip(keys, out.tolist()))

    def close(self):
        if self.h:
            self.g.bemgpu_server_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
