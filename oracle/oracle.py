"""ctypes access to the CHECKERS: the C restatement and the reference built from source.

TEST INFRASTRUCTURE ONLY.  Imported by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline / reference arm -- never by the engine package.

    Oracle()      -> oracle/_build/liboracle.so      (restatement, oracle.c)
    Reference()   -> oracle/_ref/libhsps_ref.so      (the reference's own code, pinning build)
    Reference(fast=True) -> oracle/_ref/libhsps_ref_fast.so (release flags, timed baseline)
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "hybrid-sparse-pde-solver_b200"))
from hsps_b200._abi import Escalation, Params, Stats, default_params  # noqa: E402

ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libhsps_ref.so")
REF_FAST_SO = os.path.join(HERE, "_ref", "libhsps_ref_fast.so")

_i32 = np.int32
_f64 = np.float64


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


class _Csr:
    def __init__(self, rp, ci, v):
        self.rp, self.ci, self.v = _c(rp, _i32), _c(ci, _i32), _c(v, _f64)
        self.n = len(self.rp) - 1

    def args(self):
        return (self.n, _p(self.rp), _p(self.ci), _p(self.v))


def build_if_needed():
    if not os.path.exists(ORACLE_SO):
        import subprocess

        subprocess.run(["make", "-C", HERE, "oracle"], check=True, capture_output=True)


class Oracle:
    """The C restatement of the reference path (oracle.c)."""

    def __init__(self):
        build_if_needed()
        L = C.CDLL(ORACLE_SO)
        V, I32, D = C.c_void_p, C.c_int32, C.c_double
        L.orc_poisson_2d.restype = C.c_int64
        L.orc_poisson_2d.argtypes = [I32, V, V, V]
        L.orc_convdiff_2d.restype = C.c_int64
        L.orc_convdiff_2d.argtypes = [I32, D, D, D, V, V, V]
        L.orc_spmv.argtypes = [I32, V, V, V, V, V]
        L.orc_dot.restype = D
        L.orc_dot.argtypes = [I32, V, V]
        L.orc_jacobi_setup.argtypes = [I32, V, V, V, D, V]
        L.orc_ilu0_factor.argtypes = [I32, V, V, V, V]
        L.orc_ilut_factor.argtypes = [I32, V, V, V, D, I32, V, V, V, C.POINTER(C.c_int64)]
        L.orc_ilu_apply.argtypes = [I32, V, V, V, V, V]
        L.orc_levels.restype = I32
        L.orc_levels.argtypes = [I32, V, V, C.c_int, V]
        L.orc_amg_aggregate.restype = I32
        L.orc_amg_aggregate.argtypes = [I32, V, V, V, D, V]
        L.orc_amg_setup.restype = V
        L.orc_amg_setup.argtypes = [I32, V, V, V, C.POINTER(Params)]
        L.orc_amg_free.argtypes = [V]
        L.orc_amg_num_levels.restype = I32
        L.orc_amg_num_levels.argtypes = [V]
        pi = C.POINTER(C.c_int32)
        L.orc_amg_level.argtypes = [V, I32, I32, pi, pi, pi, V, V, V]
        L.orc_amg_apply.argtypes = [V, V, V]
        L.orc_prec_setup.restype = V
        L.orc_prec_setup.argtypes = [C.c_int, I32, V, V, V, C.POINTER(Params), C.POINTER(C.c_int)]
        L.orc_prec_free.argtypes = [V]
        L.orc_prec_apply.argtypes = [V, V, V]
        for f in (L.orc_cg, L.orc_fgmres, L.orc_pipelined_fgmres, L.orc_sstep_cg):
            f.argtypes = [I32, V, V, V, V, V, V, C.POINTER(Params), C.POINTER(Stats)]
        L.orc_spectral_interval.argtypes = [I32, V, V, V, C.c_int, C.POINTER(D), C.POINTER(D)]
        L.orc_extract_features.argtypes = [I32, V, V, V, V, pi]
        L.orc_solve_adaptive.argtypes = [I32, V, V, V, V, V, C.POINTER(Params), C.POINTER(Stats),
                                         C.POINTER(Escalation), I32, pi, pi]
        self.L = L

    # generators
    def poisson_2d(self, n):
        N = n * n
        rp, ci, v = np.zeros(N + 1, _i32), np.zeros(5 * N, _i32), np.zeros(5 * N, _f64)
        k = self.L.orc_poisson_2d(n, _p(rp), _p(ci), _p(v))
        return rp, ci[:k].copy(), v[:k].copy()

    def convdiff_2d(self, n, eps, bx, by):
        N = n * n
        rp, ci, v = np.zeros(N + 1, _i32), np.zeros(5 * N, _i32), np.zeros(5 * N, _f64)
        k = self.L.orc_convdiff_2d(n, eps, bx, by, _p(rp), _p(ci), _p(v))
        return rp, ci[:k].copy(), v[:k].copy()

    def spmv(self, rp, ci, v, x):
        A = _Csr(rp, ci, v)
        x = _c(x, _f64)
        y = np.empty(A.n, _f64)
        self.L.orc_spmv(*A.args(), _p(x), _p(y))
        return y

    def dot(self, a, b):
        a, b = _c(a, _f64), _c(b, _f64)
        return self.L.orc_dot(len(a), _p(a), _p(b))

    def jacobi(self, rp, ci, v, omega=1.0):
        A = _Csr(rp, ci, v)
        d = np.empty(A.n, _f64)
        rc = self.L.orc_jacobi_setup(*A.args(), omega, _p(d))
        return rc, d

    def ilu0(self, rp, ci, v):
        A = _Csr(rp, ci, v)
        lu = np.empty(len(A.v), _f64)
        rc = self.L.orc_ilu0_factor(*A.args(), _p(lu))
        return rc, lu

    def ilut(self, rp, ci, v, drop_tol, fill_p=0):
        """setup_ilut restated: the L\\U factor (rp, ci, values)."""
        A = _Csr(rp, ci, v)
        nnz = C.c_int64()
        self.L.orc_ilut_factor(*A.args(), drop_tol, fill_p, None, None, None, C.byref(nnz))
        frp = np.empty(A.n + 1, _i32)
        fci = np.empty(max(nnz.value, 1), _i32)
        flu = np.empty(max(nnz.value, 1), _f64)
        self.L.orc_ilut_factor(*A.args(), drop_tol, fill_p, _p(frp), _p(fci), _p(flu), C.byref(nnz))
        return frp, fci[:nnz.value], flu[:nnz.value]

    def ilu_apply(self, rp, ci, lu, r):
        A = _Csr(rp, ci, lu)
        r = _c(r, _f64)
        z = np.empty(A.n, _f64)
        rc = self.L.orc_ilu_apply(*A.args(), _p(r), _p(z))
        return rc, z

    def levels(self, rp, ci, which):
        rp, ci = _c(rp, _i32), _c(ci, _i32)
        lev = np.empty(len(rp) - 1, _i32)
        n = self.L.orc_levels(len(rp) - 1, _p(rp), _p(ci), which, _p(lev))
        return n, lev

    def aggregate(self, rp, ci, v, theta=0.25):
        A = _Csr(rp, ci, v)
        agg = np.empty(A.n, _i32)
        m = self.L.orc_amg_aggregate(*A.args(), theta, _p(agg))
        return m, agg

    def amg_hierarchy(self, rp, ci, v, params=None):
        """List of levels, each a dict with A (and P, R except at the coarsest)."""
        A = _Csr(rp, ci, v)
        p = params or default_params()
        h = self.L.orc_amg_setup(*A.args(), C.byref(p))
        try:
            return _read_levels(self.L.orc_amg_num_levels(h), lambda *a: self.L.orc_amg_level(h, *a))
        finally:
            self.L.orc_amg_free(h)

    def amg_apply(self, rp, ci, v, r, params=None):
        A = _Csr(rp, ci, v)
        p = params or default_params()
        h = self.L.orc_amg_setup(*A.args(), C.byref(p))
        try:
            r = _c(r, _f64)
            z = np.empty(A.n, _f64)
            self.L.orc_amg_apply(h, _p(r), _p(z))
            return z
        finally:
            self.L.orc_amg_free(h)

    def precond_apply(self, kind, rp, ci, v, r, params=None):
        A = _Csr(rp, ci, v)
        p = params or default_params()
        st = C.c_int(0)
        M = self.L.orc_prec_setup(kind, *A.args(), C.byref(p), C.byref(st))
        if st.value != 0:
            return st.value, None
        r = _c(r, _f64)
        z = np.empty(A.n, _f64)
        try:
            if M:
                rc = self.L.orc_prec_apply(M, _p(r), _p(z))
            else:
                z[:] = r
                rc = 0
        finally:
            self.L.orc_prec_free(M)
        return rc, z

    def solve(self, solver, precond, rp, ci, v, b, x0=None, params=None):
        """Factory make(solver, precond) + solve; returns (rc, x, Stats)."""
        A = _Csr(rp, ci, v)
        p = params or default_params()
        st = C.c_int(0)
        M = self.L.orc_prec_setup(precond, *A.args(), C.byref(p), C.byref(st))
        if st.value != 0:
            return st.value, None, None
        b = _c(b, _f64)
        x = np.zeros(A.n, _f64) if x0 is None else _c(x0, _f64).copy()
        s = Stats()
        # 0 CGSolver, 1 FGMRESSolver, 3 SStepCGSolver, 5 PipelinedFGMRESSolver
        f = {0: self.L.orc_cg, 1: self.L.orc_fgmres, 2: self.L.orc_fgmres, 3: self.L.orc_sstep_cg,
             5: self.L.orc_pipelined_fgmres}[solver]
        try:
            rc = f(*A.args(), M, _p(b), _p(x), C.byref(p), C.byref(s))
        finally:
            self.L.orc_prec_free(M)
        return rc, x, s

    def spectral_interval(self, rp, ci, v, steps=20):
        A = _Csr(rp, ci, v)
        lo, hi = C.c_double(), C.c_double()
        self.L.orc_spectral_interval(*A.args(), steps, C.byref(lo), C.byref(hi))
        return lo.value, hi.value

    def features(self, rp, ci, v):
        A = _Csr(rp, ci, v)
        f = np.empty(24, _f64)
        s = C.c_int32(0)
        self.L.orc_extract_features(*A.args(), _p(f), C.byref(s))
        return f, s.value

    def solve_adaptive(self, rp, ci, v, b, x0=None, params=None, log_cap=8):
        A = _Csr(rp, ci, v)
        p = params or default_params()
        b = _c(b, _f64)
        x = np.zeros(A.n, _f64) if x0 is None else _c(x0, _f64).copy()
        s = Stats()
        log = (Escalation * log_cap)()
        nlog, init = C.c_int32(0), C.c_int32(0)
        rc = self.L.orc_solve_adaptive(*A.args(), _p(b), _p(x), C.byref(p), C.byref(s), log,
                                       log_cap, C.byref(nlog), C.byref(init))
        return rc, x, s, [log[i] for i in range(min(nlog.value, log_cap))], init.value


def _read_levels(nlev, level_fn):
    out = []
    for l in range(nlev):
        d = {}
        for which, name in ((0, "A"), (1, "P"), (2, "R")):
            rows, cols, nnz = C.c_int32(), C.c_int32(), C.c_int32()
            if level_fn(l, which, C.byref(rows), C.byref(cols), C.byref(nnz), None, None, None) != 0:
                continue
            rp = np.empty(rows.value + 1, _i32)
            ci = np.empty(nnz.value, _i32)
            v = np.empty(nnz.value, _f64)
            level_fn(l, which, None, None, None, _p(rp), _p(ci), _p(v))
            if name != "A" and rows.value == 0:
                continue
            d[name] = (rows.value, cols.value, rp, ci, v)
        out.append(d)
    return out


def reference_available(fast=False) -> bool:
    return os.path.exists(REF_FAST_SO if fast else REF_SO)


class Reference:
    """The reference's own implementation, built from its sources (oracle/Makefile)."""

    def __init__(self, fast=False, threads=None):
        path = REF_FAST_SO if fast else REF_SO
        if not os.path.exists(path):
            raise RuntimeError(f"{path} not built (make -C oracle ref)")
        L = C.CDLL(path)
        V, I32, D = C.c_void_p, C.c_int32, C.c_double
        pi = C.POINTER(C.c_int32)
        L.ref_set_threads.argtypes = [C.c_int]
        L.ref_max_threads.restype = C.c_int
        L.ref_gen_poisson.restype = C.c_int64
        L.ref_gen_poisson.argtypes = [I32, V, V, V]
        L.ref_gen_convdiff.restype = C.c_int64
        L.ref_gen_convdiff.argtypes = [I32, D, D, D, V, V, V]
        L.ref_from_coo.restype = C.c_int64
        L.ref_from_coo.argtypes = [I32, I32, C.c_int64, V, V, V, V, V, V]
        L.ref_spmv.argtypes = [I32, V, V, V, V, V]
        L.ref_dot.restype = D
        L.ref_dot.argtypes = [I32, V, V]
        L.ref_pipelined_solve.argtypes = [C.c_int, I32, V, V, V, V, V, C.POINTER(Params),
                                          C.POINTER(Stats)]
        L.ref_spectral_interval.argtypes = [I32, V, V, V, C.c_int, C.POINTER(D), C.POINTER(D)]
        L.ref_solve.argtypes = [C.c_int, C.c_int, I32, V, V, V, V, V, C.POINTER(Params),
                                C.POINTER(Stats)]
        L.ref_precond_apply.argtypes = [C.c_int, I32, V, V, V, C.POINTER(Params), V, V]
        L.ref_amg_aggregate.restype = I32
        L.ref_amg_aggregate.argtypes = [I32, V, V, V, D, V]
        L.ref_amg_setup.restype = V
        L.ref_amg_setup.argtypes = [I32, V, V, V, C.POINTER(Params)]
        L.ref_amg_free.argtypes = [V]
        L.ref_amg_num_levels.restype = I32
        L.ref_amg_num_levels.argtypes = [V]
        L.ref_amg_level.argtypes = [V, I32, I32, pi, pi, pi, V, V, V]
        L.ref_amg_apply.argtypes = [V, I32, V, V]
        L.ref_ilu0_factor.argtypes = [I32, V, V, V, V]
        L.ref_extract_features.argtypes = [I32, V, V, V, V, pi]
        L.ref_solve_adaptive.argtypes = [I32, V, V, V, V, V, C.POINTER(Params), C.POINTER(Stats),
                                         C.POINTER(Escalation), I32, pi]
        L.ref_mtx_load_matrix.argtypes = [C.c_char_p, pi, pi, pi, V, V, V]
        L.ref_ilut_factor.argtypes = [I32, V, V, V, D, I32, V, V, V, C.POINTER(C.c_int64)]
        L.ref_mtx_load_vector.argtypes = [C.c_char_p, I32, V, pi]
        self.L = L
        self.set_threads(1 if threads is None else threads)

    def set_threads(self, t):
        self.L.ref_set_threads(int(t))
        self.threads = int(t)

    def poisson_2d(self, n):
        N = n * n
        rp, ci, v = np.zeros(N + 1, _i32), np.zeros(5 * N, _i32), np.zeros(5 * N, _f64)
        k = self.L.ref_gen_poisson(n, _p(rp), _p(ci), _p(v))
        return rp, ci[:k].copy(), v[:k].copy()

    def convdiff_2d(self, n, eps, bx, by):
        N = n * n
        rp, ci, v = np.zeros(N + 1, _i32), np.zeros(5 * N, _i32), np.zeros(5 * N, _f64)
        k = self.L.ref_gen_convdiff(n, eps, bx, by, _p(rp), _p(ci), _p(v))
        return rp, ci[:k].copy(), v[:k].copy()

    def from_coo(self, rows, cols, r, c, v):
        r, c, v = _c(r, _i32), _c(c, _i32), _c(v, _f64)
        rp = np.zeros(rows + 1, _i32)
        ci = np.zeros(len(r), _i32)
        vo = np.zeros(len(r), _f64)
        k = self.L.ref_from_coo(rows, cols, len(r), _p(r), _p(c), _p(v), _p(rp), _p(ci), _p(vo))
        return rp, ci[:k].copy(), vo[:k].copy()

    def spmv(self, rp, ci, v, x):
        A = _Csr(rp, ci, v)
        x = _c(x, _f64)
        y = np.empty(A.n, _f64)
        self.L.ref_spmv(*A.args(), _p(x), _p(y))
        return y

    def dot(self, a, b):
        a, b = _c(a, _f64), _c(b, _f64)
        return self.L.ref_dot(len(a), _p(a), _p(b))

    def solve(self, solver, precond, rp, ci, v, b, x0=None, params=None):
        A = _Csr(rp, ci, v)
        p = params or default_params()
        b = _c(b, _f64)
        x = np.zeros(A.n, _f64) if x0 is None else _c(x0, _f64).copy()
        s = Stats()
        if solver == 5:        # PipelinedFGMRESSolver, built directly (no SolverType)
            rc = self.L.ref_pipelined_solve(precond, *A.args(), _p(b), _p(x), C.byref(p), C.byref(s))
        else:
            rc = self.L.ref_solve(solver, precond, *A.args(), _p(b), _p(x), C.byref(p), C.byref(s))
        return rc, x, s

    def spectral_interval(self, rp, ci, v, steps=20):
        A = _Csr(rp, ci, v)
        lo, hi = C.c_double(), C.c_double()
        self.L.ref_spectral_interval(*A.args(), steps, C.byref(lo), C.byref(hi))
        return lo.value, hi.value

    def precond_apply(self, kind, rp, ci, v, r, params=None):
        A = _Csr(rp, ci, v)
        p = params or default_params()
        r = _c(r, _f64)
        z = np.empty(A.n, _f64)
        rc = self.L.ref_precond_apply(kind, *A.args(), C.byref(p), _p(r), _p(z))
        return rc, z

    def aggregate(self, rp, ci, v, theta=0.25):
        A = _Csr(rp, ci, v)
        agg = np.empty(A.n, _i32)
        m = self.L.ref_amg_aggregate(*A.args(), theta, _p(agg))
        return m, agg

    def amg_hierarchy(self, rp, ci, v, params=None):
        A = _Csr(rp, ci, v)
        p = params or default_params()
        h = self.L.ref_amg_setup(*A.args(), C.byref(p))
        if not h:
            raise RuntimeError("reference AMG setup failed")
        try:
            return _read_levels(self.L.ref_amg_num_levels(h), lambda *a: self.L.ref_amg_level(h, *a))
        finally:
            self.L.ref_amg_free(h)

    def amg_apply(self, rp, ci, v, r, params=None):
        A = _Csr(rp, ci, v)
        p = params or default_params()
        h = self.L.ref_amg_setup(*A.args(), C.byref(p))
        try:
            r = _c(r, _f64)
            z = np.empty(A.n, _f64)
            self.L.ref_amg_apply(h, A.n, _p(r), _p(z))
            return z
        finally:
            self.L.ref_amg_free(h)

    def ilu0(self, rp, ci, v):
        A = _Csr(rp, ci, v)
        lu = np.empty(len(A.v), _f64)
        rc = self.L.ref_ilu0_factor(*A.args(), _p(lu))
        return rc, lu

    def features(self, rp, ci, v):
        A = _Csr(rp, ci, v)
        f = np.empty(24, _f64)
        s = C.c_int32(0)
        self.L.ref_extract_features(*A.args(), _p(f), C.byref(s))
        return f, s.value

    def ilut(self, rp, ci, v, drop_tol, fill_p=0):
        """ILUPreconditioner::setup_ilut: the L\\U factor (rp, ci, values)."""
        A = _Csr(rp, ci, v)
        nnz = C.c_int64()
        rc = self.L.ref_ilut_factor(*A.args(), drop_tol, fill_p, None, None, None, C.byref(nnz))
        if rc:
            raise RuntimeError(f"reference ILUT failed ({rc})")
        frp = np.empty(A.n + 1, _i32)
        fci = np.empty(max(nnz.value, 1), _i32)
        flu = np.empty(max(nnz.value, 1), _f64)
        self.L.ref_ilut_factor(*A.args(), drop_tol, fill_p, _p(frp), _p(fci), _p(flu), C.byref(nnz))
        return frp, fci[:nnz.value], flu[:nnz.value]

    def mtx_load_matrix(self, path):
        """MatrixMarketIO::load_matrix: (rows, cols, rp, ci, v), or None on an exception."""
        r, c, nz = C.c_int32(), C.c_int32(), C.c_int32()
        p = os.fsencode(path)
        if self.L.ref_mtx_load_matrix(p, C.byref(r), C.byref(c), C.byref(nz), None, None, None):
            return None
        rp = np.empty(r.value + 1, _i32)
        ci = np.empty(max(nz.value, 1), _i32)
        v = np.empty(max(nz.value, 1), _f64)
        self.L.ref_mtx_load_matrix(p, C.byref(r), C.byref(c), C.byref(nz), _p(rp), _p(ci), _p(v))
        return r.value, c.value, rp, ci[:nz.value], v[:nz.value]

    def mtx_load_vector(self, path, expected_n=0):
        n = C.c_int32()
        p = os.fsencode(path)
        if self.L.ref_mtx_load_vector(p, expected_n, None, C.byref(n)):
            return None
        out = np.empty(max(n.value, 1), _f64)
        self.L.ref_mtx_load_vector(p, expected_n, _p(out), C.byref(n))
        return out[:n.value]

    def solve_adaptive(self, rp, ci, v, b, x0=None, params=None, log_cap=8):
        A = _Csr(rp, ci, v)
        p = params or default_params()
        b = _c(b, _f64)
        x = np.zeros(A.n, _f64) if x0 is None else _c(x0, _f64).copy()
        s = Stats()
        log = (Escalation * log_cap)()
        nlog = C.c_int32(0)
        rc = self.L.ref_solve_adaptive(*A.args(), _p(b), _p(x), C.byref(p), C.byref(s), log,
                                       log_cap, C.byref(nlog))
        return rc, x, s, [log[i] for i in range(min(nlog.value, log_cap))]
