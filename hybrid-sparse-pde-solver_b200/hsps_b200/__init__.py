"""hsps_b200 -- Python binding of the B200 solve engine, mirroring the reference's API.

The classes keep the names, arguments and error behaviour of the reference's C++17
interface (namespace hsps): SparseMatrix, SolverParams, SolverStats, CGSolver,
FGMRESSolver, JacobiPreconditioner, ILUPreconditioner, AMGPreconditioner, SolverFactory,
AdaptiveSelector.  All arithmetic runs in libhamlss_b200.so through include/hamlss.h;
this module only marshals arguments.  Vectors are numpy float64 arrays (host) or CUDA
tensors exposing data_ptr() (device, e.g. torch tensors already resident in HBM).

Differences forced by Python: `solve(A, b, x, stats)` updates x in place, so x must
already have A.rows() entries (the reference resizes a wrong-sized x to zeros; here a
wrong size raises ValueError).
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _abi
from ._abi import (DEVICE, HOST, PREC_AMG, PREC_ILU, PREC_JACOBI, PREC_NONE, SOLVER_CG,
                   SOLVER_PIPELINED_FGMRES, SOLVER_SSTEP_CG,
                   SOLVER_FGMRES, STATE_EASY, STATE_HARD, STATE_MODERATE, Escalation, Params,
                   Stats, default_params, lib)
from . import problems

SolverParams = default_params          # SolverParams() -> reference defaults
SolverStats = Stats


class HamlssError(RuntimeError):
    """A negative status from the engine (std::runtime_error in the reference)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def _check(rc: int) -> int:
    if rc < 0:
        msg = lib().hamlss_last_error().decode(errors="replace")
        if rc == _abi.ERR_INVALID and "unknown" in msg:
            raise ValueError(msg)              # std::invalid_argument
        raise HamlssError(rc, msg)
    return rc


def _is_device(a) -> bool:
    return hasattr(a, "data_ptr") and getattr(a, "is_cuda", False)


def _ptr(a):
    if _is_device(a):
        return C.c_void_p(a.data_ptr())
    return a.ctypes.data_as(C.c_void_p)


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


class Context:
    """One device + one CUDA stream (hamlss_ctx)."""

    _default: Optional["Context"] = None

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        _check(lib().hamlss_ctx_create(device, C.byref(h)))
        self.h = h
        self.device = device

    @classmethod
    def default(cls) -> "Context":
        if cls._default is None:
            cls._default = Context(0)
        return cls._default

    def synchronize(self):
        _check(lib().hamlss_ctx_synchronize(self.h))

    def stream(self) -> int:
        s = C.c_void_p()
        _check(lib().hamlss_ctx_stream(self.h, C.byref(s)))
        return s.value or 0

    def __del__(self):
        try:
            if getattr(self, "h", None):
                lib().hamlss_ctx_destroy(self.h)
                self.h = None
        except Exception:
            pass


class SparseMatrix:
    """CSR matrix (SparseMatrix, sparse_matrix.hpp:34-170), resident on the device.

    Host copies of row_ptr / col_idx / values are kept for inspection; the device copy
    is made on construction (a deep copy, like the reference's constructor).
    """

    def __init__(self, rows, cols, row_ptr, col_idx, values, ctx: Optional[Context] = None):
        self.ctx = ctx or Context.default()
        self._rows, self._cols = int(rows), int(cols)
        self._rp = np.ascontiguousarray(row_ptr, dtype=np.int32)
        self._ci = np.ascontiguousarray(col_idx, dtype=np.int32)
        self._v = np.ascontiguousarray(values, dtype=np.float64)
        if len(self._rp) != self._rows + 1 or len(self._ci) != len(self._v):
            raise HamlssError(_abi.ERR_MALFORMED, "CSR array lengths do not match")
        h = C.c_void_p()
        _check(lib().hamlss_mat_upload(self.ctx.h, self._rows, self._cols, len(self._v),
                                       _ptr(self._rp), _ptr(self._ci), _ptr(self._v), HOST,
                                       C.byref(h)))
        self.h = h

    # ---- builders (sparse_matrix.hpp:108-121)
    @classmethod
    def from_coo(cls, rows, cols, row_vec, col_vec, val_vec, ctx=None):
        r = np.asarray(row_vec, np.int64)
        c = np.asarray(col_vec, np.int64)
        v = np.asarray(val_vec, np.float64)
        order = np.lexsort((c, r))
        r, c, v = r[order], c[order], v[order]
        if len(r):
            key = r * max(cols, 1) + c
            first = np.ones(len(key), bool)
            first[1:] = key[1:] != key[:-1]
            grp = np.cumsum(first) - 1
            vals = np.zeros(int(grp[-1]) + 1)
            np.add.at(vals, grp, v)          # duplicates accumulate (sparse_matrix.cpp:268-272)
            r, c, v = r[first], c[first], vals
        rp = np.zeros(rows + 1, np.int64)
        np.add.at(rp, r + 1, 1)
        return cls(rows, cols, np.cumsum(rp), c, v, ctx)

    @classmethod
    def poisson_2d(cls, n, ctx=None):
        rp, ci, v = problems.poisson_2d(n)
        return cls(n * n, n * n, rp, ci, v, ctx)

    @classmethod
    def convection_diffusion_2d(cls, n, epsilon=1.0, beta_x=0.0, beta_y=0.0, ctx=None):
        rp, ci, v = problems.convection_diffusion_2d(n, epsilon, beta_x, beta_y)
        return cls(n * n, n * n, rp, ci, v, ctx)

    # ---- accessors
    def rows(self):
        return self._rows

    def cols(self):
        return self._cols

    def nnz(self):
        return len(self._v)

    def row_ptr(self):
        return self._rp

    def col_idx(self):
        return self._ci

    def values(self):
        return self._v

    def set_values(self, values):
        """Replace the values (same pattern); the device copy is updated."""
        self._v = np.ascontiguousarray(values, dtype=np.float64)
        _check(lib().hamlss_mat_update_values(self.h, _ptr(self._v), HOST))

    def spmv(self, x, y=None):
        """y = A x (SparseMatrix::spmv, sparse_matrix.cpp:68-87)."""
        if _is_device(x):
            if y is None:
                raise ValueError("device spmv needs an output tensor")
            _check(lib().hamlss_spmv(self.ctx.h, self.h, _ptr(x), _ptr(y), DEVICE))
            return y
        x = _f64(x)
        if len(x) != self._cols:
            raise HamlssError(_abi.ERR_SIZE, "SpMV: x size != cols")
        out = np.empty(self._rows) if y is None else y
        _check(lib().hamlss_spmv(self.ctx.h, self.h, _ptr(x), _ptr(out), HOST))
        return out

    __matmul__ = spmv

    def __del__(self):
        try:
            if getattr(self, "h", None):
                lib().hamlss_mat_release(self.h)
                self.h = None
        except Exception:
            pass


# ------------------------------------------------------------------ preconditioners
class PreconditionerBase:
    """PreconditionerBase (preconditioner_base.hpp:16-48)."""

    kind = PREC_NONE
    tier = "CHEAP"

    def __init__(self):
        self.h = None
        self._A = None
        self.ready = False

    def _params(self) -> Params:
        return default_params()

    def setup(self, A: SparseMatrix) -> float:
        self.release()
        h = C.c_void_p()
        t = C.c_double()
        p = self._params()
        _check(lib().hamlss_precond_setup(A.ctx.h, A.h, self.kind, C.byref(p), C.byref(h),
                                          C.byref(t)))
        self.h, self._A, self.ready = h, A, True
        return t.value

    def apply(self, r, z=None):
        if not self.ready:
            raise HamlssError(_abi.ERR_NOT_READY, "preconditioner used before setup")
        if _is_device(r):
            _check(lib().hamlss_precond_apply(self._A.ctx.h, self.h, _ptr(r), _ptr(z), DEVICE))
            return z
        r = _f64(r)
        out = np.empty(len(r)) if z is None else z
        _check(lib().hamlss_precond_apply(self._A.ctx.h, self.h, _ptr(r), _ptr(out), HOST))
        return out

    def type(self):
        return self.kind

    def is_ready(self):
        return self.ready

    def energy_tier(self):
        return self.tier

    def release(self):
        if self.h:
            lib().hamlss_precond_release(self.h)
            self.h = None
            self.ready = False

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


class JacobiPreconditioner(PreconditionerBase):
    kind, tier = PREC_JACOBI, "CHEAP"

    def __init__(self, omega: float = 1.0):
        super().__init__()
        self.omega = omega

    def set_omega(self, omega):
        self.omega = omega

    def _params(self):
        return default_params(jacobi_omega=self.omega)


class ILUPreconditioner(PreconditionerBase):
    """ILU(0) (ilu.cpp:41-89), or ILUT(drop_tol, fill_per_row) (ilu.cpp:94-220) when
    drop_tol > 0 or fill_per_row > 0 -- the dispatch of ilu.cpp:31-36."""

    kind, tier = PREC_ILU, "MODERATE"

    def __init__(self):
        super().__init__()
        self.drop_tol, self.fill_p = 0.0, 0

    def set_drop_tol(self, tau):
        self.drop_tol = tau

    def set_fill_per_row(self, p):
        self.fill_p = p

    def _params(self):
        return default_params(drop_tol=self.drop_tol, fill_per_row=self.fill_p)

    def factors(self):
        """Factor values in the factor's pattern (A's for ILU(0))."""
        nnz = C.c_int32()
        _check(lib().hamlss_ilu_factor_csr(self.h, C.byref(nnz), None, None, None))
        lu = np.empty(max(nnz.value, 1))
        _check(lib().hamlss_ilu_factors(self.h, _ptr(lu)))
        return lu[:nnz.value]

    def factor_csr(self):
        """(row_ptr, col_idx, values) of the L\\U factor (ilu.cpp's lu_row_ptr_, lu_col_ind_,
        lu_val_)."""
        nnz = C.c_int32()
        _check(lib().hamlss_ilu_factor_csr(self.h, C.byref(nnz), None, None, None))
        rp = np.empty(self._A.rows() + 1, np.int32)
        ci = np.empty(max(nnz.value, 1), np.int32)
        v = np.empty(max(nnz.value, 1))
        _check(lib().hamlss_ilu_factor_csr(self.h, C.byref(nnz), _ptr(rp), _ptr(ci), _ptr(v)))
        return rp, ci[:nnz.value], v[:nnz.value]

    def level_sets(self, which: int):
        lev = np.empty(self._A.rows(), np.int32)
        n = C.c_int32()
        _check(lib().hamlss_ilu_levels(self.h, which, _ptr(lev), C.byref(n)))
        return n.value, lev


class AMGPreconditioner(PreconditionerBase):
    """Smoothed-aggregation AMG (amg.cpp), defaults of amg.hpp:96-103."""

    kind, tier = PREC_AMG, "EXPENSIVE"

    def __init__(self, **over):
        super().__init__()
        self.p = default_params(**over)

    def set_max_levels(self, n):
        self.p.amg_levels = n

    def set_strength_thresh(self, t):
        self.p.amg_strong = t

    def set_smooth_pre(self, n):
        self.p.amg_smooth_pre = n

    def set_smooth_post(self, n):
        self.p.amg_smooth_post = n

    def set_coarse_limit(self, n):
        self.p.amg_coarse_limit = n

    def _params(self):
        return self.p

    def levels(self) -> int:
        n = C.c_int32()
        _check(lib().hamlss_amg_num_levels(self.h, C.byref(n)))
        return n.value

    def level_matrix(self, level: int, which: int):
        rows, cols, nnz = C.c_int32(), C.c_int32(), C.c_int32()
        _check(lib().hamlss_amg_level_matrix(self.h, level, which, C.byref(rows), C.byref(cols),
                                             C.byref(nnz), None, None, None))
        rp = np.empty(rows.value + 1, np.int32)
        ci = np.empty(nnz.value, np.int32)
        v = np.empty(nnz.value)
        _check(lib().hamlss_amg_level_matrix(self.h, level, which, None, None, None, _ptr(rp),
                                             _ptr(ci), _ptr(v)))
        return rows.value, cols.value, rp, ci, v


_PREC_CLASSES = {PREC_JACOBI: JacobiPreconditioner, PREC_ILU: ILUPreconditioner,
                 PREC_AMG: AMGPreconditioner}


# --------------------------------------------------------------------------- solvers
class SolverBase:
    """SolverBase (solver_base.hpp:20-62)."""

    solver_type = SOLVER_CG

    def __init__(self):
        self._params = default_params()
        self._precond: Optional[PreconditionerBase] = None

    def set_params(self, p: Params):
        self._params = p

    def params(self) -> Params:
        return self._params

    def set_preconditioner(self, M: Optional[PreconditionerBase]):
        self._precond = M

    def set_verbose(self, v: bool):
        self._params.verbose = int(v)

    def type(self):
        return self.solver_type

    def solve(self, A: SparseMatrix, b, x, stats: Optional[Stats] = None) -> bool:
        st = stats if stats is not None else Stats()
        M = self._precond.h if self._precond is not None else None
        if _is_device(b):
            _check(lib().hamlss_solve(A.ctx.h, self.solver_type, A.h, M, _ptr(b), _ptr(x), DEVICE,
                                      C.byref(self._params), C.byref(st)))
            return bool(st.converged)
        b = _f64(b)
        if not isinstance(x, np.ndarray) or x.dtype != np.float64 or not x.flags.c_contiguous:
            raise ValueError("x must be a contiguous float64 numpy array (updated in place)")
        if len(x) != A.rows() or len(b) != A.rows():
            raise ValueError("x and b must have A.rows() entries")
        _check(lib().hamlss_solve(A.ctx.h, self.solver_type, A.h, M, _ptr(b), _ptr(x), HOST,
                                  C.byref(self._params), C.byref(st)))
        return bool(st.converged)


class CGSolver(SolverBase):
    solver_type = SOLVER_CG


class FGMRESSolver(SolverBase):
    solver_type = SOLVER_FGMRES


class PipelinedFGMRESSolver(SolverBase):
    """PipelinedFGMRESSolver (pipelined_fgmres_solver.hpp:44-74): FGMRES(m) whose cycle
    forms A M^-1 v_{j+1} one step early; same Arnoldi values, its own lucky-breakdown exit
    and cost model (pipelined_fgmres_solver.cpp:69-242).  Reports FGMRES as solver_used."""

    solver_type = SOLVER_PIPELINED_FGMRES


class SStepCGSolver(SolverBase):
    """SStepCGSolver(k) (sstep_cg_solver.hpp:57-60, sstep_cg_solver.cpp:170-305): batches
    of k Newton-Chebyshev basis vectors, one Gram matrix per batch.  The preconditioner is
    recorded in the stats but not applied, as in the reference."""

    solver_type = SOLVER_SSTEP_CG

    def __init__(self, k: int = 4):
        super().__init__()
        self.k = k

    def solve(self, A, b, x, stats=None) -> bool:
        saved = self._params                     # the constructor's k wins over params
        self._params = Params.from_buffer_copy(saved)
        self._params.sstep_k = self.k
        try:
            return super().solve(A, b, x, stats)
        finally:
            self._params = saved


_SOLVER_NAMES = {"CG": 0, "FGMRES": 1, "BICGSTAB": 2, "SSTEP_CG": 3, "SSTEP": 3, "S-STEP": 3,
                 "ASYNC_FGMRES": 4, "ASYNC": 4}
_PREC_NAMES = {"NONE": 0, "IDENTITY": 0, "JACOBI": 1, "DIAG": 1, "ILU": 2, "ILU0": 2, "AMG": 3}


class SolverFactory:
    """SolverFactory (solver_factory.hpp:40-88 / solver_factory.cpp:24-161)."""

    @staticmethod
    def parse_solver(s: str) -> int:
        u = s.upper()
        if u not in _SOLVER_NAMES:
            raise ValueError(f"SolverFactory: unknown solver name '{s}'")
        return _SOLVER_NAMES[u]

    @staticmethod
    def parse_precond(s: str) -> int:
        u = s.upper()
        if u not in _PREC_NAMES:
            raise ValueError(f"SolverFactory: unknown precond name '{s}'")
        return _PREC_NAMES[u]

    @staticmethod
    def make_solver(solver_type: int, params: Params) -> SolverBase:
        if solver_type in (SOLVER_CG,):
            s = CGSolver()
        elif solver_type in (SOLVER_FGMRES, 2):
            s = FGMRESSolver()
        elif solver_type == SOLVER_SSTEP_CG:
            s = SStepCGSolver(params.sstep_k)    # solver_factory.cpp:38-40
        else:
            raise ValueError("SolverFactory: solver type not provided by the engine")
        s.set_params(params)
        return s

    @staticmethod
    def make_precond(precond_type: int, A: SparseMatrix, params: Params, setup_time=None):
        if precond_type == PREC_NONE:
            if setup_time is not None:
                setup_time[0] = 0.0
            return None
        if precond_type not in _PREC_CLASSES:
            raise ValueError("SolverFactory: unknown PrecondType")
        M = _PREC_CLASSES[precond_type]()
        if precond_type == PREC_ILU:
            M.set_drop_tol(params.drop_tol)          # solver_factory.cpp:75
        elif precond_type == PREC_AMG:
            M.p = params                             # levels, strength, pre/post (:83-86)
        t = M.setup(A)
        if setup_time is not None:
            setup_time[0] = t
        return M

    @staticmethod
    def make(solver, precond, A: SparseMatrix, params: Params, setup_time=None):
        if isinstance(solver, str):
            solver = SolverFactory.parse_solver(solver)
        if isinstance(precond, str):
            precond = SolverFactory.parse_precond(precond)
        M = SolverFactory.make_precond(precond, A, params, setup_time)
        s = SolverFactory.make_solver(solver, params)
        if M is not None:
            s.set_preconditioner(M)
        return s, M

    @staticmethod
    def make_for_state(state: int, A: SparseMatrix, params: Params, setup_time=None):
        table = {STATE_EASY: (SOLVER_CG, PREC_JACOBI), STATE_MODERATE: (SOLVER_FGMRES, PREC_ILU),
                 STATE_HARD: (SOLVER_FGMRES, PREC_AMG)}
        if state not in table:
            raise ValueError("SolverFactory: unknown AdaptiveState")
        return SolverFactory.make(*table[state], A, params, setup_time)


class AdaptiveSelector:
    """AdaptiveSelector (adaptive_selector.hpp:49-161), ladder run by the engine."""

    def __init__(self, params: Optional[Params] = None):
        self._params = params or default_params()
        self._log: list = []
        self._state = STATE_EASY
        self.initial_state = STATE_EASY

    def extract_features(self, A: SparseMatrix):
        f = np.empty(24)
        s = C.c_int32()
        _check(lib().hamlss_extract_features(A.ctx.h, A.h, _ptr(f), C.byref(s)))
        return f, s.value

    def select_initial_state(self, A: SparseMatrix) -> int:
        return self.extract_features(A)[1]

    def solve(self, A: SparseMatrix, b, x, stats: Optional[Stats] = None) -> bool:
        st = stats if stats is not None else Stats()
        cap = 16
        log = (Escalation * cap)()
        nlog, init = C.c_int32(), C.c_int32()
        where = DEVICE if _is_device(b) else HOST
        if where == HOST:
            b = _f64(b)
            if not isinstance(x, np.ndarray) or x.dtype != np.float64 or len(x) != A.rows():
                raise ValueError("x must be a float64 numpy array with A.rows() entries")
        _check(lib().hamlss_solve_adaptive(A.ctx.h, A.h, _ptr(b), _ptr(x), where,
                                           C.byref(self._params), C.byref(st), log, cap,
                                           C.byref(nlog), C.byref(init)))
        self._log = [log[i] for i in range(min(nlog.value, cap))]
        self._state = st.state_used
        self.initial_state = init.value
        return bool(st.converged)

    def escalation_log(self):
        return self._log

    def current_state(self):
        return self._state


def amg_aggregate(A: SparseMatrix, theta: float = 0.25):
    """Device greedy aggregation of A (amg.cpp:30-67): (count, agg[n])."""
    agg = np.empty(A.rows(), np.int32)
    n = C.c_int32()
    _check(lib().hamlss_amg_aggregate(A.ctx.h, A.h, theta, _ptr(agg), C.byref(n)))
    return n.value, agg


__all__ = [
    "Context", "SparseMatrix", "SolverParams", "SolverStats", "Params", "Stats",
    "PreconditionerBase", "JacobiPreconditioner", "ILUPreconditioner", "AMGPreconditioner",
    "SolverBase", "CGSolver", "FGMRESSolver", "SolverFactory", "AdaptiveSelector",
    "HamlssError", "amg_aggregate", "problems",
]
