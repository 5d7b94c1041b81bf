"""ctypes mirror of include/hamlss.h (structs, enums) and the loader of libhamlss_b200.so.

The engine is the compiled library; this module only describes its C ABI.  Loading
fails loudly when the library has not been built: there is no Python fallback.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG_ROOT, "lib", "libhamlss_b200.so")

# status codes (hamlss.h)
OK = 0
ERR_INVALID = -1
ERR_SIZE = -2
ERR_ZERO_DIAG = -3
ERR_ZERO_PIVOT = -4
ERR_CUDA = -5
ERR_NOMEM = -6
ERR_NOT_READY = -7
ERR_TIMEOUT = -8
ERR_NONFINITE = -9
ERR_BUDGET = -10
ERR_MALFORMED = -11
ERR_CANCELLED = -12

HOST, DEVICE = 0, 1

# hsps::SolverType / PrecondType / AdaptiveState values (include/core/types.hpp:30-54)
SOLVER_CG, SOLVER_FGMRES, SOLVER_BICGSTAB, SOLVER_SSTEP_CG, SOLVER_ASYNC_FGMRES = range(5)
SOLVER_PIPELINED_FGMRES = 5          # engine value (PipelinedFGMRESSolver has no SolverType)
PREC_NONE, PREC_JACOBI, PREC_ILU, PREC_AMG, PREC_BLOCK_JACOBI, PREC_CHEBYSHEV = range(6)
STATE_EASY, STATE_MODERATE, STATE_HARD = range(3)
FP64, MIXED = 0, 1


class Params(C.Structure):
    """hamlss_params: hsps::SolverParams (types.hpp:119-143) + engine fields."""

    _fields_ = [
        ("tol", C.c_double),
        ("max_iter", C.c_int32),
        ("restart_size", C.c_int32),
        ("drop_tol", C.c_double),
        ("amg_levels", C.c_int32),
        ("amg_strength", C.c_double),
        ("amg_strong", C.c_double),
        ("amg_smooth_pre", C.c_int32),
        ("amg_smooth_post", C.c_int32),
        ("stall_window", C.c_int32),
        ("stall_threshold", C.c_double),
        ("verbose", C.c_int32),
        ("print_every", C.c_int32),
        ("sstep_k", C.c_int32),
        ("sstep_cond_tol", C.c_double),
        ("async_enabled", C.c_int32),
        ("async_max_stale", C.c_int32),
        ("fill_per_row", C.c_int32),
        ("block_size", C.c_int32),
        ("record_hw_energy", C.c_int32),
        ("precision", C.c_int32),
        ("ir_inner_tol", C.c_double),
        ("ir_max_outer", C.c_int32),
        ("amg_omega", C.c_double),
        ("amg_coarse_limit", C.c_int32),
        ("jacobi_omega", C.c_double),
        ("ladder_mode", C.c_int32),
        ("check_every", C.c_int32),
        ("amg_stall_ratio", C.c_double),
        ("ir_update", C.c_double),
    ]


def default_params(**over) -> Params:
    """The reference defaults of SolverParams plus the engine defaults (hamlss.h)."""
    p = Params(
        tol=1e-8, max_iter=2000, restart_size=50, drop_tol=1e-4, amg_levels=10,
        amg_strength=0.25, amg_strong=0.25, amg_smooth_pre=2, amg_smooth_post=2,
        stall_window=15, stall_threshold=0.95, verbose=0, print_every=25, sstep_k=1,
        sstep_cond_tol=1e12, async_enabled=0, async_max_stale=3, fill_per_row=0,
        block_size=1, record_hw_energy=0, precision=FP64, ir_inner_tol=1e-5,
        ir_max_outer=30, amg_omega=0.67, amg_coarse_limit=50, jacobi_omega=1.0,
        ladder_mode=0, check_every=8, amg_stall_ratio=0.0, ir_update=1e-2,
    )
    for k, v in over.items():
        if not hasattr(p, k):
            raise AttributeError(f"hamlss_params has no field {k!r}")
        setattr(p, k, v)
    return p


class Stats(C.Structure):
    """hamlss_stats: hsps::SolverStats (types.hpp:91-114) + engine fields."""

    _fields_ = [
        ("iterations", C.c_int32),
        ("initial_residual", C.c_double),
        ("final_residual", C.c_double),
        ("converged", C.c_int32),
        ("solve_time_s", C.c_double),
        ("setup_time_s", C.c_double),
        ("energy_joules", C.c_double),
        ("flop_count", C.c_int64),
        ("mem_bytes", C.c_int64),
        ("solver_used", C.c_int32),
        ("precond_used", C.c_int32),
        ("state_used", C.c_int32),
        ("restarts", C.c_int32),
        ("energy_joules_hw", C.c_double),
        ("rapl_start_j", C.c_double),
        ("rapl_end_j", C.c_double),
        ("sstep_k", C.c_int32),
        ("async_mode", C.c_int32),
        ("comm_bytes", C.c_int64),
        ("comm_time_s", C.c_double),
        ("true_residual", C.c_double),
        ("outer_iterations", C.c_int32),
        ("status", C.c_int32),
        ("device_time_s", C.c_double),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class BatchResult(C.Structure):
    """hamlss_batch_result: per-system outcome of a batched solve."""

    _fields_ = [
        ("iterations", C.c_int32),
        ("outer_iterations", C.c_int32),
        ("converged", C.c_int32),
        ("status", C.c_int32),
        ("initial_residual", C.c_double),
        ("final_residual", C.c_double),
    ]


class Escalation(C.Structure):
    """hamlss_escalation: hsps::EscalationRecord (adaptive_selector.hpp:38-44)."""

    _fields_ = [
        ("at_iteration", C.c_int32),
        ("from_state", C.c_int32),
        ("to_state", C.c_int32),
        ("residual_at_escalation", C.c_double),
        ("reason", C.c_int32),
    ]


class ServerConfig(C.Structure):
    """hamlss_server_config: device, solve lanes, HBM budget, coalescing limits."""

    _fields_ = [
        ("device", C.c_int32),
        ("slots", C.c_int32),
        ("hbm_budget_bytes", C.c_int64),
        ("batch_max_rows", C.c_int32),
        ("batch_max_count", C.c_int32),
        ("order", C.c_int32),
        ("large_rows", C.c_int32),
        ("max_large", C.c_int32),
    ]


class ServerReport(C.Structure):
    """hamlss_server_report: counters, latency percentiles and throughput of a server."""

    _fields_ = [
        ("submitted", C.c_int64),
        ("completed", C.c_int64),
        ("failed", C.c_int64),
        ("cancelled", C.c_int64),
        ("coalesced", C.c_int64),
        ("batches", C.c_int64),
        ("escalated", C.c_int64),
        ("fallback", C.c_int64),
        ("queued", C.c_int64),
        ("running", C.c_int32),
        ("peak_running", C.c_int32),
        ("admitted_bytes", C.c_int64),
        ("peak_admitted_bytes", C.c_int64),
        ("p50_latency_s", C.c_double),
        ("p99_latency_s", C.c_double),
        ("mean_latency_s", C.c_double),
        ("max_latency_s", C.c_double),
        ("solves_per_s", C.c_double),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


_lib = None


def lib() -> C.CDLL:
    """Load the engine library (once).  Raises if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"engine library {LIB_PATH} is missing; build it with "
                "`make -C hybrid-sparse-pde-solver_b200` (or __graft_entry__.build())")
        _lib = C.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


def _declare(L: C.CDLL) -> None:
    P, I32, I64, D, V = C.c_void_p, C.c_int32, C.c_int64, C.c_double, C.c_void_p
    pp = C.POINTER(C.c_void_p)
    pi = C.POINTER(C.c_int32)
    pd = C.POINTER(C.c_double)
    sig = {
        "hamlss_version": (C.c_char_p, []),
        "hamlss_last_error": (C.c_char_p, []),
        "hamlss_params_default": (None, [C.POINTER(Params)]),
        "hamlss_ctx_create": (C.c_int, [C.c_int, pp]),
        "hamlss_ctx_destroy": (C.c_int, [P]),
        "hamlss_ctx_synchronize": (C.c_int, [P]),
        "hamlss_ctx_stream": (C.c_int, [P, pp]),
        "hamlss_profile_enable": (C.c_int, [P, C.c_int, I32]),
        "hamlss_profile_read": (C.c_int, [P, I32, V, V, V, V, pi]),
        "hamlss_energy_read": (C.c_int, [C.c_int, pd]),
        "hamlss_mat_upload": (C.c_int, [P, I32, I32, I32, V, V, V, C.c_int, pp]),
        "hamlss_mat_update_values": (C.c_int, [P, V, C.c_int]),
        "hamlss_mat_info": (C.c_int, [P, pi, pi, pi]),
        "hamlss_mat_download": (C.c_int, [P, V, V, V]),
        "hamlss_mat_release": (C.c_int, [P]),
        "hamlss_spmv": (C.c_int, [P, P, V, V, C.c_int]),
        "hamlss_dot": (C.c_int, [P, I32, V, V, pd]),
        "hamlss_norm2": (C.c_int, [P, I32, V, pd]),
        "hamlss_axpy": (C.c_int, [P, I32, D, V, V]),
        "hamlss_axpby": (C.c_int, [P, I32, D, V, D, V]),
        "hamlss_scale": (C.c_int, [P, I32, D, V]),
        "hamlss_dot_noalloc": (C.c_int, [I32, V, V, pd, V]),
        "hamlss_precond_setup": (C.c_int, [P, P, C.c_int, C.POINTER(Params), pp, pd]),
        "hamlss_precond_apply": (C.c_int, [P, P, V, V, C.c_int]),
        "hamlss_precond_type": (C.c_int, [P, pi]),
        "hamlss_precond_release": (C.c_int, [P]),
        "hamlss_solve": (C.c_int, [P, C.c_int, P, P, V, V, C.c_int, C.POINTER(Params),
                                   C.POINTER(Stats)]),
        "hamlss_solve_adaptive": (C.c_int, [P, P, V, V, C.c_int, C.POINTER(Params),
                                            C.POINTER(Stats), C.POINTER(Escalation), I32, pi,
                                            pi]),
        "hamlss_extract_features": (C.c_int, [P, P, P, pi]),
        "hamlss_amg_aggregate": (C.c_int, [P, P, D, V, pi]),
        "hamlss_amg_num_levels": (C.c_int, [P, pi]),
        "hamlss_amg_level_matrix": (C.c_int, [P, I32, I32, pi, pi, pi, V, V, V]),
        "hamlss_ilu_factors": (C.c_int, [P, V]),
        "hamlss_ilu_factor_csr": (C.c_int, [P, pi, V, V, V]),
        "hamlss_ilu_levels": (C.c_int, [P, I32, V, pi]),
        "hamlss_batch_create": (C.c_int, [P, I32, V, V, V, V, V, V, C.c_int, C.POINTER(Params),
                                          pp]),
        "hamlss_batch_solve": (C.c_int, [P, P, V, V, C.c_int, V, C.POINTER(Stats)]),
        "hamlss_batch_set_widths": (C.c_int, [P, V]),
        "hamlss_batch_get_widths": (C.c_int, [P, V]),
        "hamlss_batch_autotune": (C.c_int, [P, P, V, C.c_int, C.c_char_p, V]),
        "hamlss_batch_release": (C.c_int, [P]),
        "hamlss_mtx_read_header": (C.c_int, [C.c_char_p, pi, pi, pi, C.POINTER(C.c_int64),
                                             C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
        "hamlss_mtx_read_matrix": (C.c_int, [C.c_char_p, pi, pi, pi, V, V, V]),
        "hamlss_mtx_read_vector": (C.c_int, [C.c_char_p, I32, V, pi]),
        "hamlss_mtx_write_vector": (C.c_int, [C.c_char_p, I32, V, C.c_char_p]),
        "hamlss_mtx_write_matrix": (C.c_int, [C.c_char_p, I32, I32, I32, V, V, V, C.c_char_p]),
        "hamlss_mat_load_mtx": (C.c_int, [P, C.c_char_p, pp]),
        "hamlss_server_config_default": (None, [C.POINTER(ServerConfig)]),
        "hamlss_server_create": (C.c_int, [C.POINTER(ServerConfig), pp]),
        "hamlss_server_submit": (C.c_int, [P, I32, I32, V, V, V, V, V, C.POINTER(Params),
                                           C.POINTER(C.c_int64)]),
        "hamlss_server_wait": (C.c_int, [P, I64, D, C.POINTER(Stats)]),
        "hamlss_server_test": (C.c_int, [P, I64, pi]),
        "hamlss_server_cancel": (C.c_int, [P, I64]),
        "hamlss_server_get_report": (C.c_int, [P, C.POINTER(ServerReport)]),
        "hamlss_server_reset_report": (C.c_int, [P]),
        "hamlss_server_destroy": (C.c_int, [P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args


def declared_symbols(header_path: str) -> list[str]:
    """Names of the functions a C header declares (for the export check)."""
    import re

    text = open(header_path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(hamlss_[a-z0-9_]+)\s*\(", text)))
