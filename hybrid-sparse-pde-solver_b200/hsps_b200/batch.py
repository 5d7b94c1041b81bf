"""Batched solves: many independent systems in one persistent launch (hamlss_batch_*).

The reference solves one system per ``SolverBase::solve`` call; a batch keeps each
system's algorithm (CG + Jacobi, FGMRES + ILU(0), ...) and runs all of them inside one
kernel, FP32 inner iterations with FP64 refinement to ``params.tol``.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from . import _abi
from ._abi import BatchResult, Params, Stats, default_params, lib

HOST = _abi.HOST


def assemble(systems: Sequence[tuple]) -> tuple:
    """Lay local CSR systems (rp, ci, v) end to end as one block-diagonal CSR.

    Returns (row_off[count+1], row_ptr[N+1], col_idx[nnz], values[nnz]) with global
    row pointers and column indices."""
    sizes = np.array([len(s[0]) - 1 for s in systems], dtype=np.int64)
    nnzs = np.array([len(s[2]) for s in systems], dtype=np.int64)
    row_off = np.zeros(len(systems) + 1, np.int64)
    row_off[1:] = np.cumsum(sizes)
    nz_off = np.zeros(len(systems) + 1, np.int64)
    nz_off[1:] = np.cumsum(nnzs)
    if row_off[-1] >= 2**31 or nz_off[-1] >= 2**31:
        raise ValueError("batch exceeds 2^31 rows or nonzeros")
    rp = np.empty(row_off[-1] + 1, np.int32)
    ci = np.empty(nz_off[-1], np.int32)
    v = np.empty(nz_off[-1], np.float64)
    for k, (r, c, val) in enumerate(systems):
        r = np.asarray(r, np.int64)
        rp[row_off[k]:row_off[k + 1]] = (r[:-1] + nz_off[k]).astype(np.int32)
        ci[nz_off[k]:nz_off[k + 1]] = (np.asarray(c, np.int64) + row_off[k]).astype(np.int32)
        v[nz_off[k]:nz_off[k + 1]] = val
    rp[-1] = nz_off[-1]
    return row_off.astype(np.int32), rp, ci, v


class BatchSolver:
    """One batch of systems resident on the device.

    solvers / preconds: per system, engine enums (SOLVER_CG / SOLVER_FGMRES,
    PREC_NONE / PREC_JACOBI / PREC_ILU) or a single value for all."""

    def __init__(self, systems: Sequence[tuple], solvers, preconds,
                 params: Optional[Params] = None, ctx=None):
        from . import Context, _check

        self.ctx = ctx or Context.default()
        self.params = params or default_params()
        count = len(systems)
        self.count = count
        self.row_off, rp, ci, v = assemble(systems)
        self.N = int(self.row_off[-1])
        sv = np.broadcast_to(np.asarray(solvers, np.int32), (count,)).copy()
        pv = np.broadcast_to(np.asarray(preconds, np.int32), (count,)).copy()
        h = C.c_void_p()
        _check(lib().hamlss_batch_create(
            self.ctx.h, count, self.row_off.ctypes.data_as(C.c_void_p),
            rp.ctypes.data_as(C.c_void_p), ci.ctypes.data_as(C.c_void_p),
            v.ctypes.data_as(C.c_void_p), sv.ctypes.data_as(C.c_void_p),
            pv.ctypes.data_as(C.c_void_p), HOST, C.byref(self.params), C.byref(h)))
        self.h = h

    def split(self, flat: np.ndarray) -> list:
        return [flat[self.row_off[k]:self.row_off[k + 1]] for k in range(self.count)]

    def join(self, parts: Sequence[np.ndarray]) -> np.ndarray:
        out = np.concatenate([np.asarray(p, np.float64) for p in parts])
        if len(out) != self.N:
            raise ValueError("right-hand sides do not match the systems' sizes")
        return out

    def solve(self, b, x=None):
        """b, x: flat host arrays of N entries (or lists of per-system arrays).

        Returns (x_flat, results[count] as dicts, total Stats)."""
        from . import _check

        bf = self.join(b) if isinstance(b, (list, tuple)) else np.ascontiguousarray(b, np.float64)
        if x is None:
            xf = np.zeros(self.N)
        else:
            xf = self.join(x) if isinstance(x, (list, tuple)) else np.array(x, np.float64)
        res = (BatchResult * self.count)()
        tot = Stats()
        _check(lib().hamlss_batch_solve(self.ctx.h, self.h, bf.ctypes.data_as(C.c_void_p),
                                        xf.ctypes.data_as(C.c_void_p), HOST, res, C.byref(tot)))
        out = [{f: getattr(r, f) for f, _ in BatchResult._fields_} for r in res]
        return xf, out, tot

    def widths(self) -> list:
        from . import _check

        w = (C.c_int32 * 4)()
        _check(lib().hamlss_batch_get_widths(self.h, w))
        return list(w)

    def set_widths(self, widths) -> None:
        from . import _check

        w = (C.c_int32 * 4)(*widths)
        _check(lib().hamlss_batch_set_widths(self.h, w))

    def autotune(self, b, cache_path: Optional[str] = None) -> list:
        from . import _check

        bf = self.join(b) if isinstance(b, (list, tuple)) else np.ascontiguousarray(b, np.float64)
        w = (C.c_int32 * 4)()
        _check(lib().hamlss_batch_autotune(self.ctx.h, self.h, bf.ctypes.data_as(C.c_void_p), HOST,
                                           cache_path.encode() if cache_path else None, w))
        return list(w)

    def release(self) -> None:
        if getattr(self, "h", None):
            lib().hamlss_batch_release(self.h)
            self.h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass
