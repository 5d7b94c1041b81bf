"""MatrixMarket files and the dataset runner.

``MatrixMarketIO`` mirrors the reference's class of the same name
(include/utils/matrix_market_io.hpp:80-130) over the engine's C ABI (hamlss_mtx_*).
``run_dataset`` mirrors examples/run_dataset.cpp: every matrix of a directory (or the
listed files) with its ``<name>_rhs.mtx`` when present (else b = 1), solved by the
adaptive ladder on the device, one result row per matrix.
"""
from __future__ import annotations

import ctypes as C
import os
import time
from typing import Optional

import numpy as np

from . import _abi
from ._abi import default_params, lib

FORMATS = ("coordinate", "array")
FIELDS = ("real", "integer", "complex", "pattern")
SYMMETRIES = ("general", "symmetric", "skew-symmetric", "hermitian")


def _b(path) -> bytes:
    return os.fsencode(os.fspath(path))


class MatrixMarketIO:
    """MatrixMarketIO (utils/matrix_market_io.hpp); static methods, same names."""

    @staticmethod
    def read_header(path) -> dict:
        from . import _check

        f, fl, sy = C.c_int32(), C.c_int32(), C.c_int32()
        r, c, e = C.c_int64(), C.c_int64(), C.c_int64()
        _check(lib().hamlss_mtx_read_header(_b(path), C.byref(f), C.byref(fl), C.byref(sy),
                                            C.byref(r), C.byref(c), C.byref(e)))
        sym = SYMMETRIES[sy.value]
        nnz_full = e.value if sym == "general" or f.value == 1 else 2 * e.value - r.value
        return {"format": FORMATS[f.value], "field": FIELDS[fl.value], "symmetry": sym,
                "rows": r.value, "cols": c.value, "nnz": e.value, "nnz_full": nnz_full,
                "kind": f"{FORMATS[f.value]} {FIELDS[fl.value]} {sym}"}

    @staticmethod
    def read_csr(path):
        """(rows, cols, row_ptr, col_idx, values) on the host."""
        from . import _check

        r, c, nz = C.c_int32(), C.c_int32(), C.c_int32()
        _check(lib().hamlss_mtx_read_matrix(_b(path), C.byref(r), C.byref(c), C.byref(nz),
                                            None, None, None))
        rp = np.empty(r.value + 1, np.int32)
        ci = np.empty(max(nz.value, 1), np.int32)
        v = np.empty(max(nz.value, 1), np.float64)
        _check(lib().hamlss_mtx_read_matrix(_b(path), C.byref(r), C.byref(c), C.byref(nz),
                                            rp.ctypes.data, ci.ctypes.data, v.ctypes.data))
        return r.value, c.value, rp, ci[:nz.value], v[:nz.value]

    @staticmethod
    def load_matrix(path, ctx=None):
        from . import SparseMatrix

        rows, cols, rp, ci, v = MatrixMarketIO.read_csr(path)
        return SparseMatrix(rows, cols, rp, ci, v, ctx)

    @staticmethod
    def load_vector(path, expected_n: int = 0) -> np.ndarray:
        from . import _check

        n = C.c_int32()
        _check(lib().hamlss_mtx_read_vector(_b(path), expected_n, None, C.byref(n)))
        out = np.empty(max(n.value, 1), np.float64)
        _check(lib().hamlss_mtx_read_vector(_b(path), expected_n, out.ctypes.data, C.byref(n)))
        return out[:n.value]

    @staticmethod
    def make_default_rhs(n: int, value: float = 1.0) -> np.ndarray:
        return np.full(n, value, np.float64)

    @staticmethod
    def load_problem(matrix_path, rhs_path: str = "", ctx=None):
        """(SparseMatrix, b): the RHS file if it loads with the matrix's size, else b = 1
        (MatrixMarketIO::load_problem, matrix_market_io.cpp)."""
        A = MatrixMarketIO.load_matrix(matrix_path, ctx)
        b = None
        if rhs_path:
            try:
                b = MatrixMarketIO.load_vector(rhs_path, A.rows())
                if len(b) != A.rows():
                    b = None
            except Exception:
                b = None
        if b is None:
            b = MatrixMarketIO.make_default_rhs(A.rows())
        return A, b

    @staticmethod
    def save_vector(path, v, comment: str = "") -> None:
        from . import _check

        a = np.ascontiguousarray(v, np.float64)
        _check(lib().hamlss_mtx_write_vector(_b(path), len(a), a.ctypes.data,
                                             comment.encode() if comment else None))

    @staticmethod
    def save_matrix(path, A, comment: str = "") -> None:
        from . import _check

        rp, ci, v = (np.ascontiguousarray(A.row_ptr(), np.int32),
                     np.ascontiguousarray(A.col_idx(), np.int32),
                     np.ascontiguousarray(A.values(), np.float64))
        _check(lib().hamlss_mtx_write_matrix(_b(path), A.rows(), A.cols(), len(v), rp.ctypes.data,
                                             ci.ctypes.data, v.ctypes.data,
                                             comment.encode() if comment else None))

    @staticmethod
    def list_mtx_files(directory) -> list:
        """The .mtx files of a directory, sorted, without the *_rhs / *_b right-hand sides."""
        out = []
        for name in os.listdir(directory):
            stem, ext = os.path.splitext(name)
            if ext != ".mtx" or stem.endswith("_rhs") or stem.endswith("_b"):
                continue
            out.append(os.path.join(directory, name))
        return sorted(out)


def run_dataset(paths, params=None, verbose: bool = True) -> list:
    """Solve every listed matrix (or every matrix of a directory) with the adaptive ladder
    on the device; one dict per matrix: name, n, nnz, spd (symmetric with a positive
    diagonal), final state, iterations, escalations, rel_res, solve time, energy (the
    reference's proxy model), converged -- examples/run_dataset.cpp's columns."""
    from . import AdaptiveSelector, SolverStats

    if isinstance(paths, (str, os.PathLike)) and os.path.isdir(paths):
        paths = MatrixMarketIO.list_mtx_files(paths)
    # examples/run_dataset.cpp:305-310: tol 1e-8, max_iter 5000, restart 60, stall window 20;
    # drop_tol keeps its default (1e-4: the MODERATE rung's ILU is ILUT)
    p = params or default_params(tol=1e-8, max_iter=5000, restart_size=60, stall_window=20)
    rows = []
    for path in paths:
        name = os.path.splitext(os.path.basename(path))[0]
        rhs = os.path.join(os.path.dirname(path), name + "_rhs.mtx")
        try:
            A, b = MatrixMarketIO.load_problem(path, rhs if os.path.exists(rhs) else "")
            rp, ci, v = A.row_ptr(), A.col_idx(), A.values()
            sym = _spd_like(A.rows(), rp, ci, v)
            sel = AdaptiveSelector(p)
            x = np.zeros(A.rows())
            st = SolverStats()
            t0 = time.perf_counter()
            ok = sel.solve(A, b, x, st)
            dt = time.perf_counter() - t0
            r = np.linalg.norm(b - A.spmv(x)) / max(np.linalg.norm(b), 1e-300)
            rows.append({"name": name, "n": A.rows(), "nnz": A.nnz(), "spd": sym,
                         "state": st.state_used, "iterations": st.iterations,
                         "escalations": len(sel.escalation_log()), "rel_res": float(r),
                         "solve_time_s": dt, "energy_j": st.energy_joules, "converged": bool(ok)})
        except Exception as e:      # one bad file does not stop the run
            rows.append({"name": name, "error": str(e)})
    if verbose:
        _print_table(rows)
    return rows


def _spd_like(n, rp, ci, v) -> bool:
    rows = np.repeat(np.arange(n), np.diff(rp))
    if np.any(v[ci == rows] <= 0):
        return False
    key = rows.astype(np.int64) * n + ci
    tkey = ci.astype(np.int64) * n + rows
    o1, o2 = np.argsort(key), np.argsort(tkey)
    return bool(np.array_equal(key[o1], tkey[o2]) and np.array_equal(v[o1], v[o2]))


def _print_table(rows) -> None:
    states = ("EASY", "MODERATE", "HARD")
    print(f"{'Matrix':28s}{'n':>10s}{'nnz':>10s}{'SPD':>6s}  {'Final State':18s}{'Iters':>10s}"
          f"{'Esc':>6s}{'Rel-Res':>12s}{'Time(s)':>10s}{'Energy(J)':>12s}{'Conv':>7s}")
    for r in rows:
        if "error" in r:
            print(f"{r['name']:28s}  ERROR: {r['error']}")
            continue
        print(f"{r['name']:28s}{r['n']:>10d}{r['nnz']:>10d}{('yes' if r['spd'] else 'no'):>6s}  "
              f"{states[r['state']]:18s}{r['iterations']:>10d}{r['escalations']:>6d}"
              f"{r['rel_res']:>12.2e}{r['solve_time_s']:>10.4f}{r['energy_j']:>12.2e}"
              f"{('YES' if r['converged'] else 'NO'):>7s}")
