"""Bulk-copy SpMV and the reliable-update mixed-precision PCG (-m gpu).

SpMV: operators of at least 32,768 rows with short rows go through the bulk-copy kernel
(row tiles staged in shared memory by cp.async.bulk).  In FP64 it sums each row in column
order with separate multiply and add, so y = A x must equal the oracle's bit for bit --
also for ragged rows, empty rows and a row longer than a whole stage (read from global
memory by the same loop).

Mixed precision: the FP32 iteration runs the bulk-copy kernel with 1, 2, 4 and 8 lanes
per row (banded SPD operators of 5 to 41 entries per row); every solve must reach an FP64
true residual below 1e-10, recomputed on the host, and keep the FP64 iteration count
within a few trips (the search direction survives the FP64 residual replacements).
"""
import numpy as np
import pytest

from gpu_util import need_gpu
import hsps_b200 as H
from hsps_b200 import problems as P
from hsps_b200._abi import default_params

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    need_gpu()


def _csr_from_rows(n, rows):
    rp = np.zeros(n + 1, np.int32)
    rp[1:] = np.cumsum([len(r[0]) for r in rows])
    ci = np.concatenate([np.asarray(r[0], np.int32) for r in rows]) if rp[-1] else np.zeros(0, np.int32)
    v = np.concatenate([np.asarray(r[1], np.float64) for r in rows]) if rp[-1] else np.zeros(0)
    return rp, ci, v


def ragged(n, seed, long_row=None, long_len=0):
    """Random rows of 0..9 entries (sorted distinct columns), optionally one long row."""
    rng = np.random.default_rng(seed)
    rows = []
    for i in range(n):
        k = long_len if i == long_row else int(rng.integers(0, 10))
        cols = np.sort(rng.choice(n, size=min(k, n), replace=False))
        rows.append((cols, rng.uniform(-1.0, 1.0, len(cols))))
    return _csr_from_rows(n, rows)


def banded_spd(n, w, seed):
    """Symmetric, strictly diagonally dominant: off-diagonals -u (u in (0.5, 1]) for
    |i - j| <= w, diagonal = row sum of |off| + 0.25."""
    rng = np.random.default_rng(seed)
    offs = np.arange(1, w + 1)
    wts = {d: rng.uniform(0.5, 1.0, n - d) for d in offs}
    rp = np.zeros(n + 1, np.int64)
    cols, vals = [], []
    for i in range(n):
        c, v = [], []
        dsum = 0.0
        for d in offs[::-1]:
            if i - d >= 0:
                c.append(i - d); v.append(-wts[d][i - d]); dsum += wts[d][i - d]
        c.append(i); v.append(0.0)
        di = len(c) - 1
        for d in offs:
            if i + d < n:
                c.append(i + d); v.append(-wts[d][i]); dsum += wts[d][i]
        v[di] = dsum + 0.25
        cols.extend(c); vals.extend(v)
        rp[i + 1] = len(cols)
    return rp.astype(np.int32), np.array(cols, np.int32), np.array(vals)


SPMV_CASES = [
    ("varkappa256", lambda: P.varkappa_poisson_2d(256, 1.0, 9)),
    ("poisson300", lambda: P.poisson_2d(300)),
    ("ragged40k", lambda: ragged(40_000, 3)),
    ("ragged_long_row", lambda: ragged(40_000, 4, long_row=20_001, long_len=5_000)),
]


@pytest.mark.parametrize("name,make", SPMV_CASES, ids=[c[0] for c in SPMV_CASES])
def test_stream_spmv_fp64_bitwise(orc, name, make):
    rp, ci, v = make()
    n = len(rp) - 1
    assert n >= 32768 and len(v) / n <= 5.5          # the bulk-copy kernel's operators
    M = H.SparseMatrix(n, n, rp, ci, v)
    for seed in (1, 2):
        x = P.rhs(n, seed, -1.0, 1.0)
        y = M.spmv(x)
        assert np.array_equal(y, orc.spmv(rp, ci, v, x)), name


def skewed(n, seed, avg, long_lens):
    """Random rows of about `avg` entries and a few rows of the given lengths (power-law-like
    hubs), at rows spread over the matrix."""
    rng = np.random.default_rng(seed)
    hubs = {int(r): L for r, L in zip(rng.choice(n, size=len(long_lens), replace=False), long_lens)}
    rows = []
    for i in range(n):
        k = hubs.get(i, int(rng.integers(0, 2 * avg + 1)))
        cols = np.sort(rng.choice(n, size=min(k, n), replace=False))
        rows.append((cols, rng.uniform(-1.0, 1.0, len(cols))))
    return _csr_from_rows(n, rows), sorted(hubs)


SKEWED = [
    # bulk-copy kernel for the short rows (avg <= 5.5), three hubs
    ("stream_hubs", lambda: skewed(60_000, 11, 2, [30_000, 8_000, 2_000])),
    # plain kernel (avg > 5.5), two hubs
    ("plain_hubs", lambda: skewed(40_000, 12, 8, [20_000, 5_000])),
    # a small operator (plain kernel), one hub
    ("small_hub", lambda: skewed(3_000, 13, 3, [2_500])),
]


@pytest.mark.parametrize("name,make", SKEWED, ids=[c[0] for c in SKEWED])
def test_spmv_skewed_rows_fp64_bitwise(orc, name, make):
    """A skewed row-length profile: the few very long rows go to a warp each (products in
    parallel, the sum in column order by one lane), the rest to the usual kernels, which
    skip them.  FP64 results stay bit-identical to the reference's row-by-row sums, and
    the row profile built on the first call is reused by the second."""
    (rp, ci, v), hubs = make()
    n = len(rp) - 1
    assert max(np.diff(rp)[hubs]) > 32 * len(v) / n
    M = H.SparseMatrix(n, n, rp, ci, v)
    for seed in (1, 2):
        x = P.rhs(n, seed, -1.0, 1.0)
        assert np.array_equal(M.spmv(x), orc.spmv(rp, ci, v, x)), name


@pytest.mark.parametrize("w", [2, 4, 6, 12, 20])
def test_mixed_pcg_jacobi_lanes_per_row(orc, w):
    # 2w + 1 entries per row: w = 2 -> 1 lane per row, 4 -> 2, 6 -> 4, 12 -> 8 (FP32),
    # 20 -> the plain kernel
    n = 60_000
    rp, ci, v = banded_spd(n, w, 10 + w)
    b = P.rhs(n, 7, -1.0, 1.0)
    M = H.SparseMatrix(n, n, rp, ci, v)
    its = {}
    for prec in (0, H._abi.MIXED):
        p = default_params(tol=1e-10, max_iter=3000, precision=prec)
        s, _ = H.SolverFactory.make("CG", "JACOBI", M, p)
        x = np.zeros(n)
        st = H.SolverStats()
        assert s.solve(M, b, x, st), (w, prec, st.as_dict())
        r = b - orc.spmv(rp, ci, v, x)
        assert np.linalg.norm(r) / np.linalg.norm(b) < 1e-10
        its[prec] = st.iterations
    assert its[H._abi.MIXED] <= its[0] + max(3, its[0] // 10), its


def test_reliable_update_keeps_fp64_iterations(orc):
    side = 300
    A = P.varkappa_poisson_2d(side, 1.0, 5)
    n = side * side
    b = P.rhs(n, 5, -1.0, 1.0)
    M = H.SparseMatrix(n, n, *A)
    common = dict(tol=1e-10, max_iter=1000, amg_omega=2.0 / 3.0, amg_coarse_limit=512, amg_levels=25)
    out = {}
    for name, kw in (("fp64", dict(precision=0)), ("reliable", dict(precision=H._abi.MIXED)),
                     ("refinement", dict(precision=H._abi.MIXED, ir_update=0.0))):
        s, _ = H.SolverFactory.make("CG", "AMG", M, default_params(**common, **kw))
        x = np.zeros(n)
        st = H.SolverStats()
        assert s.solve(M, b, x, st), name
        r = b - orc.spmv(*A, x)
        assert np.linalg.norm(r) / np.linalg.norm(b) < 1e-10, name
        out[name] = (st.iterations, st.outer_iterations, x)
    it64, itr = out["fp64"][0], out["reliable"][0]
    assert itr <= it64 + 2, {k: v[:2] for k, v in out.items()}
    assert out["reliable"][1] >= 1                    # at least the confirming update
    x64 = out["fp64"][2]
    for name in ("reliable", "refinement"):
        assert np.max(np.abs(out[name][2] - x64)) <= 1e-6 * np.max(np.abs(x64)), name
    print({k: v[:2] for k, v in out.items()})
