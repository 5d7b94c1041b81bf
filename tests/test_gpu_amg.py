"""SA-AMG on the device against the reference and the oracle (-m gpu).

Bit-exact: aggregation (every level), P, R and A_c (structure and values), and the
V-cycle output, against the reference where it can set up (<= 240^2 grids) and against
the oracle beyond.  Solves: iteration count within +-1 of the reference (FP64), and the
mixed-precision path reaches an FP64 true residual below tol.
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


def small_cases():
    yield "poisson32", P.poisson_2d(32)
    yield "varkappa40", P.varkappa_poisson_2d(40, 1.0, 8)
    bx, by = P.convdiff_wind(30, 10.0)
    yield "convdiff30_pe10", P.convection_diffusion_2d(30, 1.0, bx, by)
    yield "helmholtz25", P.helmholtz_2d(25, 5.0)


SMALL = list(small_cases())
SIDS = [c[0] for c in SMALL]


def dev(A):
    n = len(A[0]) - 1
    return H.SparseMatrix(n, n, *A)


@pytest.mark.parametrize("name,A", SMALL, ids=SIDS)
def test_aggregation_bitwise_vs_reference(ref, name, A):
    M = dev(A)
    for theta in (0.25, 0.1, 0.5):
        m_ref, agg_ref = ref.aggregate(*A, theta)
        m_dev, agg_dev = H.amg_aggregate(M, theta)
        assert m_dev == m_ref
        assert np.array_equal(agg_dev, agg_ref)


@pytest.mark.parametrize("side,sigma", [(256, 1.0), (400, 0.5)])
def test_aggregation_bitwise_large_vs_oracle(orc, side, sigma):
    A = P.varkappa_poisson_2d(side, sigma, 3)
    m_o, agg_o = orc.aggregate(*A, 0.25)
    m_d, agg_d = H.amg_aggregate(dev(A), 0.25)
    assert m_d == m_o and np.array_equal(agg_d, agg_o)
    A = P.poisson_2d(side)
    assert np.array_equal(H.amg_aggregate(dev(A), 0.25)[1], orc.aggregate(*A, 0.25)[1])


def hierarchy(M):
    out = []
    for l in range(M.levels()):
        d = {"A": M.level_matrix(l, 0)}
        if l < M.levels() - 1:
            d["P"] = M.level_matrix(l, 1)
            d["R"] = M.level_matrix(l, 2)
        out.append(d)
    return out


def assert_same_hierarchy(h_dev, h_ref):
    # The reference also stores, on each coarse level, a copy of the P and R that lead to
    # it (amg.cpp:220-229); the coarsest level's copy is the previous level's operator, so
    # P and R are compared on the levels that own them: every level but the coarsest.
    assert len(h_dev) == len(h_ref)
    for l, (a, b) in enumerate(zip(h_dev, h_ref)):
        for k in ("A", "P", "R"):
            if k not in b or (k != "A" and l == len(h_ref) - 1):
                continue
            assert a[k][:2] == b[k][:2], (l, k)
            for x, y in zip(a[k][2:], b[k][2:]):
                assert np.array_equal(x, y), (l, k)


@pytest.mark.parametrize("name,A", SMALL, ids=SIDS)
def test_hierarchy_bitwise_vs_reference(ref, name, A):
    M = H.AMGPreconditioner()
    M.setup(dev(A))
    assert_same_hierarchy(hierarchy(M), ref.amg_hierarchy(*A))


def test_hierarchy_bitwise_large_vs_oracle(orc):
    # 384^2 is beyond what the reference can set up (dense n_f x n_c buffer)
    A = P.varkappa_poisson_2d(384, 1.0, 2)
    M = H.AMGPreconditioner()
    M.setup(dev(A))
    assert_same_hierarchy(hierarchy(M), orc.amg_hierarchy(*A))


def test_hierarchy_bitwise_wide_coarse_vs_oracle(orc):
    # 1024^2: coarse operators with more columns (132,780 and 35,719) than a shared-memory
    # accumulator holds, where long Galerkin rows take the windowed accumulator
    A = P.varkappa_poisson_2d(1024, 1.0, 2)
    M = H.AMGPreconditioner()
    M.setup(dev(A))
    assert_same_hierarchy(hierarchy(M), orc.amg_hierarchy(*A))


@pytest.mark.parametrize("name,A", SMALL, ids=SIDS)
def test_vcycle_bitwise_vs_reference(ref, name, A):
    n = len(A[0]) - 1
    M = H.AMGPreconditioner()
    M.setup(dev(A))
    r = P.rhs(n, 17, -1.0, 1.0)
    rc, z = ref.precond_apply(3, *A, r)
    assert np.array_equal(M.apply(r), z)


@pytest.mark.parametrize("name,A", SMALL, ids=SIDS)
@pytest.mark.parametrize("solver", [H.SOLVER_CG, H.SOLVER_FGMRES])
def test_amg_solve_parity(orc, ref, name, A, solver):
    n = len(A[0]) - 1
    b = P.rhs(n, 19)
    p = default_params(tol=1e-8, max_iter=500, restart_size=30)
    rc, xo, so = ref.solve(solver, 3, *A, b, params=p)
    M = dev(A)
    s, _ = H.SolverFactory.make(solver, H.PREC_AMG, M, p)
    x = np.zeros(n)
    st = H.SolverStats()
    ok = s.solve(M, b, x, st)
    assert ok == bool(so.converged)
    assert abs(st.iterations - so.iterations) <= 1, (st.iterations, so.iterations)
    if ok:
        r = b - orc.spmv(*A, x)
        assert np.linalg.norm(r) / np.linalg.norm(b) < 10 * p.tol


@pytest.mark.parametrize("side", [64, 300])
def test_mixed_precision_amg_pcg(orc, side):
    A = P.varkappa_poisson_2d(side, 1.0, 5)
    n = side * side
    b = P.rhs(n, 5, -1.0, 1.0)
    M = dev(A)
    for omega, coarse in ((0.67, 50), (2.0 / 3.0, 512)):
        p64 = default_params(tol=1e-10, max_iter=1000, amg_omega=omega, amg_coarse_limit=coarse,
                             amg_levels=25)
        pm = default_params(tol=1e-10, max_iter=1000, amg_omega=omega, amg_coarse_limit=coarse,
                            amg_levels=25, precision=H._abi.MIXED)
        s64, _ = H.SolverFactory.make("CG", "AMG", M, p64)
        x64 = np.zeros(n)
        st64 = H.SolverStats()
        assert s64.solve(M, b, x64, st64)
        sm, _ = H.SolverFactory.make("CG", "AMG", M, pm)
        xm = np.zeros(n)
        stm = H.SolverStats()
        assert sm.solve(M, b, xm, stm)
        r = b - orc.spmv(*A, xm)
        assert np.linalg.norm(r) / np.linalg.norm(b) < 1e-10
        assert stm.true_residual < 1e-10 and stm.outer_iterations >= 2
        # error against the FP64 solve, relative to the solution size
        assert np.max(np.abs(xm - x64)) <= 1e-6 * np.max(np.abs(x64))


def test_mixed_precision_fgmres_ilu(orc):
    bx, by = P.convdiff_wind(64, 10.0)
    A = P.convection_diffusion_2d(64, 1.0, bx, by)
    n = 64 * 64
    b = P.rhs(n, 2)
    M = dev(A)
    p = default_params(tol=1e-10, max_iter=2000, restart_size=30, drop_tol=0.0, precision=H._abi.MIXED)
    s, _ = H.SolverFactory.make("FGMRES", "ILU", M, p)
    x = np.zeros(n)
    st = H.SolverStats()
    assert s.solve(M, b, x, st)
    r = b - orc.spmv(*A, x)
    assert np.linalg.norm(r) / np.linalg.norm(b) < 1e-9


def test_amg_single_level_and_tiny():
    # rows <= coarse_limit: the hierarchy is one level and the V-cycle is the dense solve
    A = H.SparseMatrix.poisson_2d(5)
    M = H.AMGPreconditioner()
    M.setup(A)
    assert M.levels() == 1
    b = np.arange(25, dtype=float)
    z = M.apply(b)
    d = np.zeros((25, 25))
    rp, ci, v = A.row_ptr(), A.col_idx(), A.values()
    d[np.repeat(np.arange(25), np.diff(rp)), ci] = v
    assert np.allclose(d @ z, b, atol=1e-12)


@pytest.mark.parametrize("kind", ["varkappa", "convdiff"])
def test_blocked_coarse_lu_inverse(kind):
    # a one-level hierarchy of 2025 rows (> 1024): the V-cycle is the blocked dense LU's
    # explicit inverse; compare with numpy's dense solve.  Bound: 1e-10 relative, the
    # condition numbers here are below 1e4.
    side = 45
    if kind == "varkappa":
        A = P.varkappa_poisson_2d(side, 1.0, 3)
    else:
        A = P.convection_diffusion_2d(side, 1.0, *P.convdiff_wind(side, 30.0))
    n = side * side
    M = H.AMGPreconditioner()
    M.set_coarse_limit(3000)
    M.setup(dev(A))
    assert M.levels() == 1
    r = P.rhs(n, 8, -1.0, 1.0)
    z = M.apply(r)
    d = np.zeros((n, n))
    rp, ci, v = A
    d[np.repeat(np.arange(n), np.diff(rp)), ci] = v
    want = np.linalg.solve(d, r)
    assert np.max(np.abs(z - want)) <= 1e-10 * np.max(np.abs(want))


def test_stall_ratio_cuts_hierarchy(orc):
    # amg_stall_ratio: the first level that keeps more than 70% of its rows becomes the
    # dense coarsest level (here above 1024 rows, so the blocked LU runs); PCG still
    # converges to the FP64 tolerance, in FP64 and in mixed precision
    A = P.varkappa_poisson_2d(128, 1.0, 4)
    n = 128 * 128
    b = P.rhs(n, 4, -1.0, 1.0)
    M = dev(A)
    full = H.AMGPreconditioner(amg_omega=2.0 / 3.0, amg_coarse_limit=512, amg_levels=25)
    full.setup(M)
    cut = H.AMGPreconditioner(amg_omega=2.0 / 3.0, amg_coarse_limit=512, amg_levels=25,
                              amg_stall_ratio=0.7)
    cut.setup(M)
    assert cut.levels() <= full.levels()
    for prec in (0, H._abi.MIXED):
        p = default_params(tol=1e-10, max_iter=500, amg_omega=2.0 / 3.0, amg_coarse_limit=512,
                           amg_levels=25, amg_stall_ratio=0.7, precision=prec)
        s, _ = H.SolverFactory.make("CG", "AMG", M, p)
        x = np.zeros(n)
        st = H.SolverStats()
        assert s.solve(M, b, x, st)
        assert np.linalg.norm(b - orc.spmv(*A, x)) / np.linalg.norm(b) < 1.5e-10


def test_blocked_coarse_lu_pivoting():
    # rows of a Poisson matrix shifted cyclically: most diagonal entries are zero, so the
    # blocked LU must fall back to partial pivoting; the one-level V-cycle is then the
    # explicit inverse, compared with numpy's dense solve to 1e-10 relative
    side = 45
    n = side * side
    rp0, ci0, v0 = P.poisson_2d(side)
    order = (np.arange(n) + 7) % n
    lens = np.diff(rp0)[order]
    rp = np.zeros(n + 1, np.int32)
    np.cumsum(lens, out=rp[1:])
    ci = np.concatenate([ci0[rp0[i]:rp0[i + 1]] for i in order]).astype(np.int32)
    v = np.concatenate([v0[rp0[i]:rp0[i + 1]] for i in order])
    M = H.AMGPreconditioner()
    M.set_coarse_limit(3000)
    M.setup(H.SparseMatrix(n, n, rp, ci, v))
    assert M.levels() == 1
    r = P.rhs(n, 9, -1.0, 1.0)
    z = M.apply(r)
    d = np.zeros((n, n))
    d[np.repeat(np.arange(n), np.diff(rp)), ci] = v
    want = np.linalg.solve(d, r)
    assert np.max(np.abs(z - want)) <= 1e-10 * np.max(np.abs(want))


AMG_VARIANTS = [dict(amg_levels=3), dict(amg_strong=0.5), dict(amg_strong=0.08),
                dict(amg_smooth_pre=1, amg_smooth_post=3)]


@pytest.mark.parametrize("over", AMG_VARIANTS,
                         ids=[",".join(f"{k}={v}" for k, v in o.items()) for o in AMG_VARIANTS])
def test_amg_parameters_bitwise_vs_oracle(orc, over):
    # the factory's AMG parameters (solver_factory.cpp:80-88): levels, strength threshold,
    # pre/post sweeps -- hierarchy bit for bit; the V-cycle bit for bit while the coarsest
    # level is solved by the same elimination (up to 96 rows), else within rounding (above
    # 96 rows the engine applies an explicit inverse as a GEMV)
    A = P.varkappa_poisson_2d(28, 1.0, 13)
    p = default_params(**over)
    M = H.SolverFactory.make_precond(H.PREC_AMG, dev(A), p)
    h = hierarchy(M)
    assert_same_hierarchy(h, orc.amg_hierarchy(*A, params=p))
    r = P.rhs(28 * 28, 3, -1.0, 1.0)
    z, zo = M.apply(r), orc.precond_apply(3, *A, r, p)[1]
    if h[-1]["A"][0] <= 96:
        assert np.array_equal(z, zo)
    else:
        assert np.max(np.abs(z - zo)) <= 1e-10 * np.max(np.abs(zo))
