"""ILU(0), ILUT and FGMRES(m) on the device against the reference / oracle (-m gpu).

Bit-exact: ILU(0) factor values (the reference's lu_val_), ILUT factors (pattern, order
and values), level sets (oracle definition), and the ILU apply.  FGMRES uses CGS2 instead of MGS, so iteration counts
agree within +-1 and the least-squares residual is below tol.
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


def cases():
    yield "poisson40", P.poisson_2d(40)
    yield "varkappa37", P.varkappa_poisson_2d(37, 1.0, 4)
    for pe in (1.0, 10.0, 100.0):
        bx, by = P.convdiff_wind(48, pe)
        yield f"convdiff48_pe{int(pe)}", P.convection_diffusion_2d(48, 1.0, bx, by)
    yield "helmholtz30", P.helmholtz_2d(30, 0.5)


CASES = list(cases())
IDS = [c[0] for c in CASES]


def ilu(A):
    n = len(A[0]) - 1
    M = H.SparseMatrix(n, n, *A)
    I = H.ILUPreconditioner()
    I.setup(M)
    return M, I


@pytest.mark.parametrize("name,A", CASES, ids=IDS)
def test_ilu0_factors_bitwise(orc, ref, name, A):
    M, I = ilu(A)
    rc, lu_ref = ref.ilu0(*A)
    assert rc == 0
    assert np.array_equal(I.factors(), lu_ref)


@pytest.mark.parametrize("name,A", CASES, ids=IDS)
def test_ilu_level_sets_bitwise(orc, name, A):
    M, I = ilu(A)
    for which in (0, 1):
        n_dev, lev_dev = I.level_sets(which)
        n_orc, lev_orc = orc.levels(A[0], A[1], which)
        assert n_dev == n_orc
        assert np.array_equal(lev_dev, lev_orc)


@pytest.mark.parametrize("name,A", CASES, ids=IDS)
def test_ilu_apply_bitwise(ref, name, A):
    M, I = ilu(A)
    n = len(A[0]) - 1
    r = P.rhs(n, 21, -1.0, 1.0)
    rc, z = ref.precond_apply(2, *A, r, default_params(drop_tol=0.0))
    assert np.array_equal(I.apply(r), z)


def test_ilu_zero_pivot_raises():
    # row 1 eliminates with pivot row 0 whose diagonal is 0
    M = H.SparseMatrix.from_coo(2, 2, [0, 0, 1, 1], [0, 1, 0, 1], [0.0, 1.0, 1.0, 1.0])
    with pytest.raises(H.HamlssError) as e:
        H.ILUPreconditioner().setup(M)
    assert e.value.code == H._abi.ERR_ZERO_PIVOT


# ---------------------------------------------------------------- ILUT(tau, p)

ILUT_SETTINGS = [(1e-4, 0), (1e-3, 5), (1e-2, 0), (0.0, 3), (1e-4, 10)]


def ilut(A, dt, fp):
    n = len(A[0]) - 1
    M = H.SparseMatrix(n, n, *A)
    I = H.ILUPreconditioner()
    I.set_drop_tol(dt)
    I.set_fill_per_row(fp)
    I.setup(M)
    return M, I


@pytest.mark.parametrize("name,A", CASES, ids=IDS)
@pytest.mark.parametrize("dt,fp", ILUT_SETTINGS, ids=[f"{d:g}_{f}" for d, f in ILUT_SETTINGS])
def test_ilut_factor_and_apply_bitwise(orc, name, A, dt, fp):
    # setup_ilut (ilu.cpp:94-220): the device factor equals the oracle's entry for entry
    # (pattern, order and bits), and so does apply (ilu.cpp:225-271)
    M, I = ilut(A, dt, fp)
    rp, ci, v = I.factor_csr()
    orp, oci, ov = orc.ilut(*A, dt, fp)
    assert np.array_equal(rp, orp) and np.array_equal(ci, oci) and np.array_equal(v, ov)
    n = len(A[0]) - 1
    r = P.rhs(n, 22, -1.0, 1.0)
    rc, z = orc.ilu_apply(orp, oci, ov, r)
    assert rc == 0 and np.array_equal(I.apply(r), z)


def test_ilut_edge_cases_bitwise(orc):
    # an empty row, tiny diagonals the fill limit may drop, equal magnitudes (tie order)
    from test_oracle_pin import ILUT_EDGE_SETTINGS, ilut_edge_cases
    for name, A in ilut_edge_cases():
        for dt, fp in ILUT_EDGE_SETTINGS:
            M, I = ilut(A, dt, fp)
            for g, w in zip(I.factor_csr(), orc.ilut(*A, dt, fp)):
                assert np.array_equal(g, w), (name, dt, fp)


def test_ilut_large_wavefront(orc):
    # 65k rows: thousands of rows in flight at once, each waiting on the rows it eliminates
    bx, by = P.convdiff_wind(256, 30.0)
    A = P.convection_diffusion_2d(256, 1.0, bx, by)
    for dt, fp in ((1e-4, 0), (1e-3, 4)):
        M, I = ilut(A, dt, fp)
        got = I.factor_csr()
        want = orc.ilut(*A, dt, fp)
        for g, w in zip(got, want):
            assert np.array_equal(g, w)


@pytest.mark.parametrize("name,A", CASES, ids=IDS)
def test_fgmres_ilut_parity(orc, ref, name, A):
    # SolverFactory::make("FGMRES", "ILU") under the default drop_tol = 1e-4
    n = len(A[0]) - 1
    b = P.rhs(n, 13)
    p = default_params(tol=1e-8, max_iter=600, restart_size=30)
    rc, xo, so = ref.solve(1, H.PREC_ILU, *A, b, params=p)
    M = H.SparseMatrix(n, n, *A)
    s, Mp = H.SolverFactory.make(H.SOLVER_FGMRES, H.PREC_ILU, M, p)
    assert np.array_equal(Mp.factor_csr()[2], orc.ilut(*A, 1e-4, 0)[2])
    x = np.zeros(n)
    st = H.SolverStats()
    ok = s.solve(M, b, x, st)
    assert ok == bool(so.converged), (st.iterations, so.iterations)
    if so.converged:
        assert abs(st.iterations - so.iterations) <= 1, (st.iterations, so.iterations)
        r = b - orc.spmv(*A, x)
        assert np.linalg.norm(r) / np.linalg.norm(b) < 10 * p.tol


def test_ilut_kats():
    # test_improvements.cpp:49-114
    A = H.SparseMatrix.poisson_2d(10)
    b = np.ones(100)
    z = []
    for _ in range(2):
        I = H.ILUPreconditioner()
        I.set_drop_tol(0.0)
        I.set_fill_per_row(0)
        I.setup(A)
        z.append(I.apply(b))
    assert np.allclose(z[0], z[1], rtol=0, atol=1e-12)
    C = H.SparseMatrix.convection_diffusion_2d(10, 0.1, 3.0, 0.0)
    for dt in (0.0, 1e-3):
        I = H.ILUPreconditioner()
        I.set_drop_tol(dt)
        I.setup(C)
        assert np.linalg.norm(I.apply(np.ones(100))) > 0
    C = H.SparseMatrix.convection_diffusion_2d(12, 0.1, 8.0, 0.0)
    p = default_params(tol=1e-8, max_iter=3000, restart_size=50)
    its = []
    for dt, fp in ((0.0, 0), (1e-4, 5)):
        I = H.ILUPreconditioner()
        I.set_drop_tol(dt)
        I.set_fill_per_row(fp)
        I.setup(C)
        s = H.FGMRESSolver()
        s.set_params(p)
        s.set_preconditioner(I)
        st = H.SolverStats()
        x = np.zeros(144)
        assert s.solve(C, np.ones(144), x, st)
        its.append(st.iterations)
    assert its[1] <= its[0]


def test_ilut_row_overflow_refused():
    # a row touching more than 512 columns is refused (HAMLSS_ERR_NOMEM), not truncated
    n = 600
    r = list(range(n)) + [n - 1] * (n - 1)
    c = list(range(n)) + list(range(n - 1))
    v = [4.0] * n + [0.5] * (n - 1)
    M = H.SparseMatrix.from_coo(n, n, r, c, v)
    I = H.ILUPreconditioner()
    I.set_drop_tol(1e-4)
    with pytest.raises(H.HamlssError) as e:
        I.setup(M)
    assert e.value.code == H._abi.ERR_NOMEM


def test_ilu_level_sets_grid_closed_form():
    n = 64
    M, I = ilu(P.poisson_2d(n))
    nl, lev = I.level_sets(0)
    ii, jj = np.divmod(np.arange(n * n), n)
    assert nl == 2 * n - 1 and np.array_equal(lev, ii + jj)


@pytest.mark.parametrize("name,A", CASES, ids=IDS)
@pytest.mark.parametrize("prec", [H.PREC_ILU, H.PREC_JACOBI, H.PREC_NONE])
def test_fgmres_parity(orc, ref, name, A, prec):
    n = len(A[0]) - 1
    b = P.rhs(n, 13)
    p = default_params(tol=1e-8, max_iter=600, restart_size=30, drop_tol=0.0)
    rc, xo, so = ref.solve(1, prec, *A, b, params=p)
    M = H.SparseMatrix(n, n, *A)
    s, Mp = H.SolverFactory.make(H.SOLVER_FGMRES, prec, M, p)
    x = np.zeros(n)
    st = H.SolverStats()
    ok = s.solve(M, b, x, st)
    assert ok == bool(so.converged), (st.iterations, so.iterations)
    if so.converged:
        assert abs(st.iterations - so.iterations) <= 1, (st.iterations, so.iterations)
        assert st.final_residual < p.tol
        assert st.restarts == so.restarts or abs(st.iterations - so.iterations) == 1
        r = b - orc.spmv(*A, x)
        assert np.linalg.norm(r) / np.linalg.norm(b) < 10 * p.tol
    else:
        assert st.iterations == so.iterations == p.max_iter
        assert st.final_residual == 0.0          # reference quirk (fgmres_solver.cpp:197-226)


def test_fgmres_reference_kats():
    # test_solvers.cpp:151-240
    p = default_params(tol=1e-9, max_iter=3000, restart_size=40, drop_tol=0.0)
    D = H.SparseMatrix.from_coo(4, 4, range(4), range(4), [2.0, 3.0, 5.0, 7.0])
    s, _ = H.SolverFactory.make("FGMRES", "JACOBI", D, p)
    x = np.zeros(4)
    assert s.solve(D, np.array([4.0, 9.0, 15.0, 21.0]), x)
    assert np.allclose(x, [2.0, 3.0, 3.0, 3.0], atol=1e-10)
    C = H.SparseMatrix.convection_diffusion_2d(12, 0.1, 5.0, 0.0)
    s, _ = H.SolverFactory.make("FGMRES", "ILU", C, p)
    x = np.zeros(144)
    st = H.SolverStats()
    assert s.solve(C, np.ones(144), x, st) and st.final_residual < 1e-9
    q = default_params(tol=1e-9, max_iter=3000, restart_size=5)
    A = H.SparseMatrix.poisson_2d(16)
    s, _ = H.SolverFactory.make("FGMRES", "NONE", A, q)
    x = np.zeros(256)
    st = H.SolverStats()
    assert s.solve(A, np.ones(256), x, st) and st.restarts > 0


def test_fgmres_zero_rhs():
    A = H.SparseMatrix.poisson_2d(8)
    s, _ = H.SolverFactory.make("FGMRES", "ILU", A, default_params(drop_tol=0.0))
    st = H.SolverStats()
    x = np.zeros(64)
    assert s.solve(A, np.zeros(64), x, st) and st.iterations == 0 and st.final_residual == 0.0
