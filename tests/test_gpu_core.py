"""Device SpMV, BLAS-1, Jacobi and PCG against the oracle / reference (-m gpu).

Tolerances: SpMV is bit-identical to the reference's row sums (same order, no fused
multiply-add).  Dots use a tree order, so they agree to 1e-14 relative.  Solves agree
on iteration count within +-1 and reach rel-res <= tol, checked in FP64 on the host.
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
    yield "poisson64", P.poisson_2d(64)
    yield "varkappa48", P.varkappa_poisson_2d(48, 1.0, 3)
    bx, by = P.convdiff_wind(40, 10.0)
    yield "convdiff40", P.convection_diffusion_2d(40, 1.0, bx, by)
    yield "helmholtz33", P.helmholtz_2d(33, 3.0)


CASES = list(cases())
IDS = [c[0] for c in CASES]


@pytest.mark.parametrize("name,A", CASES, ids=IDS)
def test_spmv_bitwise(orc, name, A):
    n = len(A[0]) - 1
    M = H.SparseMatrix(n, n, *A)
    for seed in (1, 2):
        x = P.rhs(n, seed, -1.0, 1.0)
        assert np.array_equal(M.spmv(x), orc.spmv(*A, x))


def test_spmv_large_and_ragged(orc):
    # rows of very different length (long rows cross the staging chunk)
    rng = np.random.default_rng(0)
    n = 3000
    lens = rng.integers(0, 700, n)
    lens[::97] = 0
    rp = np.zeros(n + 1, np.int32)
    rp[1:] = np.cumsum(lens)
    ci = np.concatenate([np.sort(rng.choice(n, size=l, replace=False)) for l in lens]).astype(np.int32)
    v = rng.standard_normal(len(ci))
    M = H.SparseMatrix(n, n, rp, ci, v)
    x = rng.standard_normal(n)
    assert np.array_equal(M.spmv(x), orc.spmv(rp, ci, v, x))


def test_empty_and_tiny():
    M = H.SparseMatrix(1, 1, [0, 1], [0], [2.0])
    assert M.spmv(np.array([3.0]))[0] == 6.0
    Z = H.SparseMatrix(5, 5, np.zeros(6, np.int32), [], [])
    assert np.array_equal(Z.spmv(np.ones(5)), np.zeros(5))


def test_blas1(orc):
    import torch
    import ctypes as C
    n = 1_000_003
    a = P.rhs(n, 3, -1, 1)
    b = P.rhs(n, 4, -1, 1)
    da = torch.from_numpy(a).cuda()
    db = torch.from_numpy(b).cuda()
    ctx = H.Context.default()
    L = H.lib()
    out = C.c_double()
    assert L.hamlss_dot(ctx.h, n, C.c_void_p(da.data_ptr()), C.c_void_p(db.data_ptr()), C.byref(out)) == 0
    assert abs(out.value - orc.dot(a, b)) <= 1e-13 * np.abs(a * b).sum()
    assert L.hamlss_axpy(ctx.h, n, 0.5, C.c_void_p(da.data_ptr()), C.c_void_p(db.data_ptr())) == 0
    assert np.array_equal(db.cpu().numpy(), b + 0.5 * a)
    assert L.hamlss_axpby(ctx.h, n, 2.0, C.c_void_p(da.data_ptr()), -1.0, C.c_void_p(db.data_ptr())) == 0
    assert np.array_equal(db.cpu().numpy(), 2.0 * a + (-1.0) * (b + 0.5 * a))


@pytest.mark.parametrize("name,A", CASES, ids=IDS)
def test_jacobi_apply_bitwise(orc, name, A):
    n = len(A[0]) - 1
    M = H.SparseMatrix(n, n, *A)
    J = H.JacobiPreconditioner()
    J.setup(M)
    r = P.rhs(n, 9)
    rc, z = orc.precond_apply(1, *A, r)
    assert np.array_equal(J.apply(r), z)


def test_jacobi_zero_diagonal_raises():
    M = H.SparseMatrix.from_coo(3, 3, [0, 1, 2, 2], [0, 1, 2, 0], [1.0, 0.0, 1.0, 2.0])
    with pytest.raises(H.HamlssError) as e:
        H.JacobiPreconditioner().setup(M)
    assert e.value.code == H._abi.ERR_ZERO_DIAG and "row 1" in str(e.value)


def test_malformed_csr_rejected():
    with pytest.raises(H.HamlssError) as e:
        H.SparseMatrix(3, 3, [0, 2, 3, 4], [1, 0, 2, 2], [1.0, 1.0, 1.0, 1.0])   # unsorted row 0
    assert e.value.code == H._abi.ERR_MALFORMED
    with pytest.raises(H.HamlssError):
        H.SparseMatrix(2, 2, [0, 1, 2], [0, 5], [1.0, 1.0])                   # column out of range


@pytest.mark.parametrize("name,A", CASES, ids=IDS)
@pytest.mark.parametrize("prec", [H.PREC_JACOBI, H.PREC_NONE])
def test_cg_parity_fp64(orc, ref, name, A, prec):
    n = len(A[0]) - 1
    b = P.rhs(n, 11)
    p = default_params(tol=1e-8, max_iter=1000)
    rc, xo, so = ref.solve(0, prec, *A, b, params=p)
    M = H.SparseMatrix(n, n, *A)
    s, Mp = H.SolverFactory.make(H.SOLVER_CG, prec, M, p)
    x = np.zeros(n)
    st = H.SolverStats()
    ok = s.solve(M, b, x, st)
    assert ok == bool(so.converged)
    assert abs(st.iterations - so.iterations) <= 1, (st.iterations, so.iterations)
    r = b - orc.spmv(*A, x)
    true_rel = np.linalg.norm(r) / np.linalg.norm(b)
    if so.converged:
        assert st.final_residual < p.tol
        assert true_rel < 10 * p.tol
        assert abs(st.true_residual - true_rel) <= 1e-3 * true_rel + 1e-15
        assert np.max(np.abs(x - xo)) <= 1e-5 * np.max(np.abs(xo))
    assert st.initial_residual == pytest.approx(so.initial_residual, rel=1e-12)


def test_cg_reference_kats():
    # test_solvers.cpp:42-129 in the reference
    p = default_params(tol=1e-9, max_iter=3000, restart_size=40)
    A = H.SparseMatrix.from_coo(1, 1, [0], [0], [2.0])
    s, _ = H.SolverFactory.make("CG", "JACOBI", A, p)
    x = np.zeros(1)
    assert s.solve(A, np.array([4.0]), x) and abs(x[0] - 2.0) < 1e-10
    D = H.SparseMatrix.from_coo(4, 4, range(4), range(4), [2.0, 3.0, 5.0, 7.0])
    s, _ = H.SolverFactory.make("CG", "JACOBI", D, p)
    x = np.zeros(4)
    s.solve(D, np.array([4.0, 9.0, 15.0, 21.0]), x)
    assert np.allclose(x, [2.0, 3.0, 3.0, 3.0], atol=1e-10)
    A = H.SparseMatrix.poisson_2d(8)
    s, _ = H.SolverFactory.make("CG", "JACOBI", A, p)
    st = H.SolverStats()
    x = np.zeros(64)
    assert s.solve(A, np.zeros(64), x, st) and st.iterations == 0


def test_cg_warm_start_and_max_iter(orc):
    A = P.poisson_2d(32)
    n = 1024
    b = P.rhs(n, 2)
    M = H.SparseMatrix(n, n, *A)
    s, _ = H.SolverFactory.make("CG", "JACOBI", M, default_params(tol=1e-10, max_iter=7))
    x = np.zeros(n)
    st = H.SolverStats()
    assert not s.solve(M, b, x, st)
    assert st.iterations == 7 and not st.converged
    rc, xo, so = orc.solve(0, 1, *A, b, params=default_params(tol=1e-10, max_iter=7))
    assert abs(st.final_residual - so.final_residual) <= 1e-9 * so.final_residual
    s.set_params(default_params(tol=1e-10, max_iter=1000))
    assert s.solve(M, b, x, st)              # warm start from the 7-iteration iterate
    assert st.true_residual < 1e-9


def test_cg_nonfinite_rhs_reports_error():
    A = H.SparseMatrix.poisson_2d(8)
    s, _ = H.SolverFactory.make("CG", "JACOBI", A, default_params())
    b = np.ones(64)
    b[5] = np.nan
    with pytest.raises(H.HamlssError) as e:
        s.solve(A, b, np.zeros(64))
    assert e.value.code == H._abi.ERR_NONFINITE


def test_cg_device_pointers():
    import torch
    A = P.varkappa_poisson_2d(64, 1.0, 5)
    n = 4096
    b = P.rhs(n, 3)
    M = H.SparseMatrix(n, n, *A)
    s, _ = H.SolverFactory.make("CG", "JACOBI", M, default_params(tol=1e-10, max_iter=5000))
    x_h = np.zeros(n)
    st_h = H.SolverStats()
    s.solve(M, b, x_h, st_h)
    db = torch.from_numpy(b).cuda()
    dx = torch.zeros(n, dtype=torch.float64, device="cuda")
    st_d = H.SolverStats()
    s.solve(M, db, dx, st_d)
    assert st_d.iterations == st_h.iterations
    assert np.array_equal(dx.cpu().numpy(), x_h)     # deterministic reductions
