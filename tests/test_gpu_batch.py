"""Batched uneven systems in one persistent launch (-m gpu).

Every system of a batch is checked on its own:
  - converged, with the FP64 true residual ||b - A x|| / ||b|| (computed on the host by
    the oracle's SpMV) at or below the requested tolerance;
  - the solution agrees with the reference's FP64 solve of the same system alone
    (CGSolver + JacobiPreconditioner, or FGMRESSolver + ILUPreconditioner(drop_tol 0))
    to a relative error of 1e-6 (both solves stop at rel-res 1e-10; the systems here have
    condition numbers below 1e4);
  - a system's result is the same alone (a batch of one) and inside the mix: the team
    width is fixed per size class, so the order of every sum is the same and the results
    are identical bit for bit.
Setup faults of one system (zero diagonal) are reported in its own result and do not
stop the others.
"""
import numpy as np
import pytest

from gpu_util import need_gpu
import hsps_b200 as H
from hsps_b200 import batch as B
from hsps_b200 import problems as P
from hsps_b200 import _abi
from hsps_b200._abi import default_params

pytestmark = pytest.mark.gpu

TOL = 1e-10


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    need_gpu()


def mix(count, seed, lo=6, hi=40):
    """Half var-kappa Poisson (CG + Jacobi), half upwind conv-diff (FGMRES + ILU(0))."""
    rng = np.random.default_rng(seed)
    systems, solvers, precs = [], [], []
    for k in range(count):
        s = int(rng.integers(lo, hi + 1))
        if k % 2 == 0:
            systems.append(P.varkappa_poisson_2d(s, 0.5, seed * 1000 + k))
            solvers.append(H.SOLVER_CG)
            precs.append(H.PREC_JACOBI)
        else:
            pe = float(np.exp(rng.uniform(0.0, np.log(100.0))))
            systems.append(P.convection_diffusion_2d(s, 1.0, *P.convdiff_wind(s, pe)))
            solvers.append(H.SOLVER_FGMRES)
            precs.append(H.PREC_ILU)
    return systems, solvers, precs


def params():
    return default_params(tol=TOL, max_iter=4000, restart_size=20, drop_tol=0.0)


def true_rel(orc, A, b, x):
    r = b - orc.spmv(*A, x)
    return np.linalg.norm(r) / np.linalg.norm(b)


def test_batch_mix_matches_reference(orc, ref):
    systems, solvers, precs = mix(24, 1)
    bs = B.BatchSolver(systems, solvers, precs, params())
    rhs = [P.rhs(len(s[0]) - 1, 50 + k) for k, s in enumerate(systems)]
    x, res, tot = bs.solve(rhs)
    xs = bs.split(x)
    pref = default_params(tol=TOL, max_iter=20000, restart_size=20, drop_tol=0.0)
    for k, A in enumerate(systems):
        assert res[k]["status"] == 0 and res[k]["converged"] == 1, (k, res[k])
        rel = true_rel(orc, A, rhs[k], xs[k])
        assert rel <= TOL, (k, rel)
        assert abs(res[k]["final_residual"] - rel) <= 1e-3 * TOL + 1e-6 * rel
        solver = 0 if solvers[k] == H.SOLVER_CG else 1
        prec = 1 if precs[k] == H.PREC_JACOBI else 2
        rc, xr, st = ref.solve(solver, prec, *A, rhs[k], params=pref)
        assert rc == 1 and st.converged          # ref_solve returns solve()'s bool
        err = np.linalg.norm(xs[k] - xr) / np.linalg.norm(xr)
        assert err <= 1e-6, (k, err)
    assert tot.converged == 1
    assert tot.iterations == sum(r["iterations"] for r in res)
    bs.release()


def test_batch_alone_equals_mix():
    systems, solvers, precs = mix(16, 2)
    rhs = [P.rhs(len(s[0]) - 1, 70 + k) for k, s in enumerate(systems)]
    bs = B.BatchSolver(systems, solvers, precs, params())
    x_mix, res_mix, _ = bs.solve(rhs)
    parts = bs.split(x_mix)
    widths = bs.widths()
    bs.release()
    for k in (0, 1, 5, 10):
        one = B.BatchSolver([systems[k]], [solvers[k]], [precs[k]], params())
        one.set_widths(widths)
        x1, r1, _ = one.solve([rhs[k]])
        one.release()
        assert r1[0]["iterations"] == res_mix[k]["iterations"]
        assert np.array_equal(x1, parts[k]), k


def test_batch_uneven_sizes_and_classes(orc):
    # sizes spread over all four size classes (n <= 1024 ... > 16384)
    sides = [4, 31, 33, 64, 65, 128, 130, 7]
    systems = [P.varkappa_poisson_2d(s, 0.5, 5 + i) for i, s in enumerate(sides)]
    rhs = [P.rhs(s * s, 90 + i) for i, s in enumerate(sides)]
    bs = B.BatchSolver(systems, H.SOLVER_CG, H.PREC_JACOBI, params())
    x, res, _ = bs.solve(rhs)
    for k, (A, xk) in enumerate(zip(systems, bs.split(x))):
        assert res[k]["converged"] == 1, (k, res[k])
        assert true_rel(orc, A, rhs[k], xk) <= TOL
    bs.release()


def test_batch_warm_start_and_zero_rhs(orc):
    systems, solvers, precs = mix(6, 3)
    rhs = [P.rhs(len(s[0]) - 1, 11 + k) for k, s in enumerate(systems)]
    rhs[2] = np.zeros_like(rhs[2])
    bs = B.BatchSolver(systems, solvers, precs, params())
    x, res, _ = bs.solve(rhs)
    assert res[2]["converged"] == 1 and res[2]["iterations"] == 0
    assert not np.any(bs.split(x)[2])
    # restarting from the converged solution needs no inner iterations
    x2, res2, _ = bs.solve(rhs, x)
    assert all(r["iterations"] == 0 and r["converged"] == 1 for r in res2)
    bs.release()


def test_batch_zero_diagonal_isolated(orc):
    good = P.poisson_2d(10)
    rp, ci, v = (a.copy() for a in P.poisson_2d(8))
    v[rp[3]:rp[4]][ci[rp[3]:rp[4]] == 3] = 0.0          # zero a_33: Jacobi setup fails
    systems = [good, (rp, ci, v), good]
    rhs = [P.rhs(100, 1), P.rhs(64, 2), P.rhs(100, 3)]
    bs = B.BatchSolver(systems, H.SOLVER_CG, H.PREC_JACOBI, params())
    x, res, _ = bs.solve(rhs)
    assert res[1]["status"] == _abi.ERR_ZERO_DIAG
    for k in (0, 2):
        assert res[k]["status"] == 0 and res[k]["converged"] == 1
        assert true_rel(orc, good, rhs[k], bs.split(x)[k]) <= TOL
    bs.release()


def test_batch_autotune_keeps_results(tmp_path):
    systems, solvers, precs = mix(12, 4, 10, 70)
    rhs = [P.rhs(len(s[0]) - 1, 30 + k) for k, s in enumerate(systems)]
    bs = B.BatchSolver(systems, solvers, precs, params())
    cache = str(tmp_path / "tune.txt")
    w = bs.autotune(rhs, cache)
    assert all(x in (32, 64, 128, 256, 512) for x in w)
    assert bs.widths() == w
    x, res, _ = bs.solve(rhs)
    assert all(r["converged"] == 1 for r in res)
    # a second batch of the same shape reads the cache instead of timing again
    bs2 = B.BatchSolver(systems, solvers, precs, params())
    assert bs2.autotune(rhs, cache) == w
    bs.release()
    bs2.release()
