"""Pin the oracle (oracle/oracle.c) before trusting it.

1. The reference's own known-answer tests (tests/test_sparse_matrix.cpp,
   test_preconditioners.cpp, test_solvers.cpp in the reference project), restated.
2. The committed golden fixtures (tests/golden/*.npz, written by the reference itself).
3. Where the reference is built from source here (oracle/_ref), bit-for-bit agreement
   with it on fresh seeded inputs.
CPU only.
"""
import glob
import os

import numpy as np
import pytest

from hsps_b200 import problems as P
from hsps_b200._abi import default_params

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


def coo_csr(rows, r, c, v):
    order = np.lexsort((c, r))
    r, c, v = np.asarray(r)[order], np.asarray(c)[order], np.asarray(v, float)[order]
    rp = np.zeros(rows + 1, np.int32)
    np.add.at(rp, np.asarray(r) + 1, 1)
    return np.cumsum(rp).astype(np.int32), c.astype(np.int32), v


# ------------------------------------------------------------ reference KATs, restated

def test_kat_spmv_identity_and_tridiag(orc):
    # test_sparse_matrix.cpp:28-64
    rp, ci, v = coo_csr(4, range(4), range(4), [1.0] * 4)
    assert np.array_equal(orc.spmv(rp, ci, v, [1.0, 2.0, 3.0, 4.0]), [1.0, 2.0, 3.0, 4.0])
    r, c, vals = [], [], []
    for i in range(4):
        for j, a in ((i - 1, -1.0), (i, 2.0), (i + 1, -1.0)):
            if 0 <= j < 4:
                r.append(i); c.append(j); vals.append(a)
    rp, ci, v = coo_csr(4, r, c, vals)
    assert np.allclose(orc.spmv(rp, ci, v, np.ones(4)), [1.0, 0.0, 0.0, 1.0])


def test_kat_poisson_symmetric_diag4(orc):
    # test_sparse_matrix.cpp:66-78
    rp, ci, v = orc.poisson_2d(8)
    rows = np.repeat(np.arange(64), np.diff(rp))
    dense = np.zeros((64, 64))
    dense[rows, ci] = v
    assert np.array_equal(dense, dense.T)
    assert np.all(np.diag(dense) == 4.0)


def test_kat_convdiff_nonsymmetric(orc):
    # test_sparse_matrix.cpp:113-117
    rp, ci, v = orc.convdiff_2d(8, 0.1, 1.0, 0.5)
    rows = np.repeat(np.arange(64), np.diff(rp))
    dense = np.zeros((64, 64))
    dense[rows, ci] = v
    assert not np.array_equal(dense, dense.T)


def test_kat_cg_1x1_and_diagonal(orc):
    # test_solvers.cpp:42-76
    p = default_params(tol=1e-9, max_iter=3000, restart_size=40)
    rc, x, s = orc.solve(0, 1, [0, 1], [0], [2.0], [4.0], params=p)
    assert rc == 1 and abs(x[0] - 2.0) < 1e-10
    rp, ci, v = coo_csr(4, range(4), range(4), [2.0, 3.0, 5.0, 7.0])
    rc, x, s = orc.solve(0, 1, rp, ci, v, [4.0, 9.0, 15.0, 21.0], params=p)
    assert np.allclose(x, [2.0, 3.0, 3.0, 3.0], atol=1e-10)


def test_kat_cg_zero_rhs_and_poisson(orc):
    # test_solvers.cpp:78-129
    p = default_params(tol=1e-9, max_iter=3000, restart_size=40)
    A = orc.poisson_2d(8)
    rc, x, s = orc.solve(0, 1, *A, np.zeros(64), params=p)
    assert rc == 1 and s.iterations == 0
    A = orc.poisson_2d(16)
    b = np.ones(256)
    rc, x, s = orc.solve(0, 1, *A, b, params=p)
    r = b - orc.spmv(*A, x)
    assert rc == 1 and np.linalg.norm(r) / np.linalg.norm(b) < 1e-8
    rc2, x2, s2 = orc.solve(0, 2, *A, b, params=default_params(tol=1e-9, max_iter=3000, drop_tol=0.0))
    assert s2.iterations < s.iterations


def test_kat_jacobi(orc):
    # test_preconditioners.cpp:26-58
    rp, ci, v = coo_csr(3, range(3), range(3), [2.0, 4.0, 8.0])
    rc, z = orc.precond_apply(1, rp, ci, v, [4.0, 8.0, 16.0])
    assert np.array_equal(z, [2.0, 2.0, 2.0])
    rc, z = orc.precond_apply(1, *orc.poisson_2d(8), np.ones(64))
    assert np.all(z == 0.25)


def test_kat_ilu_diagonal_and_amg_levels(orc):
    # test_preconditioners.cpp:71-122
    rp, ci, v = coo_csr(3, range(3), range(3), [2.0, 4.0, 8.0])
    rc, z = orc.precond_apply(2, rp, ci, v, [2.0, 4.0, 8.0], default_params(drop_tol=0.0))
    assert np.allclose(z, 1.0)
    hier = orc.amg_hierarchy(*orc.poisson_2d(16))
    assert len(hier) >= 2


def test_kat_fgmres_amg_and_convdiff(orc):
    # test_solvers.cpp:195-224
    p = default_params(tol=1e-9, max_iter=3000, restart_size=40)
    A = orc.poisson_2d(16)
    b = np.ones(256)
    rc, x, s = orc.solve(1, 3, *A, b, params=p)
    assert rc == 1
    A = orc.convdiff_2d(12, 0.1, 5.0, 0.0)
    rc, x, s = orc.solve(1, 2, *A, np.ones(144), params=default_params(
        tol=1e-9, max_iter=3000, restart_size=40, drop_tol=0.0))
    assert rc == 1


def test_kat_level_sets(orc):
    # no reference counterpart: the level of row (i, j) of an n x n 5-point grid in natural
    # order is i + j for the lower triangle and (n-1-i) + (n-1-j) for the upper one
    n = 9
    A = orc.poisson_2d(n)
    nl, lev = orc.levels(A[0], A[1], 0)
    ii, jj = np.divmod(np.arange(n * n), n)
    assert nl == 2 * n - 1 and np.array_equal(lev, ii + jj)
    nu, lev = orc.levels(A[0], A[1], 1)
    assert nu == 2 * n - 1 and np.array_equal(lev, (n - 1 - ii) + (n - 1 - jj))


# ------------------------------------------------------------------ golden fixtures

@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_oracle_matches_golden(orc, path):
    g = np.load(path)
    rp, ci, v, b = g["rp"], g["ci"], g["v"], g["b"]
    m, agg = orc.aggregate(rp, ci, v, 0.25)
    assert np.array_equal(agg, g["agg"])
    hier = orc.amg_hierarchy(rp, ci, v)
    assert len(hier) == int(g["amg_levels"])
    for l, lev in enumerate(hier):
        for k, (rows, cols, hrp, hci, hv) in lev.items():
            assert [rows, cols] == list(g[f"amg{l}_{k}_shape"])
            assert np.array_equal(hrp, g[f"amg{l}_{k}_rp"])
            assert np.array_equal(hci, g[f"amg{l}_{k}_ci"])
            assert np.array_equal(hv, g[f"amg{l}_{k}_v"])
    rc, lu = orc.ilu0(rp, ci, v)
    assert np.array_equal(lu, g["ilu0"])
    p0 = default_params(drop_tol=0.0)
    for kind, tag in ((1, "jacobi"), (2, "ilu"), (3, "amg")):
        rc, z = orc.precond_apply(kind, rp, ci, v, b, p0)
        assert np.array_equal(z, g[f"apply_{tag}"])
    for solver, prec, tag in ((0, 1, "cg_jacobi"), (1, 2, "fgmres_ilu"), (1, 3, "fgmres_amg"),
                              (0, 3, "cg_amg"), (1, 1, "fgmres_jacobi")):
        p = default_params(drop_tol=0.0, tol=1e-8, max_iter=1000, restart_size=30)
        rc, x, s = orc.solve(solver, prec, rp, ci, v, b, params=p)
        st = g[f"{tag}_stats"]
        assert rc == int(st[0]) and s.iterations == int(st[1]) and s.restarts == int(st[3])
        assert s.final_residual == st[2] and s.initial_residual == st[4]
        assert np.array_equal(x, g[f"{tag}_x"])
    f, st = orc.features(rp, ci, v)
    assert np.array_equal(f, g["features"]) and st == int(g["initial_state"])
    for tag, dt, fp in (("ilut_a", 1e-4, 0), ("ilut_b", 1e-3, 5)):
        for x, k in zip(orc.ilut(rp, ci, v, dt, fp), ("rp", "ci", "v")):
            assert np.array_equal(x, g[f"{tag}_{k}"]), tag
    for prec, tag in ((2, "pfgmres_ilu"), (1, "pfgmres_jacobi")):
        p = default_params(drop_tol=0.0, tol=1e-8, max_iter=1000, restart_size=20)
        rc, x, s = orc.solve(5, prec, rp, ci, v, b, params=p)
        assert np.array_equal(x, g[f"{tag}_x"])
        assert [rc, s.iterations, s.final_residual, s.restarts, s.flop_count, s.mem_bytes] == \
               list(g[f"{tag}_stats"])
    vs = g["unit_v"]
    assert np.array_equal(np.array(orc.spectral_interval(rp, ci, vs, 20)), g["spectral_interval"])
    rc, x, s = orc.solve(3, 1, rp, ci, vs, b, params=default_params(tol=1e-8, max_iter=400, sstep_k=4))
    assert np.array_equal(x, g["sstep_x"], equal_nan=True)
    assert [rc, s.iterations, s.comm_bytes, s.sstep_k, s.flop_count] == \
           [g["sstep_stats"][k] for k in (0, 1, 3, 4, 5)]
    rc, x, s, log, init = orc.solve_adaptive(rp, ci, v, b, params=default_params(max_iter=5))
    assert np.array_equal(x, g["ladder_x"])
    assert [rc, s.iterations, s.state_used, len(log)] == list(g["ladder_stats"])


def test_generators_match_oracle(orc):
    for n in (1, 3, 16, 33):
        for a, b in zip(P.poisson_2d(n), orc.poisson_2d(n)):
            assert np.array_equal(a, b)
    for n, pe in ((7, 1.0), (20, 10.0), (31, 100.0)):
        bx, by = P.convdiff_wind(n, pe)
        for a, b in zip(P.convection_diffusion_2d(n, 1.0, bx, by), orc.convdiff_2d(n, 1.0, bx, by)):
            assert np.array_equal(a, b)
        for a, b in zip(P.convection_diffusion_2d(n, 0.5, -bx, by), orc.convdiff_2d(n, 0.5, -bx, by)):
            assert np.array_equal(a, b)


# ---------------------------------------------------- live pin against the reference

def _cases():
    yield "poisson24", P.poisson_2d(24)
    yield "varkappa32", P.varkappa_poisson_2d(32, 1.0, 11)
    bx, by = P.convdiff_wind(18, 100.0)
    yield "convdiff18_pe100", P.convection_diffusion_2d(18, 1.0, bx, by)
    yield "helmholtz10", P.helmholtz_2d(10, 7.0)


@pytest.mark.parametrize("name,A", list(_cases()), ids=[c[0] for c in _cases()])
def test_oracle_equals_reference(orc, ref, name, A):
    n = len(A[0]) - 1
    b = P.rhs(n, 5)
    assert np.array_equal(orc.spmv(*A, b), ref.spmv(*A, b))
    assert orc.dot(b, b) == ref.dot(b, b)
    assert np.array_equal(orc.aggregate(*A)[1], ref.aggregate(*A)[1])
    for (l1, l2) in zip(orc.amg_hierarchy(*A), ref.amg_hierarchy(*A)):
        for k in l1:
            for a, c in zip(l1[k][2:], l2[k][2:]):
                assert np.array_equal(a, c)
    assert np.array_equal(orc.ilu0(*A)[1], ref.ilu0(*A)[1])
    for solver, prec in ((0, 1), (1, 2), (1, 3), (0, 0), (1, 0)):
        p = default_params(drop_tol=0.0, tol=1e-8, max_iter=600, restart_size=25)
        r1 = orc.solve(solver, prec, *A, b, params=p)
        r2 = ref.solve(solver, prec, *A, b, params=p)
        assert r1[0] == r2[0] and r1[2].iterations == r2[2].iterations
        assert np.array_equal(r1[1], r2[1])
    f1, s1 = orc.features(*A)
    f2, s2 = ref.features(*A)
    assert np.array_equal(f1, f2) and s1 == s2
    p = default_params(drop_tol=0.0, max_iter=150)
    o = orc.solve_adaptive(*A, b, params=p)
    q = ref.solve_adaptive(*A, b, params=p)
    assert o[0] == q[0] and o[2].iterations == q[2].iterations
    assert [(e.from_state, e.to_state, e.at_iteration) for e in o[3]] == \
           [(e.from_state, e.to_state, e.at_iteration) for e in q[3]]
    assert np.array_equal(o[1], q[1])


def test_reference_from_coo_matches_generators(ref):
    # from_coo sorts by (row, col) and accumulates duplicates (sparse_matrix.cpp:242-282)
    rp, ci, v = ref.from_coo(3, 3, [2, 0, 0, 1, 0], [1, 2, 0, 1, 0], [1.0, 2.0, 3.0, 4.0, 5.0])
    assert list(rp) == [0, 2, 3, 4] and list(ci) == [0, 2, 1, 1] and list(v) == [8.0, 2.0, 4.0, 1.0]


# ------------------------------------------------------------------------ ILUT(tau, p)

ILUT_SETTINGS = [(1e-4, 0), (1e-3, 5), (1e-2, 0), (0.0, 3), (1e-4, 10), (0.3, 1)]


@pytest.mark.parametrize("name,A", list(_cases()), ids=[c[0] for c in _cases()])
def test_oracle_ilut_equals_reference(orc, ref, name, A):
    # setup_ilut (ilu.cpp:94-220), including keep_largest's heap select (ilu.cpp:186-197)
    for dt, fp in ILUT_SETTINGS:
        a, b = orc.ilut(*A, dt, fp), ref.ilut(*A, dt, fp)
        for x, y in zip(a, b):
            assert np.array_equal(x, y), (dt, fp)
    n = len(A[0]) - 1
    b = P.rhs(n, 5)
    # the factory path: drop_tol only, fill_per_row ignored (solver_factory.cpp:73-77)
    for dt, fp in ((1e-4, 0), (1e-3, 5)):
        p = default_params(drop_tol=dt, fill_per_row=fp, tol=1e-8, max_iter=600, restart_size=25)
        r1 = orc.solve(1, 2, *A, b, params=p)
        r2 = ref.solve(1, 2, *A, b, params=p)
        assert r1[0] == r2[0] and r1[2].iterations == r2[2].iterations
        assert np.array_equal(r1[1], r2[1])
        z = orc.precond_apply(2, *A, b, p)[1]
        assert np.array_equal(z, ref.precond_apply(2, *A, b, p)[1])
        assert np.array_equal(z, orc.ilu_apply(*orc.ilut(*A, dt, 0), b)[1])


def test_oracle_ladder_through_ilut_equals_reference(orc, ref):
    # CG+Jacobi cannot converge in 5 iterations: the ladder escalates to MODERATE, whose
    # ILU is ILUT(1e-4, 0) under the default drop_tol, then to HARD
    A = P.poisson_2d(16)
    b = np.ones(256)
    p = default_params(max_iter=5)
    o = orc.solve_adaptive(*A, b, params=p)
    q = ref.solve_adaptive(*A, b, params=p)
    assert o[0] == q[0] == 1 and o[2].iterations == q[2].iterations
    assert [(e.from_state, e.to_state, e.at_iteration) for e in o[3]] == \
           [(e.from_state, e.to_state, e.at_iteration) for e in q[3]] == [(0, 1, 5), (1, 2, 5)]
    assert np.array_equal(o[1], q[1])


def test_kat_ilut(orc):
    # test_improvements.cpp:49-114, restated on the oracle
    A = P.poisson_2d(10)
    b = np.ones(100)
    z0 = orc.precond_apply(2, *A, b, default_params(drop_tol=0.0, fill_per_row=0))[1]
    z1 = orc.precond_apply(2, *A, b, default_params(drop_tol=0.0, fill_per_row=0))[1]
    assert np.allclose(z0, z1, rtol=0, atol=1e-12)           # ILUT(0, 0) is ILU(0)
    C = P.convection_diffusion_2d(10, 0.1, 3.0, 0.0)
    for dt in (0.0, 1e-3):
        rc, z = orc.precond_apply(2, *C, np.ones(100), default_params(drop_tol=dt, fill_per_row=0))
        assert rc == 0 and np.linalg.norm(z) > 0
    C = P.convection_diffusion_2d(12, 0.1, 8.0, 0.0)
    rc, z = orc.ilu_apply(*orc.ilut(*C, 1e-4, 5), np.ones(144))
    assert rc == 0 and np.all(np.isfinite(z)) and np.linalg.norm(z) > 0


def test_ilut_capacity_fixture(orc):
    # an empty row keeps its diagonal shift; a row whose L / U exceed orig + fill is cut to
    # the largest magnitudes, kept in column order
    rp, ci, v = coo_csr(4, [0, 0, 1, 1, 2, 2, 2, 3], [0, 1, 0, 1, 0, 1, 2, 3],
                        [4.0, 1.0, 1.0, 4.0, 1.0, -3.0, 5.0, 2.0])
    frp, fci, flu = orc.ilut(rp, ci, v, 1e-6, 0)
    assert list(frp[1:] - frp[:-1]) == [2, 2, 3, 1]
    rp2 = np.array([0, 1, 1, 2], np.int32)
    frp2, fci2, flu2 = orc.ilut(rp2, np.array([0, 2], np.int32), np.array([2.0, 3.0]), 1e-4, 0)
    assert list(fci2) == [0, 1, 2] and flu2[1] == 2.220446049250313e-16 * 1e6


# ------------------------------------------------ s-step CG and pipelined FGMRES

def _unit_diagonal(A):
    """D^-1/2 A D^-1/2: the scaling under which the reference's s-step update converges."""
    rp, ci, v = A
    n = len(rp) - 1
    rows = np.repeat(np.arange(n), np.diff(rp))
    s = 1.0 / np.sqrt(v[ci == rows])
    return rp, ci, v * s[rows] * s[ci]


def _sstep_cases():
    for name, A in _cases():
        yield name, A
        yield "unit_" + name, _unit_diagonal(A)


@pytest.mark.parametrize("name,A", list(_sstep_cases()), ids=[c[0] for c in _sstep_cases()])
def test_oracle_sstep_and_pipelined_equal_reference(orc, ref, name, A):
    # spectral_interval (sparse_matrix.cpp:451-479), SStepCGSolver (sstep_cg_solver.cpp:
    # 170-305) -- divergent runs included, NaN for NaN -- and PipelinedFGMRESSolver
    # (pipelined_fgmres_solver.cpp:69-242), bit for bit
    assert orc.spectral_interval(*A) == ref.spectral_interval(*A)
    n = len(A[0]) - 1
    b = P.rhs(n, 3)
    for k in (1, 2, 4, 8):
        p = default_params(tol=1e-8, max_iter=400, sstep_k=k)
        o, r = orc.solve(3, 1, *A, b, params=p), ref.solve(3, 1, *A, b, params=p)
        assert o[0] == r[0] and o[2].iterations == r[2].iterations
        assert np.array_equal(o[1], r[1], equal_nan=True)
        assert (o[2].flop_count, o[2].mem_bytes, o[2].comm_bytes, o[2].sstep_k) == \
               (r[2].flop_count, r[2].mem_bytes, r[2].comm_bytes, r[2].sstep_k)
    for prec in (0, 1, 2):
        p = default_params(tol=1e-8, max_iter=400, restart_size=20, drop_tol=0.0)
        o, r = orc.solve(5, prec, *A, b, params=p), ref.solve(5, prec, *A, b, params=p)
        assert o[0] == r[0] and o[2].iterations == r[2].iterations and o[2].restarts == r[2].restarts
        assert np.array_equal(o[1], r[1])
        assert (o[2].flop_count, o[2].mem_bytes) == (r[2].flop_count, r[2].mem_bytes)


def test_kat_pipelined_fgmres(orc):
    # test_improvements.cpp:240-290, restated on the oracle
    p = default_params(tol=1e-8, max_iter=3000, restart_size=50, drop_tol=0.0)
    A = P.poisson_2d(16)
    rc, x, st = orc.solve(5, 2, *A, np.ones(256), params=p)
    assert rc == 1 and np.linalg.norm(np.ones(256) - orc.spmv(*A, x)) / 16.0 < 1e-7
    A = P.poisson_2d(12)
    x_std = orc.solve(1, 2, *A, np.ones(144), params=p)[1]
    x_pip = orc.solve(5, 2, *A, np.ones(144), params=p)[1]
    assert np.linalg.norm(x_std - x_pip) / np.linalg.norm(x_std) < 1e-5
    C = P.convection_diffusion_2d(10, 0.1, 5.0, 0.0)
    assert orc.solve(5, 2, *C, np.ones(100), params=p)[0] == 1


def test_oracle_pipelined_lucky_breakdown_equals_reference(orc, ref):
    # b along an eigenvector: h_10 = 0 exactly; the pipelined cycle leaves before rotating
    # that column and restarts once (pipelined_fgmres_solver.cpp:117-123)
    A = (np.arange(5, dtype=np.int32), np.arange(4, dtype=np.int32), np.array([2.0, 3.0, 5.0, 7.0]))
    b = np.array([2.0, 0.0, 0.0, 0.0])
    p = default_params(tol=1e-10, max_iter=50, restart_size=4, drop_tol=0.0)
    o, r = orc.solve(5, 0, *A, b, params=p), ref.solve(5, 0, *A, b, params=p)
    assert (o[2].converged, o[2].iterations, o[2].restarts) == (r[2].converged, r[2].iterations,
                                                                 r[2].restarts) == (1, 1, 1)
    assert np.array_equal(o[1], r[1])
    s = orc.solve(1, 0, *A, b, params=p)[2]
    assert (s.iterations, s.restarts) == (1, 0)


def ilut_edge_cases():
    """ILUT corner cases: an empty row, tiny diagonals under large off-diagonals (the fill
    limit can drop a diagonal, and later rows then skip that pivot), and equal magnitudes
    (the heap select's tie order)."""
    rng = np.random.default_rng(5)
    n, r, c, v = 40, [], [], []
    for i in range(n):
        r.append(i); c.append(i); v.append(1e-3 if i % 3 == 0 else 4.0)
        for j in rng.choice(n, 6, replace=False):
            if j != i:
                r.append(i); c.append(int(j)); v.append(float(rng.choice([-1.0, 1.0, 2.0])))
    yield "empty_row", coo_csr(4, [0, 0, 1, 1, 3, 3], [0, 3, 0, 1, 1, 3], [4.0, 1.0, 1.0, 4.0, 2.0, 5.0])
    yield "small_diag", coo_csr(n, r, c, v)
    yield "poisson_ties", P.poisson_2d(12)


ILUT_EDGE_SETTINGS = [(1e-4, 0), (1e3, 0), (1e-2, 2), (1e-8, 20), (0.5, 0)]


@pytest.mark.parametrize("name,A", list(ilut_edge_cases()), ids=[c[0] for c in ilut_edge_cases()])
def test_oracle_ilut_edge_cases_equal_reference(orc, ref, name, A):
    for dt, fp in ILUT_EDGE_SETTINGS:
        for x, y in zip(orc.ilut(*A, dt, fp), ref.ilut(*A, dt, fp)):
            assert np.array_equal(x, y), (dt, fp)


AMG_VARIANTS = [dict(amg_levels=3), dict(amg_strong=0.5), dict(amg_strong=0.08),
                dict(amg_smooth_pre=1, amg_smooth_post=3)]


@pytest.mark.parametrize("over", AMG_VARIANTS, ids=[",".join(f"{k}={v}" for k, v in o.items()) for o in AMG_VARIANTS])
def test_oracle_amg_parameters_equal_reference(orc, ref, over):
    # the factory forwards amg_levels, amg_strong and the pre/post sweep counts
    # (solver_factory.cpp:80-88): hierarchy and V-cycle bit for bit under each
    A = P.varkappa_poisson_2d(28, 1.0, 13)
    p = default_params(**over)
    for l1, l2 in zip(orc.amg_hierarchy(*A, params=p), ref.amg_hierarchy(*A, params=p)):
        for k in l1:
            for a, b in zip(l1[k][2:], l2[k][2:]):
                assert np.array_equal(a, b), k
    r = P.rhs(28 * 28, 3, -1.0, 1.0)
    assert np.array_equal(orc.precond_apply(3, *A, r, p)[1], ref.precond_apply(3, *A, r, p)[1])
