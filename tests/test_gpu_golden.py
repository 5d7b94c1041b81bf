"""The device against the committed golden fixtures (tests/golden/*.npz), which hold the
reference's own outputs (written by tests/golden/make_golden.py from the reference built
from its sources) -- so the GPU box, where the reference is not built, still checks the
engine against the reference directly (-m gpu).

Bars: AMG hierarchies, ILU(0) factors, Jacobi / ILU / AMG applies and ILUT factors bit for
bit; Krylov solves within +-1 iteration of the reference with the same outcome and a
solution within 1e-5 (relative, max norm); s-step CG (k = 4, unit-diagonal scaling) with
the same outcome and trip count within one batch; the adaptive ladder under the default
drop_tol with the same final state and escalation count.
"""
import glob
import os

import numpy as np
import pytest

from gpu_util import need_gpu
import hsps_b200 as H
from hsps_b200._abi import default_params

pytestmark = pytest.mark.gpu

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))
IDS = [os.path.basename(p)[:-4] for p in GOLDEN]


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    need_gpu()


def mat(g, v=None):
    n = len(g["rp"]) - 1
    return H.SparseMatrix(n, n, g["rp"], g["ci"], g["v"] if v is None else v)


def close(x, y, rel=1e-5):
    return np.max(np.abs(x - y)) <= rel * max(np.max(np.abs(y)), 1e-300)


@pytest.mark.parametrize("path", GOLDEN, ids=IDS)
def test_factors_and_applies_bitwise(path):
    g = np.load(path)
    M = mat(g)
    A = H.AMGPreconditioner()
    A.setup(M)
    assert A.levels() == int(g["amg_levels"])
    for l in range(A.levels()):
        for which, k in ((0, "A"), (1, "P"), (2, "R")):
            if f"amg{l}_{k}_rp" not in g.files or (k != "A" and l == A.levels() - 1):
                continue
            rows, cols, rp, ci, v = A.level_matrix(l, which)
            assert [rows, cols] == list(g[f"amg{l}_{k}_shape"])
            assert np.array_equal(rp, g[f"amg{l}_{k}_rp"]) and np.array_equal(ci, g[f"amg{l}_{k}_ci"])
            assert np.array_equal(v, g[f"amg{l}_{k}_v"]), (l, k)
    I = H.ILUPreconditioner()
    I.setup(M)
    assert np.array_equal(I.factors(), g["ilu0"])
    J = H.JacobiPreconditioner()
    J.setup(M)
    for P_, tag in ((J, "jacobi"), (I, "ilu"), (A, "amg")):
        assert np.array_equal(P_.apply(g["b"]), g[f"apply_{tag}"]), tag
    for tag, dt, fp in (("ilut_a", 1e-4, 0), ("ilut_b", 1e-3, 5)):
        T = H.ILUPreconditioner()
        T.set_drop_tol(dt)
        T.set_fill_per_row(fp)
        T.setup(M)
        for x, k in zip(T.factor_csr(), ("rp", "ci", "v")):
            assert np.array_equal(x, g[f"{tag}_{k}"]), (tag, k)


@pytest.mark.parametrize("path", GOLDEN, ids=IDS)
def test_solves_against_reference(path):
    g = np.load(path)
    b = g["b"]
    M = mat(g)
    n = len(b)
    cases = [(H.SOLVER_CG, H.PREC_JACOBI, "cg_jacobi", 30), (H.SOLVER_FGMRES, H.PREC_ILU, "fgmres_ilu", 30),
             (H.SOLVER_FGMRES, H.PREC_AMG, "fgmres_amg", 30), (H.SOLVER_CG, H.PREC_AMG, "cg_amg", 30),
             (H.SOLVER_FGMRES, H.PREC_JACOBI, "fgmres_jacobi", 30),
             (H._abi.SOLVER_PIPELINED_FGMRES, H.PREC_ILU, "pfgmres_ilu", 20),
             (H._abi.SOLVER_PIPELINED_FGMRES, H.PREC_JACOBI, "pfgmres_jacobi", 20)]
    classes = {H.SOLVER_CG: H.CGSolver, H.SOLVER_FGMRES: H.FGMRESSolver,
               H._abi.SOLVER_PIPELINED_FGMRES: H.PipelinedFGMRESSolver}
    for solver, prec, tag, m in cases:
        p = default_params(drop_tol=0.0, tol=1e-8, max_iter=1000, restart_size=m)
        s = classes[solver]()
        s.set_params(p)
        s.set_preconditioner(H.SolverFactory.make_precond(prec, M, p))
        x = np.zeros(n)
        st = H.SolverStats()
        ok = s.solve(M, b, x, st)
        ref = g[f"{tag}_stats"]
        assert ok == bool(ref[0]), tag
        assert abs(st.iterations - int(ref[1])) <= 1, (tag, st.iterations, int(ref[1]))
        if ok:
            assert close(x, g[f"{tag}_x"]), tag


@pytest.mark.parametrize("path", GOLDEN, ids=IDS)
def test_sstep_and_ladder_against_reference(path):
    g = np.load(path)
    b = g["b"]
    n = len(b)
    M = mat(g, g["unit_v"])
    s = H.SStepCGSolver(4)
    s.set_params(default_params(tol=1e-8, max_iter=400, sstep_k=4))
    x = np.zeros(n)
    st = H.SolverStats()
    ok = s.solve(M, b, x, st)
    ref = g["sstep_stats"]
    assert ok == bool(ref[0]) and st.sstep_k == int(ref[4])
    if ok:
        assert abs(st.iterations - int(ref[1])) <= 4
        assert close(x, g["sstep_x"], 1e-4)
    sel = H.AdaptiveSelector(default_params(max_iter=5))
    x = np.zeros(n)
    st = H.SolverStats()
    ok = sel.solve(mat(g), b, x, st)
    ref = g["ladder_stats"]
    assert ok == bool(ref[0]) and st.state_used == int(ref[2]) and len(sel.escalation_log()) == int(ref[3])
    assert abs(st.iterations - int(ref[1])) <= 1
    if ok:
        assert close(x, g["ladder_x"])
