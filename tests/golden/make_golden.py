"""Generate tests/golden/*.npz from the REFERENCE implementation itself.

Run in a checkout where the reference has been built from its sources
(`make -C oracle ref`, which reads the reference sources in place):

    python tests/golden/make_golden.py

Each fixture stores the inputs (CSR + rhs, generated by hsps_b200.problems from fixed
seeds) and the reference's outputs at OMP_NUM_THREADS=1, so the oracle and the engine can
be checked against the reference on machines where it is not built.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "hybrid-sparse-pde-solver_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle  # noqa: E402
from hsps_b200 import problems as P  # noqa: E402
from hsps_b200._abi import default_params  # noqa: E402


def problems():
    yield "poisson16", P.poisson_2d(16), P.rhs(256, 1)
    yield "varkappa24", P.varkappa_poisson_2d(24, 1.0, 7), P.rhs(576, 2, -1.0, 1.0)
    bx, by = P.convdiff_wind(20, 10.0)
    yield "convdiff20_pe10", P.convection_diffusion_2d(20, 1.0, bx, by), P.rhs(400, 3)
    yield "helmholtz12", P.helmholtz_2d(12, 2.5), P.rhs(144, 4)


def main():
    ref = oracle.Reference(threads=1)
    for name, (rp, ci, v), b in problems():
        out = dict(rp=rp, ci=ci, v=v, b=b)
        m, agg = ref.aggregate(rp, ci, v, 0.25)
        out["agg"] = agg
        hier = ref.amg_hierarchy(rp, ci, v)
        out["amg_levels"] = np.int32(len(hier))
        for l, lev in enumerate(hier):
            for k, (rows, cols, hrp, hci, hv) in lev.items():
                out[f"amg{l}_{k}_shape"] = np.array([rows, cols], np.int32)
                out[f"amg{l}_{k}_rp"], out[f"amg{l}_{k}_ci"], out[f"amg{l}_{k}_v"] = hrp, hci, hv
        rc, lu = ref.ilu0(rp, ci, v)
        out["ilu0"] = lu
        p0 = default_params(drop_tol=0.0)
        for kind, tag in ((1, "jacobi"), (2, "ilu"), (3, "amg")):
            rc, z = ref.precond_apply(kind, rp, ci, v, b, p0)
            out[f"apply_{tag}"] = z
        for solver, prec, tag in ((0, 1, "cg_jacobi"), (1, 2, "fgmres_ilu"), (1, 3, "fgmres_amg"),
                                  (0, 3, "cg_amg"), (1, 1, "fgmres_jacobi")):
            p = default_params(drop_tol=0.0, tol=1e-8, max_iter=1000, restart_size=30)
            rc, x, s = ref.solve(solver, prec, rp, ci, v, b, params=p)
            out[f"{tag}_x"] = x
            out[f"{tag}_stats"] = np.array([rc, s.iterations, s.final_residual, s.restarts,
                                            s.initial_residual], np.float64)
        f, st = ref.features(rp, ci, v)
        out["features"], out["initial_state"] = f, np.int32(st)
        # ILUT factors (ilu.cpp:94-220) at two settings
        for tag, dt, fp in (("ilut_a", 1e-4, 0), ("ilut_b", 1e-3, 5)):
            frp, fci, flu = ref.ilut(rp, ci, v, dt, fp)
            out[f"{tag}_rp"], out[f"{tag}_ci"], out[f"{tag}_v"] = frp, fci, flu
        # PipelinedFGMRESSolver with ILU(0) and with Jacobi
        for prec, tag in ((2, "pfgmres_ilu"), (1, "pfgmres_jacobi")):
            p = default_params(drop_tol=0.0, tol=1e-8, max_iter=1000, restart_size=20)
            rc, x, s = ref.solve(5, prec, rp, ci, v, b, params=p)
            out[f"{tag}_x"] = x
            out[f"{tag}_stats"] = np.array([rc, s.iterations, s.final_residual, s.restarts,
                                            s.flop_count, s.mem_bytes], np.float64)
        # SStepCGSolver(k = 4) on the unit-diagonal scaling D^-1/2 A D^-1/2, and the
        # spectral interval it uses
        rows = np.repeat(np.arange(len(rp) - 1), np.diff(rp))
        dsc = 1.0 / np.sqrt(np.abs(v[ci == rows]))
        vs = v * dsc[rows] * dsc[ci]
        out["unit_v"] = vs
        out["spectral_interval"] = np.array(ref.spectral_interval(rp, ci, vs, 20))
        p = default_params(tol=1e-8, max_iter=400, sstep_k=4)
        rc, x, s = ref.solve(3, 1, rp, ci, vs, b, params=p)
        out["sstep_x"] = x
        out["sstep_stats"] = np.array([rc, s.iterations, s.final_residual, s.comm_bytes, s.sstep_k,
                                       s.flop_count], np.float64)
        # the adaptive ladder under the default drop_tol (ILUT in the MODERATE rung)
        p = default_params(max_iter=5)
        rc, x, s, log = ref.solve_adaptive(rp, ci, v, b, params=p)
        out["ladder_x"] = x
        out["ladder_stats"] = np.array([rc, s.iterations, s.state_used, len(log)], np.float64)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print("wrote", name)


if __name__ == "__main__":
    main()
