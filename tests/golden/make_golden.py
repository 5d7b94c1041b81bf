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
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print("wrote", name)


if __name__ == "__main__":
    main()
