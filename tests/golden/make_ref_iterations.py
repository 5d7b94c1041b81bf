"""Iteration count of the reference's own complete solve of the benchmark system.

The 2048^2 variable-coefficient Poisson system of bench.py (sigma 1, rhs U[-1, 1), seed
1000) solved to 1e-10 by the reference's only path at that size, CGSolver +
JacobiPreconditioner (its AMG cannot be set up above 240^2: amg.cpp:113), built from its
sources with its release flags (oracle/_ref/libhsps_ref_fast.so) and run on every host
thread.  The count is what the CPU baseline's bounded sample is scaled by; the complete
solve's own wall time is recorded beside it.

    python tests/golden/make_ref_iterations.py   # writes tests/golden/ref_cg_jacobi_2048.json
"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "hybrid-sparse-pde-solver_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def main():
    import oracle
    from hsps_b200 import problems as P
    from hsps_b200._abi import default_params

    side, sigma, seed, tol = 2048, 1.0, 1000, 1e-10
    rp, ci, v = P.varkappa_poisson_2d(side, sigma, seed)
    b = P.rhs(len(rp) - 1, seed, -1.0, 1.0)
    threads = len(os.sched_getaffinity(0))
    R = oracle.Reference(fast=True, threads=threads)
    p = default_params(tol=tol, max_iter=100000)
    t0 = time.perf_counter()
    rc, x, st = R.solve(0, 1, rp, ci, v, b, params=p)
    wall = time.perf_counter() - t0
    out = {"problem": f"var-kappa Poisson {side}^2, sigma {sigma}, rhs U[-1,1), seed {seed}",
           "solver": "reference CGSolver + JacobiPreconditioner (release build)",
           "tol": tol, "iterations": int(st.iterations), "converged": bool(st.converged),
           "final_residual": float(st.final_residual), "threads": threads,
           "wall_s": round(wall, 2)}
    path = os.path.join(HERE, f"ref_cg_jacobi_{side}.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")
    print(json.dumps(out))


if __name__ == "__main__":
    main()
