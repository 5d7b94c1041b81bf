#!/usr/bin/env python
"""Headline benchmark: solves/s of the variable-coefficient 2-D Poisson problem.

Workload (one "step" = one complete solve of one system, preconditioner setup included):
  -div(kappa grad u) = f, 5-point, 2048 x 2048 interior grid (n = 4,194,304,
  nnz = 20,963,328), kappa lognormal (sigma = 1) per cell with harmonic face averages,
  rhs uniform [-1, 1) from the seed, x0 = 0, solved to 1e-10 relative residual.
  Inputs are synthetic (seeded); the matrix (335 MB in FP64) is larger than L2 (126 MB),
  so no L2 flush is needed between steps.

  value : solves/s with the matrix and rhs resident in HBM (device pointers), per-step
          device time from CUDA events on the engine's stream; whole-job aggregate over
          all ranks (each rank solves its own seeded instance: weak scaling, no collective
          on the data path).
  e2e   : the same solve through the public C ABI with HOST buffers -- upload of the CSR
          and rhs from pinned host memory, setup, solve, download of x -- all timed.

--impl reference times the reference's own CPU implementation (built from its sources
by oracle/Makefile into oracle/_ref/) on the host cores, on the same problem.
"""
import argparse
import atexit
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "hybrid-sparse-pde-solver_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

_T0 = time.perf_counter()


def log(msg):
    """Progress on stderr (the JSON result alone goes to stdout)."""
    print(f"[bench {time.perf_counter() - _T0:8.1f}s] {msg}", file=sys.stderr, flush=True)


N_SIDE = 2048
SIGMA = 1.0
TOL = 1e-10
# SA-AMG hierarchy: theta 0.25, omega 2/3, coarsest level dense at <= 512 rows -- or at the
# first level that keeps more than 75% of its rows (the reference's aggregation stalls on
# the dense coarse operators of this problem; stalled levels cost much and help little)
STALL = 0.75
METRIC = "solves/sec at 1e-10 rel-res (var-kappa Poisson 2048^2)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--solver", default="auto",
                    choices=["auto", "cg_jacobi", "amg_fp64", "amg_mixed"])
    ap.add_argument("--n-side", type=int, default=N_SIDE)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-same-algorithm", action="store_true",
                    help="skip the device vs reference AMG-PCG side measurement at 240^2")
    ap.add_argument("--no-coarse512", action="store_true",
                    help="skip the coarsest <= 512 (no stall cut) hierarchy side measurement")
    ap.add_argument("--cpu-sample-iters", type=int, default=40)
    ap.add_argument("--serving-requests", type=int, default=200,
                    help="requests in the serving stream (0 skips the serving measurement)")
    ap.add_argument("--serving-n-max", type=float, default=2.6e5)
    ap.add_argument("--serving-full", type=int, default=0,
                    help="requests of the full serving size range (1e3..4.2e6 rows); 0 skips")
    ap.add_argument("--serving-rate", type=float, default=2.0,
                    help="Poisson arrival rate of the full-range serving stream (requests/s)")
    ap.add_argument("--serving-ref-sample", type=int, default=40,
                    help="requests of the full-range stream the reference replays")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the C1 / C2 latency side measurement")
    ap.add_argument("--no-batch", action="store_true",
                    help="skip the batched-systems side measurement (4096 uneven systems)")
    ap.add_argument("--batch-count", type=int, default=4096)
    ap.add_argument("--no-variants", action="store_true",
                    help="skip the Krylov-variant side measurement (s-step CG, pipelined FGMRES)")
    ap.add_argument("--no-ilut", action="store_true",
                    help="skip the ILUT side measurement (device vs reference setup_ilut)")
    ap.add_argument("--profile-step", action="store_true",
                    help="run the warm-up, then ONE step between cudaProfilerStart/Stop and exit "
                         "(for ncu --profile-from-start off); prints no result line")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def problem(n_side, seed):
    from hsps_b200 import problems as P

    rp, ci, v = P.varkappa_poisson_2d(n_side, SIGMA, seed)
    b = P.rhs(len(rp) - 1, seed, -1.0, 1.0)
    return rp, ci, v, b


# ------------------------------------------------------------- replicas over ranks
def max_over_ranks(v, device):
    """The largest of every rank's `v` (the slowest replica sets the job's time).  Every
    rank must call it the same number of times; with one process it returns `v`."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(v)
    t = torch.tensor([float(v)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(steps_per_rank, world, max_ms):
    """Whole-job solves/s: every rank solved `steps_per_rank` systems of its own (weak
    scaling, no collective on the data path) within the slowest rank's time."""
    return world * steps_per_rank / (max_ms / 1e3)


def replica_seed(rank):
    """Each rank solves its own seeded instance of the workload."""
    return 1000 + rank


# ----------------------------------------------------------------- clocks sampling
class Clocks:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        """Start sampling.  On a fresh machine the first nvidia-smi call initialises the
        management library, which takes about a second and disturbs the GPU meanwhile, so
        the sampler is started ahead of the warm-up and `ready` waits for its first row;
        `mark` then keeps only the rows sampled from the timed region on."""
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, FileNotFoundError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def ready(self, timeout=10.0):
        t0 = time.time()
        while self.proc and not self.rows and time.time() - t0 < timeout:
            time.sleep(0.05)

    def mark(self):
        self.rows = []

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4)
                          if r[5 + k].lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def launches_of_one_step(step):
    """Kernel launches of one step, counted live by the CUDA activity profiler
    (torch.profiler over CUPTI, which sees every kernel of the process): (engine kernels --
    every kernel of the engine lives in namespace hamlss --, other kernels by name, e.g. the
    benchmark's own torch fills).  None when the profiler yields nothing."""
    import torch
    from torch.autograd import DeviceType
    from torch.profiler import ProfilerActivity, profile

    try:
        torch.cuda.synchronize()
        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            step()
            torch.cuda.synchronize()
        own, lib = 0, {}
        for e in prof.events():
            if e.device_type != DeviceType.CUDA:
                continue
            name = e.name
            low = name.lower()
            if low.startswith(("memcpy", "memset")):
                continue
            if "hamlss" in name:
                own += 1
            else:
                lib[name] = lib.get(name, 0) + 1
        if own == 0 and not lib:
            return None
        return own, lib
    except Exception as exc:         # profiler unavailable: report the op count instead
        log(f"launch count: activity profiler unavailable ({exc})")
        return None


def ncu_traffic(kernel_family):
    """DRAM bytes per launch of the family's largest launch, from the committed ncu
    summary (profiles/traffic.json): (bytes, which launch, its algorithmic bytes)."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(path):
        return None, None, None
    try:
        d = json.load(open(path)).get(kernel_family, {})
        return (d.get("dram_bytes_per_launch"), d.get("launch"),
                d.get("algorithmic_bytes_per_launch"))
    except (ValueError, OSError):
        return None, None, None


# ------------------------------------------------------------------ CPU reference
def reference_cpu_sample(rp, ci, v, b, iters, threads):
    """Time `iters` CG+Jacobi iterations of the reference (release build) on the host.

    The reference's AMG cannot be set up at this size (its smoothed prolongation uses a
    dense n_fine x n_coarse buffer), so its full-size path for this problem is
    CGSolver + JacobiPreconditioner (SolverFactory::make(CG, JACOBI)).
    """
    import oracle
    from hsps_b200._abi import default_params

    R = oracle.Reference(fast=True, threads=threads)
    p = default_params(tol=TOL, max_iter=iters)
    t0 = time.perf_counter()
    rc, x, st = R.solve(0, 1, rp, ci, v, b, params=p)
    dt = time.perf_counter() - t0
    return dt, st.iterations


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# --------------------------------------------------------------------- our engine
def solver_choice(name):
    import hsps_b200 as H

    if name != "auto":
        return name
    try:
        A = H.SparseMatrix.poisson_2d(8)
        M = H.AMGPreconditioner()
        M.setup(A)
        return "amg_mixed"
    except Exception:
        return "cg_jacobi"


def make_params(solver):
    import hsps_b200 as H

    if solver == "cg_jacobi":
        return H.SolverParams(tol=TOL, max_iter=100000), H.SOLVER_CG, H.PREC_JACOBI
    prec = 0 if solver == "amg_fp64" else 1
    p = H.SolverParams(tol=TOL, max_iter=1000, precision=prec, amg_omega=2.0 / 3.0,
                       amg_coarse_limit=512, amg_levels=25, amg_stall_ratio=STALL)
    return p, H.SOLVER_CG, H.PREC_AMG


def workload_name(n_side, solver, hierarchy):
    base = f"var-kappa Poisson {n_side}^2 5-point, sigma={SIGMA}, rtol {TOL}"
    if solver == "cg_jacobi":
        return base + ", PCG + Jacobi (FP64)"
    prec = "FP32 V-cycle, FP64 refinement" if solver == "amg_mixed" else "FP64"
    cut = ""
    if hierarchy:
        cut = (f", {hierarchy['levels']} levels, coarsest {hierarchy['coarsest_rows']} rows dense "
               f"(hierarchy cut at the first level keeping > {int(STALL * 100)}% of its rows; "
               f"<= 512 otherwise)")
    return base + f", PCG + SA-AMG (theta 0.25, omega 2/3{cut}), {prec}"


def amg_config(solver, hierarchy):
    if solver == "cg_jacobi":
        return None
    out = {"theta": 0.25, "omega": 2.0 / 3.0, "coarse_limit": 512, "max_levels": 25,
           "stall_ratio": STALL, "smooth_pre": 2, "smooth_post": 2}
    if hierarchy:
        out.update(hierarchy)
    return out


def run_ours(args, rank, world, local):
    import ctypes as C

    import torch

    import hsps_b200 as H
    from hsps_b200 import _abi

    torch.cuda.set_device(local)
    ctx = H.Context(local)
    L = _abi.lib()
    solver = solver_choice(args.solver)
    params, stype, ptype = make_params(solver)
    log(f"solver {solver}; generating the {args.n_side}^2 system")
    rp, ci, v, b = problem(args.n_side, replica_seed(rank))
    log(f"n={len(rp) - 1} nnz={len(v)}; uploading")
    n, nnz = len(rp) - 1, len(v)
    A = H.SparseMatrix(n, n, rp, ci, v, ctx)
    db = torch.from_numpy(b).cuda()
    dx = torch.zeros(n, dtype=torch.float64, device="cuda")
    stream = torch.cuda.ExternalStream(ctx.stream())

    def one_solve():
        dx.zero_()
        torch.cuda.synchronize()
        h = C.c_void_p()
        if ptype != H.PREC_NONE:
            rc = L.hamlss_precond_setup(ctx.h, A.h, ptype, C.byref(params), C.byref(h), None)
            if rc:
                raise RuntimeError(L.hamlss_last_error())
        st = _abi.Stats()
        rc = L.hamlss_solve(ctx.h, stype, A.h, h, C.c_void_p(db.data_ptr()),
                            C.c_void_p(dx.data_ptr()), H.DEVICE, C.byref(params), C.byref(st))
        if rc:
            raise RuntimeError(L.hamlss_last_error())
        if h:
            L.hamlss_precond_release(h)
        return st

    clocks = Clocks(local)
    if not args.profile_step:
        clocks.start()                  # its start-up cost stays out of the timed region
        atexit.register(clocks.stop)    # no sampler left running if a warm-up step fails
    for _ in range(args.warmup):
        st = one_solve()
        log(f"warm-up solve: {st.iterations} iterations, {st.outer_iterations} outer, "
            f"true rel {st.true_residual:.2e}, {st.solve_time_s:.3f} s")
    if not st.converged or st.true_residual > 1.5 * TOL:
        raise RuntimeError(f"warm-up solve did not reach tolerance: {st.as_dict()}")
    if args.profile_step:
        # one step between cudaProfilerStart / Stop, for `ncu --profile-from-start off`
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        st = one_solve()
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        log(f"profiled step: {st.iterations} iterations, true rel {st.true_residual:.2e}")
        return None, None

    # ---- timed region: device-resident inputs
    clocks.ready()
    dist = world > 1
    if dist:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clocks.mark()
    L.hamlss_profile_enable(ctx.h, 1, 2_000_000)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    iters, true_res = [], []
    for _ in range(args.steps):
        st = one_solve()
        iters.append(st.iterations)
        true_res.append(st.true_residual)
    ev1.record(stream)
    torch.cuda.synchronize()
    dev_ms = ev0.elapsed_time(ev1)
    log(f"timed {args.steps} solves: {dev_ms:.1f} ms")
    cap = 64
    names = C.create_string_buffer(32 * cap)
    launches = (C.c_int32 * cap)()
    tms = (C.c_double * cap)()
    tby = (C.c_double * cap)()
    cnt = C.c_int32()
    L.hamlss_profile_read(ctx.h, cap, names, launches, tms, tby, C.byref(cnt))
    L.hamlss_profile_enable(ctx.h, 0, 0)
    clocks.stop()
    fams = []
    for i in range(cnt.value):
        nm = names.raw[32 * i:32 * i + 32].split(b"\0")[0].decode()
        fams.append((nm, launches[i], tms[i], tby[i]))
    total_launches = sum(f[1] for f in fams)
    max_ms = max_over_ranks(dev_ms, "cuda")
    value = replica_throughput(args.steps, world, max_ms)
    # kernel launches of one more (identical) step, counted by the activity profiler
    counted = launches_of_one_step(one_solve)
    if counted is not None:
        log(f"one step launches {counted[0]} engine kernels and "
            f"{sum(counted[1].values())} other kernels")

    # ---- solve phase alone, hierarchy resident: mixed precision against all-FP64 on the
    #      same AMG hierarchy (the two arithmetic schemes compared on equal terms)
    solve_only = None
    hierarchy = None
    if ptype == H.PREC_AMG:
        h = C.c_void_p()
        rc = L.hamlss_precond_setup(ctx.h, A.h, ptype, C.byref(params), C.byref(h), None)
        if rc:
            raise RuntimeError(L.hamlss_last_error())
        p64 = _abi.Params.from_buffer_copy(params)
        p64.precision = 0
        nlev = C.c_int32()
        L.hamlss_amg_num_levels(h, C.byref(nlev))
        level_rows = []
        for lv in range(nlev.value):
            r_, c_, z_ = C.c_int32(), C.c_int32(), C.c_int32()
            L.hamlss_amg_level_matrix(h, lv, 0, C.byref(r_), C.byref(c_), C.byref(z_),
                                      None, None, None)
            level_rows.append((r_.value, z_.value))
        hierarchy = {"levels": nlev.value, "rows": [r for r, _ in level_rows],
                     "nnz": [z for _, z in level_rows], "coarsest_rows": level_rows[-1][0]}

        def timed_solves(pp, k):
            its = []
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            for _ in range(k):
                dx.zero_()
                st = _abi.Stats()
                rc = L.hamlss_solve(ctx.h, stype, A.h, h, C.c_void_p(db.data_ptr()),
                                    C.c_void_p(dx.data_ptr()), H.DEVICE, C.byref(pp), C.byref(st))
                if rc or not st.converged:
                    raise RuntimeError(f"solve-only run failed: {L.hamlss_last_error()}")
                its.append(st.iterations)
            e1.record(stream)
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) / k, int(np.median(its))

        timed_solves(params, 1)
        timed_solves(p64, 1)
        k = max(3, args.steps)
        mixed_ms, mixed_it = timed_solves(params, k)
        fp64_ms, fp64_it = timed_solves(p64, k)
        L.hamlss_precond_release(h)
        setup_ms = max_ms / args.steps - mixed_ms
        solve_only = {"mixed_ms": round(mixed_ms, 3), "mixed_iterations": mixed_it,
                      "fp64_ms": round(fp64_ms, 3), "fp64_iterations": fp64_it,
                      "speedup_mixed_vs_fp64": round(fp64_ms / mixed_ms, 3),
                      "step_speedup_with_setup": round((setup_ms + fp64_ms) / (setup_ms + mixed_ms), 3),
                      "note": "hierarchy set up once and kept resident; both arithmetic schemes "
                              "use the same hierarchy; x0 = 0 each solve"}
        log(f"solve only: mixed {mixed_ms:.1f} ms ({mixed_it} it), fp64 {fp64_ms:.1f} ms ({fp64_it} it)")

    # ---- end to end through the C ABI with host buffers (pinned)
    hb = torch.from_numpy(b).pin_memory()
    hx = torch.zeros(n, dtype=torch.float64).pin_memory()
    hrp = torch.from_numpy(rp).pin_memory()
    hci = torch.from_numpy(ci).pin_memory()
    hv = torch.from_numpy(v).pin_memory()

    def e2e_step():
        hx.zero_()
        mh = C.c_void_p()
        rc = L.hamlss_mat_upload(ctx.h, n, n, nnz, C.c_void_p(hrp.data_ptr()),
                                 C.c_void_p(hci.data_ptr()), C.c_void_p(hv.data_ptr()), H.HOST,
                                 C.byref(mh))
        if rc:
            raise RuntimeError(L.hamlss_last_error())
        ph = C.c_void_p()
        if ptype != H.PREC_NONE:
            L.hamlss_precond_setup(ctx.h, mh, ptype, C.byref(params), C.byref(ph), None)
        st = _abi.Stats()
        rc = L.hamlss_solve(ctx.h, stype, mh, ph, C.c_void_p(hb.data_ptr()),
                            C.c_void_p(hx.data_ptr()), H.HOST, C.byref(params), C.byref(st))
        if rc:
            raise RuntimeError(L.hamlss_last_error())
        if ph:
            L.hamlss_precond_release(ph)
        L.hamlss_mat_release(mh)
        return st

    e2e_step()
    if dist:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    e_steps = max(1, min(args.steps, 3))
    t0 = time.perf_counter()
    for _ in range(e_steps):
        e2e_step()
    torch.cuda.synchronize()
    e_dt = max_over_ranks(time.perf_counter() - t0, "cuda")
    e2e_value = replica_throughput(e_steps, world, e_dt * 1e3)
    log(f"e2e {e_steps} solves: {e_dt:.3f} s")
    h2d = 4 * (n + 1) + 12 * nnz + 8 * n + 8 * n       # CSR + b + initial x
    d2h = 8 * n                                         # solution

    # ---- roofline of the dominant kernel family
    # The AMG setup ("setup": aggregation, SpGEMM, dense LU -- many small kernels with no
    # streaming-byte model) is reported by its share; the roofline is for the solve kernel
    # family that takes the most device time.
    peak, peak_kind = peaks()
    dev_total = max(sum(f[2] for f in fams), 1e-9)
    solve_fams = [f for f in fams if f[0] != "setup" and f[3] > 0]
    dom = max(solve_fams, key=lambda f: f[2]) if solve_fams else ("none", 0, 0.0, 0.0)
    achieved = (dom[3] / (dom[2] / 1e3)) / 1e9 if dom[2] > 0 else 0.0
    traffic, traffic_launch, traffic_alg = ncu_traffic(dom[0])
    setup_ms = sum(f[2] for f in fams if f[0] == "setup")
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": traffic,
                "kernel": dom[0], "launches": dom[1],
                "bytes_per_launch": dom[3] / max(dom[1], 1),
                "share_of_device_time": round(dom[2] / dev_total, 4),
                "setup_share_of_device_time": round(setup_ms / dev_total, 4),
                "traffic_launch": traffic_launch, "traffic_launch_algorithmic_bytes": traffic_alg,
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs, of measured)"
                if peak_kind == "measured" else "fallback 6.65 TB/s (of fallback)"}

    out = {
        "metric": METRIC, "value": round(value, 4), "unit": "solves/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(max_ms / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64" if solver == "amg_mixed" else "f64",
        "data": "synthetic (seeded lognormal kappa, uniform rhs)",
        "config": {"workload": workload_name(args.n_side, solver, hierarchy),
                   "n": n, "nnz": nnz, "solver": solver, "global_batch": world,
                   "amg": amg_config(solver, hierarchy),
                   "l2": "inputs larger than L2 (no flush)", "parallelism": f"replicas x{world}"},
        "iterations": int(np.median(iters)), "true_residual_max": float(max(true_res)),
        "e2e": {"value": round(e2e_value, 4), "unit": "solves/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "roofline": roofline,
        "gpu_launches": (counted[0] * args.steps) if counted else int(total_launches),
        "gpu_launches_source": ("engine kernels of one step counted by the CUDA activity profiler "
                                "(CUPTI) after the timed region, times the steps" if counted else
                                "engine profiler's outermost operations (activity profiler "
                                "unavailable)"),
        "other_launches_per_step": counted[1] if counted else None,
        "profiled_operations": int(total_launches),
        "kernel_families": {f[0]: {"launches": f[1], "ms": round(f[2], 3),
                                   "GB/s": round(f[3] / max(f[2], 1e-9) / 1e6, 1)} for f in fams},
        "clocks": clocks.summary(),
        "solve_only": solve_only,
    }
    return out, (rp, ci, v, b)


REF_FIXTURE = os.path.join(ROOT, "tests", "golden", "ref_cg_jacobi_2048.json")
# the largest grid side on which the reference's AMG can be set up: its smoothed
# prolongation forms a dense n_fine x n_coarse buffer whose size overflows int at 256^2
# (amg.cpp:113)
REF_AMG_MAX_SIDE = 240


def ref_full_solve():
    """The reference's own complete CG+Jacobi solve of the 2048^2 benchmark system
    (iterations, wall time, threads), recorded by tests/golden/make_ref_iterations.py."""
    try:
        with open(REF_FIXTURE) as f:
            return json.load(f)
    except (OSError, ValueError):
        return None


def cpu_baseline(args, data):
    """The reference's CG+Jacobi (its only path at this size) timed on a bounded sample of
    iterations of the same system, scaled by the iteration count of the reference's own
    complete solve (fixture written by the reference itself)."""
    rp, ci, v, b = data
    full = ref_full_solve()
    if args.n_side != 2048 or not full:
        return None
    threads = cpu_threads()
    dt, it = reference_cpu_sample(rp, ci, v, b, args.cpu_sample_iters, threads)
    per_iter = dt / max(it, 1)
    value = 1.0 / (per_iter * full["iterations"])
    return {"value": value, "unit": "solves/s", "cores": threads, "kind": "reference",
            "sample": f"{it} CG+Jacobi iterations of the reference (release build, {threads} "
                      f"OpenMP threads) on the same 2048^2 system, {dt:.1f} s, scaled to the "
                      f"{full['iterations']} iterations of the reference's own complete solve "
                      f"of this system to 1e-10 ({full['wall_s']} s on {full['threads']} "
                      f"threads, tests/golden/ref_cg_jacobi_2048.json); its AMG cannot be set "
                      f"up at this size (amg.cpp:113)"}


def same_algorithm_side(args, local, side=REF_AMG_MAX_SIDE):
    """Device PCG + SA-AMG against the reference's CGSolver + AMGPreconditioner on the
    largest grid the reference's AMG can set up: variable-kappa Poisson side^2 (sigma 1,
    rhs U[-1, 1)), rtol 1e-10, the reference's own AMG defaults (theta 0.25, omega 0.67,
    coarse limit 50, 10 levels, V(2, 2)), FP64 on both sides.  One complete solve each
    (matrix in, preconditioner setup, solve, solution out); device: median of 5 through
    the C ABI with host buffers; reference: all host threads."""
    import ctypes as C

    import hsps_b200 as H
    import oracle
    from hsps_b200 import _abi
    from hsps_b200._abi import default_params

    rp, ci, v, b = problem(side, 4242)
    n, nnz = len(rp) - 1, len(v)
    p = default_params(tol=TOL, max_iter=1000)
    L = _abi.lib()
    ctx = H.Context(local)

    def device_once():
        x = np.zeros(n)
        t0 = time.perf_counter()
        mh = C.c_void_p()
        if L.hamlss_mat_upload(ctx.h, n, n, nnz, rp.ctypes.data, ci.ctypes.data, v.ctypes.data,
                               H.HOST, C.byref(mh)):
            raise RuntimeError(L.hamlss_last_error())
        M = C.c_void_p()
        if L.hamlss_precond_setup(ctx.h, mh, H.PREC_AMG, C.byref(p), C.byref(M), None):
            raise RuntimeError(L.hamlss_last_error())
        st = _abi.Stats()
        rc = L.hamlss_solve(ctx.h, H.SOLVER_CG, mh, M, b.ctypes.data, x.ctypes.data, H.HOST,
                            C.byref(p), C.byref(st))
        dt = time.perf_counter() - t0
        L.hamlss_precond_release(M)
        L.hamlss_mat_release(mh)
        if rc:
            raise RuntimeError(L.hamlss_last_error())
        return dt, st

    device_once()
    runs = [device_once() for _ in range(5)]
    dev_s = float(np.median([r[0] for r in runs]))
    dst = runs[-1][1]
    threads = cpu_threads()
    R = oracle.Reference(fast=True, threads=threads)
    t0 = time.perf_counter()
    rc, xr, sr = R.solve(H.SOLVER_CG, H.PREC_AMG, rp, ci, v, b, params=p)
    ref_s = time.perf_counter() - t0
    rr = b - oracle.Oracle().spmv(rp, ci, v, xr)
    return {"problem": f"var-kappa Poisson {side}^2 (n {n}, nnz {nnz}), sigma 1, rtol 1e-10, "
                       "PCG + SA-AMG with the reference's AMG defaults, FP64 both sides",
            "device": {"solve_s": round(dev_s, 5), "solves_per_s": round(1.0 / dev_s, 2),
                       "iterations": int(dst.iterations), "true_residual": float(dst.true_residual)},
            "reference": {"solve_s": round(ref_s, 3), "solves_per_s": round(1.0 / ref_s, 4),
                          "setup_s": round(sr.setup_time_s, 3), "iterations": int(sr.iterations),
                          "true_residual": float(np.linalg.norm(rr) / np.linalg.norm(b)),
                          "threads": threads},
            "speedup": round(ref_s / dev_s, 1)}


def coarse512_side(args, local, solver):
    """The same 2048^2 solve with the hierarchy taken down to a dense coarsest level of at
    most 512 rows (no stall cut), as the configuration states it: one complete solve
    (setup + solve), its levels, coarsest size and iterations."""
    import ctypes as C

    import torch

    import hsps_b200 as H
    from hsps_b200 import _abi

    params, stype, ptype = make_params(solver)
    if ptype != H.PREC_AMG:
        return None
    params.amg_stall_ratio = 0.0
    rp, ci, v, b = problem(args.n_side, replica_seed(0))
    n = len(rp) - 1
    ctx = H.Context(local)
    A = H.SparseMatrix(n, n, rp, ci, v, ctx)
    L = _abi.lib()
    db = torch.from_numpy(b).cuda()
    dx = torch.zeros(n, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    h = C.c_void_p()
    if L.hamlss_precond_setup(ctx.h, A.h, ptype, C.byref(params), C.byref(h), None):
        raise RuntimeError(L.hamlss_last_error())
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    st = _abi.Stats()
    rc = L.hamlss_solve(ctx.h, stype, A.h, h, C.c_void_p(db.data_ptr()), C.c_void_p(dx.data_ptr()),
                        H.DEVICE, C.byref(params), C.byref(st))
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    nlev = C.c_int32()
    L.hamlss_amg_num_levels(h, C.byref(nlev))
    r_, c_, z_ = C.c_int32(), C.c_int32(), C.c_int32()
    L.hamlss_amg_level_matrix(h, nlev.value - 1, 0, C.byref(r_), C.byref(c_), C.byref(z_),
                              None, None, None)
    L.hamlss_precond_release(h)
    if rc:
        raise RuntimeError(L.hamlss_last_error())
    return {"hierarchy": "coarsest level <= 512 rows dense, no stall cut", "levels": nlev.value,
            "coarsest_rows": r_.value, "setup_s": round(t1 - t0, 3), "solve_s": round(t2 - t1, 3),
            "iterations": int(st.iterations), "true_residual": float(st.true_residual),
            "solves_per_s": round(1.0 / (t2 - t0), 4)}


def run_reference(args, rank, world):
    """The reference's own CPU solver on the host cores, for this workload.  At 2048^2 its
    AMG cannot be set up (amg.cpp:113) and its only path, CG+Jacobi, takes minutes per
    complete solve, so K complete solves do not fit the arm: the arm reports that and
    exits.  At sides the reference's AMG can set up (<= 240), each step is one complete
    reference solve with CGSolver + AMGPreconditioner (same algorithm, the reference's
    defaults)."""
    if rank != 0:
        return None
    import oracle

    if not oracle.reference_available(fast=True):
        return {"impl": "reference", "unavailable": "reference not built from source (oracle/_ref)"}
    if args.n_side > REF_AMG_MAX_SIDE:
        full = ref_full_solve()
        cost = (f"{full['wall_s']:.0f} s per complete solve ({full['iterations']} iterations on "
                f"{full['threads']} threads)") if full else "minutes per complete solve"
        return {"impl": "reference",
                "unavailable": f"the reference cannot set up its AMG above {REF_AMG_MAX_SIDE}^2 "
                               f"(dense n_fine x n_coarse buffer, amg.cpp:113); its only path at "
                               f"{args.n_side}^2, CGSolver + JacobiPreconditioner, takes {cost}, so "
                               f"{args.warmup + args.steps} complete solves do not fit the arm's "
                               f"time limit"}
    from hsps_b200._abi import default_params

    rp, ci, v, b = problem(args.n_side, 1000)
    threads = cpu_threads()
    R = oracle.Reference(fast=True, threads=threads)
    p = default_params(tol=TOL, max_iter=1000)
    for _ in range(max(0, min(args.warmup, 1))):
        R.solve(0, 3, rp, ci, v, b, params=p)
    t0 = time.perf_counter()
    its = []
    for _ in range(args.steps):
        rc, x, st = R.solve(0, 3, rp, ci, v, b, params=p)
        its.append(st.iterations)
    dt = time.perf_counter() - t0
    value = args.steps / dt
    return {"impl": "reference", "metric": METRIC.replace("2048^2", f"{args.n_side}^2"),
            "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)",
            "config": {"workload": f"var-kappa Poisson {args.n_side}^2 5-point, sigma={SIGMA}, "
                                   f"rtol {TOL}, reference CGSolver + AMGPreconditioner",
                       "n": len(rp) - 1, "nnz": len(v), "iterations": int(np.median(its))},
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": threads,
                             "kind": "reference",
                             "sample": f"{args.steps} complete solves (setup + solve)"},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


# ------------------------------------------------------------------ serving stream
def serving_params():
    import hsps_b200 as H

    return H.SolverParams(tol=TOL, max_iter=4000, restart_size=30, drop_tol=0.0,
                          precision=1, amg_omega=2.0 / 3.0, amg_coarse_limit=512, amg_levels=25,
                          amg_stall_ratio=STALL, ladder_mode=3)


def _pct(lat, q):
    lat = sorted(lat)
    k = max(0, min(len(lat) - 1, int(np.ceil(q * len(lat))) - 1))
    return lat[k]


def serve_plain(reqs, params, device):
    """One solve per call, in arrival order (the one-solve-per-launch path): upload, adaptive
    ladder, download through the C ABI on one context; when the ladder fails at its top, the
    rungs it skipped are tried from x0 as the server does (same algorithm, no concurrency,
    no coalescing).  Latency = completion - arrival."""
    import ctypes as C

    import hsps_b200 as H
    from hsps_b200 import _abi
    from hsps_b200.mtx import _spd_like

    L = _abi.lib()
    ctx = H.Context(device)
    lat, res = [], []
    setup_errors = (_abi.ERR_NOMEM, _abi.ERR_ZERO_PIVOT, _abi.ERR_TIMEOUT, _abi.ERR_ZERO_DIAG)
    t0 = time.perf_counter()
    first_arrival = None
    for rp, ci, v, b, arr, _ in reqs:
        if first_arrival is None:
            first_arrival = arr
        now = time.perf_counter() - t0
        if now < arr:
            time.sleep(arr - now)
        x = np.zeros(len(b))
        mh = C.c_void_p()
        rc = L.hamlss_mat_upload(ctx.h, len(b), len(b), len(v), rp.ctypes.data, ci.ctypes.data,
                                 v.ctypes.data, H.HOST, C.byref(mh))
        st = _abi.Stats()
        nlog, init = C.c_int32(), C.c_int32()
        if rc == 0:
            rc = L.hamlss_solve_adaptive(ctx.h, mh, b.ctypes.data, x.ctypes.data, H.HOST,
                                         C.byref(params), C.byref(st), None, 0, C.byref(nlog),
                                         C.byref(init))
            if rc in setup_errors:
                rc, st.converged = 0, 0
        for state in range(init.value - 1, -1, -1):
            if rc or st.converged:
                break
            if state == 0 and not _spd_like(len(b), rp, ci, v):
                continue
            kind, solver = (H.PREC_JACOBI, H.SOLVER_CG) if state == 0 else (H.PREC_ILU, H.SOLVER_FGMRES)
            M = C.c_void_p()
            setup = C.c_double()
            if L.hamlss_precond_setup(ctx.h, mh, kind, C.byref(params), C.byref(M), C.byref(setup)):
                continue
            x2 = np.zeros(len(b))
            s2 = _abi.Stats()
            rc2 = L.hamlss_solve(ctx.h, solver, mh, M, b.ctypes.data, x2.ctypes.data, H.HOST,
                                 C.byref(params), C.byref(s2))
            L.hamlss_precond_release(M)
            if rc2 == 0 and s2.converged:
                x, st = x2, s2
        L.hamlss_mat_release(mh)
        if rc:
            raise RuntimeError(L.hamlss_last_error())
        lat.append(time.perf_counter() - t0 - arr)
        res.append(st.true_residual if st.converged else float("inf"))
    span = time.perf_counter() - t0 - first_arrival
    return {"solves_per_s": round(len(lat) / span, 3), "p50_ms": round(1e3 * _pct(lat, 0.5), 2),
            "p99_ms": round(1e3 * _pct(lat, 0.99), 2), "max_true_residual": max(res)}


def serve_engine(reqs, params, device, order=0):
    """The continuous-batching server: requests submitted at their arrival times; order 0
    admits in arrival order, 1 fewest nonzeros first."""
    from hsps_b200.serve import Server

    with Server(device=device, slots=4, batch_max_rows=16384, order=order) as srv:
        hs = []
        t0 = time.perf_counter()
        for rp, ci, v, b, arr, _ in reqs:
            now = time.perf_counter() - t0
            if now < arr:
                time.sleep(arr - now)
            hs.append(srv.submit(rp, ci, v, b, params=params))
        res = []
        for h in hs:
            _, st = h.wait(timeout=900)
            res.append(st.true_residual if st.converged else float("inf"))
        rep = srv.report()
    return {"solves_per_s": round(rep["solves_per_s"], 2),
            "p50_ms": round(1e3 * rep["p50_latency_s"], 2),
            "p99_ms": round(1e3 * rep["p99_latency_s"], 2), "max_true_residual": max(res),
            "coalesced": rep["coalesced"], "batches": rep["batches"],
            "escalated": rep["escalated"], "peak_running": rep["peak_running"],
            "peak_admitted_gb": round(rep["peak_admitted_bytes"] / 1e9, 3)}


def run_serving(args, local):
    """Serving stream: burst capacity of both paths, then Poisson arrivals at 90% of the
    plain path's capacity, latencies measured from arrival."""
    from hsps_b200 import problems as P

    R = args.serving_requests
    params = serving_params()
    burst = P.serving_stream(R, 77, 1e3, args.serving_n_max, rate=0.0)
    serve_plain(burst[:8], params, local)           # warm-up (module load, first contexts)
    serve_engine(burst[:8], params, local)
    log("serving: burst, plain path")
    plain_b = serve_plain(burst, params, local)
    log(f"serving: burst, server ({plain_b})")
    eng_b = serve_engine(burst, params, local)
    log(f"serving: arrivals ({eng_b})")
    rate = 0.9 * plain_b["solves_per_s"]
    timed = P.serving_stream(R, 77, 1e3, args.serving_n_max, rate=rate)
    plain_r = serve_plain(timed, params, local)
    eng_r = serve_engine(timed, params, local)
    eng_s = serve_engine(timed, params, local, order=1)
    return {"requests": R, "n_range": [1e3, args.serving_n_max], "tol": TOL,
            "mix": "50% var-kappa Poisson, 35% upwind conv-diff, 15% shifted Helmholtz",
            "inner": "mixed precision (FP32 inner, FP64 refinement), adaptive ladder",
            "burst": {"server": eng_b, "plain": plain_b},
            "poisson_arrivals": {"rate_per_s": round(rate, 2), "server": eng_r,
                                 "server_fewest_nonzeros_first": eng_s, "plain": plain_r}}


class PrefetchStream:
    """The requests of a spec list, built in arrival order by a background thread at most
    `ahead` requests ahead (large systems are not all held in memory at once)."""

    def __init__(self, specs, ahead=12):
        import queue

        from hsps_b200 import problems as P

        self.q = queue.Queue(maxsize=ahead)
        self.n = len(specs)

        def work():
            for sp in specs:
                self.q.put(P.build_request(sp))

        self.t = threading.Thread(target=work, daemon=True)
        self.t.start()

    def __iter__(self):
        for _ in range(self.n):
            yield self.q.get()


def serve_engine_stream(reqs, params, device):
    """serve_engine for a lazily built stream: results are collected as they finish by a
    second thread, so finished requests' arrays are released."""
    import queue

    from hsps_b200.serve import Server

    with Server(device=device, slots=4, batch_max_rows=16384) as srv:
        pending = queue.Queue()
        res = []

        def collect():
            while True:
                h = pending.get()
                if h is None:
                    return
                _, st = h.wait(timeout=1800)
                res.append(st.true_residual if st.converged else float("inf"))

        ct = threading.Thread(target=collect, daemon=True)
        ct.start()
        t0 = time.perf_counter()
        for rp, ci, v, b, arr, _ in reqs:
            now = time.perf_counter() - t0
            if now < arr:
                time.sleep(arr - now)
            pending.put(srv.submit(rp, ci, v, b, params=params))
        pending.put(None)
        ct.join()
        rep = srv.report()
    return {"solves_per_s": round(rep["solves_per_s"], 3),
            "p50_ms": round(1e3 * rep["p50_latency_s"], 2),
            "p99_ms": round(1e3 * rep["p99_latency_s"], 2), "max_true_residual": max(res),
            "coalesced": rep["coalesced"], "escalated": rep["escalated"],
            "peak_running": rep["peak_running"],
            "peak_admitted_gb": round(rep["peak_admitted_bytes"] / 1e9, 3)}


def run_serving_full(args, local):
    """The serving configuration's full size range: `--serving-full N` requests with n
    log-uniform in [1e3, 4.2e6] (the stated mix: 50% variable-kappa Poisson, 35% upwind
    conv-diff, 15% shifted Helmholtz), Poisson arrivals at `--serving-rate` per second, the
    adaptive ladder with mixed-precision inner solves to 1e-10, 150 GB admission budget.
    Server (arrival order, at most one request of >= 2^20 rows at a time) against one
    solve per call in arrival order; both build each request just ahead of its arrival.
    Beside them, the reference's own AdaptiveSelector (drop_tol 0, all host threads) replays
    a sample of the requests it can complete (n <= 57,600: above that its AMG rung cannot
    be set up); the rest are counted as reference-unavailable."""
    import oracle
    from hsps_b200 import problems as P

    N, rate = args.serving_full, args.serving_rate
    params = serving_params()
    specs = P.serving_specs(N, 91, 1e3, 4.2e6, rate=rate)
    sizes = np.array([sp[1] * sp[1] for sp in specs])
    warm = [P.build_request(sp) for sp in P.serving_specs(4, 92, 1e3, 2e4, rate=0.0)]
    serve_plain(warm, params, local)
    serve_engine(warm, params, local)
    log(f"serving (full range): {N} requests at {rate}/s, server")
    eng = serve_engine_stream(PrefetchStream(specs), params, local)
    log(f"serving (full range): plain path ({eng})")
    plain = serve_plain(PrefetchStream(specs), params, local)
    log(f"serving (full range): reference sample ({plain})")
    ok = [k for k in range(N) if sizes[k] <= 57600]
    sample = ok[:args.serving_ref_sample]
    R = oracle.Reference(fast=True, threads=cpu_threads())
    from hsps_b200._abi import default_params

    rp_ = default_params(tol=TOL, max_iter=4000, restart_size=30, drop_tol=0.0)
    ref_t, ref_conv = [], 0
    for k in sample:
        rp, ci, v, b, _, _ = P.build_request(specs[k])
        t0 = time.perf_counter()
        rc, x, st, logr = R.solve_adaptive(rp, ci, v, b, params=rp_)
        ref_t.append(time.perf_counter() - t0)
        ref_conv += int(bool(st.converged))
    return {"requests": N, "n_range": [1e3, 4.2e6], "rate_per_s": rate, "tol": TOL,
            "mean_rows": float(sizes.mean()), "requests_over_1e6_rows": int((sizes > 1e6).sum()),
            "mix": "50% var-kappa Poisson, 35% upwind conv-diff, 15% shifted Helmholtz",
            "server": eng, "plain": plain,
            "reference": {"solvable_requests": len(ok), "unavailable_requests": N - len(ok),
                          "sample": len(sample), "threads": cpu_threads(),
                          "converged": ref_conv,
                          "solves_per_s_sample": round(len(ref_t) / max(sum(ref_t), 1e-9), 3),
                          "p50_ms_sample": round(1e3 * float(np.median(ref_t)), 2) if ref_t else None,
                          "note": "service time only (sequential replay, no queueing)"}}


def run_ilut_side(args, local):
    """ILUT(1e-4, 0) -- the factory's ILU under the default drop_tol -- set up on the device
    and by the reference (setup_ilut, one host thread: it is sequential) on the upwind
    conv-diff 128^2 (eps 1, beta (10, 5)); FGMRES(30) iterations with each; then the device
    setup alone at 1024^2, where the reference's O(n^2) scans would take hours."""
    import hsps_b200 as H
    import oracle
    from hsps_b200 import problems as P
    from hsps_b200._abi import default_params

    def device(A, solve):
        n = len(A[0]) - 1
        M = H.SparseMatrix(n, n, *A)
        times = []
        for _ in range(5):
            I = H.ILUPreconditioner()
            I.set_drop_tol(1e-4)
            times.append(I.setup(M))
        out = {"n": n, "setup_ms": round(1e3 * float(np.median(times)), 3),
               "factor_nnz": int(len(I.factor_csr()[1]))}
        if solve:
            s = H.FGMRESSolver()
            s.set_params(default_params(tol=1e-8, max_iter=2000, restart_size=30))
            s.set_preconditioner(I)
            st = H.SolverStats()
            x = np.zeros(n)
            t0 = time.perf_counter()
            s.solve(M, np.ones(n), x, st)
            out.update(iterations=st.iterations, solve_ms=round(1e3 * (time.perf_counter() - t0), 3))
        return out

    A = P.convection_diffusion_2d(128, 1.0, 10.0, 5.0)
    dev = device(A, True)
    R = oracle.Reference(fast=True, threads=1)
    t0 = time.perf_counter()
    frp, fci, flu = R.ilut(*A, 1e-4, 0)
    ref_setup = time.perf_counter() - t0
    p = default_params(tol=1e-8, max_iter=2000, restart_size=30)
    rc, x, st = R.solve(1, 2, *A, np.ones(len(A[0]) - 1), params=p)
    big = device(P.convection_diffusion_2d(1024, 1.0, 10.0, 5.0), False)
    return {"problem": "upwind conv-diff eps 1, beta (10, 5); ILUT(1e-4, 0); FGMRES(30) to 1e-8, b = 1",
            "device_128": dev,
            "reference_128": {"setup_ms": round(1e3 * ref_setup, 3), "factor_nnz": int(len(fci)),
                              "iterations": st.iterations, "threads": 1},
            "device_1024": big}


def run_config_side(args, local):
    """Latency of one complete solve call (host buffers in, solution out; preconditioner
    setup included) for the small configurations: C1 Poisson 64^2 PCG + Jacobi and C2
    upwind conv-diff 512^2 (cell Peclet 10) FGMRES(30) + ILU(0), both to rtol 1e-8 -- the
    device (median of 10) against the reference's own solvers (all host threads, median of
    3)."""
    import hsps_b200 as H
    import oracle
    from hsps_b200 import problems as P
    from hsps_b200._abi import default_params

    R = oracle.Reference(fast=True, threads=cpu_threads())
    ctx = H.Context(local)
    out = {"reference_threads": cpu_threads()}
    cases = (("C1_poisson64_pcg_jacobi", P.poisson_2d(64), 0, "CG", "JACOBI",
              default_params(tol=1e-8, max_iter=1000)),
             ("C2_convdiff512_pe10_fgmres30_ilu0",
              P.convection_diffusion_2d(512, 1.0, *P.convdiff_wind(512, 10.0)), 2, "FGMRES", "ILU",
              default_params(tol=1e-8, max_iter=3000, restart_size=30, drop_tol=0.0)))
    for name, A, seed, sname, pname, p in cases:
        n = len(A[0]) - 1
        b = P.rhs(n, seed)
        dev = []
        for _ in range(11):
            t0 = time.perf_counter()
            M = H.SparseMatrix(n, n, *A, ctx)
            s, _ = H.SolverFactory.make(sname, pname, M, p)
            x = np.zeros(n)
            st = H.SolverStats()
            s.solve(M, b, x, st)
            dev.append(time.perf_counter() - t0)
        ref = []
        for _ in range(3):
            t0 = time.perf_counter()
            rc, xr, sr = R.solve(0 if sname == "CG" else 1, 1 if pname == "JACOBI" else 2, *A, b, params=p)
            ref.append(time.perf_counter() - t0)
        out[name] = {"n": n, "nnz": len(A[2]), "device_ms": round(1e3 * float(np.median(dev[1:])), 3),
                     "iterations": st.iterations, "reference_ms": round(1e3 * float(np.median(ref)), 3),
                     "reference_iterations": sr.iterations}
    return out


def run_batch_side(args, local):
    """Batched uneven systems: `count` problems with side s ~ U{16..128}, half
    variable-kappa Poisson (sigma 0.5; CG + Jacobi), half upwind conv-diff (cell Peclet
    log-uniform in [1, 100]; FGMRES(20) + ILU(0)), rhs U[0, 1), rtol 1e-8, FP32 inner
    iterations inside FP64 refinement -- all of them in one persistent launch.  Beside it:
    one solve call per problem through the C ABI (a sample of 256, scaled), and the
    reference's own solvers one after another on a sample of 64 (scaled)."""
    import hsps_b200 as H
    import oracle
    from hsps_b200 import batch as B
    from hsps_b200 import problems as P
    from hsps_b200._abi import default_params

    count = args.batch_count
    rng = np.random.default_rng(2024)
    systems, solvers, precs, rhs = [], [], [], []
    for k in range(count):
        side = int(rng.integers(16, 129))
        if k % 2 == 0:
            systems.append(P.varkappa_poisson_2d(side, 0.5, 7000 + k))
            solvers.append(H.SOLVER_CG)
            precs.append(H.PREC_JACOBI)
        else:
            pe = float(np.exp(rng.uniform(0.0, np.log(100.0))))
            systems.append(P.convection_diffusion_2d(side, 1.0, *P.convdiff_wind(side, pe)))
            solvers.append(H.SOLVER_FGMRES)
            precs.append(H.PREC_ILU)
        rhs.append(P.rhs(side * side, 9000 + k))
    p = default_params(tol=1e-8, max_iter=4000, restart_size=20, drop_tol=0.0)
    n_tot = sum(len(sy[0]) - 1 for sy in systems)
    nnz_tot = sum(len(sy[2]) for sy in systems)
    bs = B.BatchSolver(systems, solvers, precs, p)
    bflat = bs.join(rhs)
    bs.solve(bflat)                                          # warm-up (autotune defaults)
    times = []
    for _ in range(3):
        t0 = time.perf_counter()
        x, res, tot = bs.solve(bflat)
        times.append(time.perf_counter() - t0)
    conv = sum(r["converged"] for r in res)
    worst = max(r["final_residual"] for r in res)
    bs.release()
    batch_s = float(np.median(times))
    # one solve call per problem (host buffers), a sample
    ctx = H.Context(local)
    sample = list(range(0, count, max(1, count // 256)))[:256]
    t0 = time.perf_counter()
    for k in sample:
        rp, ci, v = systems[k]
        n = len(rp) - 1
        M = H.SparseMatrix(n, n, rp, ci, v, ctx)
        s, _ = H.SolverFactory.make(solvers[k], precs[k], M, p)
        x = np.zeros(n)
        s.solve(M, rhs[k], x)
    loop_s = (time.perf_counter() - t0) * count / len(sample)
    R = oracle.Reference(fast=True, threads=1)
    rsample = sample[:64]
    t0 = time.perf_counter()
    for k in rsample:
        R.solve(0 if solvers[k] == H.SOLVER_CG else 1, 1 if precs[k] == H.PREC_JACOBI else 2,
                *systems[k], rhs[k], params=p)
    ref_s = (time.perf_counter() - t0) * count / len(rsample)
    return {"problem": f"{count} systems, side U{{16..128}}, half var-kappa Poisson (CG+Jacobi), "
                       "half upwind conv-diff Pe 1-100 (FGMRES(20)+ILU(0)), rtol 1e-8",
            "rows": n_tot, "nnz": nnz_tot, "converged": conv, "max_final_residual": worst,
            "batch_s": round(batch_s, 4), "batch_solves_per_s": round(count / batch_s, 1),
            "one_call_per_problem_s": round(loop_s, 3), "one_call_sample": len(sample),
            "reference_sequential_s": round(ref_s, 3), "reference_sample": len(rsample),
            "reference_threads": 1}


def run_variants_side(args, local):
    """CG, FGMRES(30), PipelinedFGMRES(30) (Jacobi) and SStepCG(k = 4) on the unit-diagonal
    shifted Helmholtz operator D^-1/2 (A + cI) D^-1/2 on 512^2 (c = 7; a spectrum inside
    (0, 2), where the reference's s-step update converges), to 1e-8: device time and
    iterations, and the reference's own solvers on the same system (all host threads)."""
    import hsps_b200 as H
    import oracle
    from hsps_b200 import problems as P
    from hsps_b200._abi import default_params

    rp, ci, v = P.helmholtz_2d(512, 7.0)
    n = len(rp) - 1
    rows = np.repeat(np.arange(n), np.diff(rp))
    d = 1.0 / np.sqrt(v[ci == rows])
    v = v * d[rows] * d[ci]
    b = P.rhs(n, 5)
    p = default_params(tol=1e-8, max_iter=2000, restart_size=30, sstep_k=4)
    M = H.SparseMatrix(n, n, rp, ci, v)
    R = oracle.Reference(fast=True, threads=cpu_threads())
    out = {"problem": "unit-diagonal shifted Helmholtz 512^2 (c = 7), tol 1e-8, Jacobi"}
    for name, solver, code in (("cg", H.CGSolver, 0), ("fgmres", H.FGMRESSolver, 1),
                               ("pipelined_fgmres", H.PipelinedFGMRESSolver, 5),
                               ("sstep_cg_k4", lambda: H.SStepCGSolver(4), 3)):
        times = []
        for _ in range(4):
            s = solver()
            s.set_params(p)
            s.set_preconditioner(H.SolverFactory.make_precond(H.PREC_JACOBI, M, p))
            st = H.SolverStats()
            x = np.zeros(n)
            s.solve(M, b, x, st)
            times.append(st.device_time_s)
        t0 = time.perf_counter()
        rc, xr, sr = R.solve(code, H.PREC_JACOBI, rp, ci, v, b, params=p)
        ref_s = time.perf_counter() - t0
        out[name] = {"device_ms": round(1e3 * float(np.median(times[1:])), 3), "iterations": st.iterations,
                     "converged": bool(st.converged), "reference_ms": round(1e3 * ref_s, 3),
                     "reference_iterations": sr.iterations, "reference_converged": bool(sr.converged)}
    out["reference_threads"] = cpu_threads()
    return out


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "reference":
        out = run_reference(args, rank, world)
        if out is not None:
            print(json.dumps(out), flush=True)
        return
    if world > 1:
        import datetime

        import torch

        torch.cuda.set_device(local)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                             device_id=torch.device("cuda", local))
    out, data = run_ours(args, rank, world, local)
    if out is None:
        return
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        log("timing the reference sample")
        cb = cpu_baseline(args, data)
        if cb:
            out["cpu_baseline"] = cb
        log("cpu baseline done")
    if rank == 0 and world == 1 and not args.no_same_algorithm:
        log(f"same-algorithm side measurement at {REF_AMG_MAX_SIDE}^2 (device vs reference AMG-PCG)")
        out["reference_same_algorithm"] = same_algorithm_side(args, local)
    if rank == 0 and world == 1 and not args.no_coarse512:
        log("coarsest <= 512 hierarchy side measurement")
        out["hierarchy_coarse512"] = coarse512_side(args, local, out["config"]["solver"])
    if rank == 0 and world == 1 and args.serving_full > 0:
        out["serving_full_range"] = run_serving_full(args, local)
    if rank == 0 and world == 1 and args.serving_requests > 0:
        out["serving"] = run_serving(args, local)
    if rank == 0 and world == 1 and not args.no_configs:
        log("C1 / C2 latency side measurement")
        out["configs"] = run_config_side(args, local)
    if rank == 0 and world == 1 and not args.no_batch:
        log("batched-systems side measurement")
        out["batched"] = run_batch_side(args, local)
    if rank == 0 and world == 1 and not args.no_variants:
        log("Krylov-variant side measurement")
        out["krylov_variants"] = run_variants_side(args, local)
    if rank == 0 and world == 1 and not args.no_ilut:
        log("ILUT side measurement")
        out["ilut"] = run_ilut_side(args, local)
    if world > 1:
        import torch

        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
