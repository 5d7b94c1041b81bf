"""The continuous-batching server (hamlss_server_*, -m gpu).

A mixed stream (variable-kappa Poisson, upwind convection-diffusion, shifted Helmholtz;
sizes log-uniform, small ones coalesced into batched launches, large ones on concurrent
solve lanes; mixed-precision inner path with the adaptive ladder) is checked for:
  - every request converged, its FP64 true residual ||b - A x|| / ||b|| (recomputed on the
    host with the oracle's SpMV) at most 1.5 x the tolerance 1e-10 (the factor covers the
    host's different summation order only);
  - the same result alone and in the mix: each request is then solved alone on the same
    server, and the two solutions agree to a relative max-norm difference of 1e-9.  Both
    paths are deterministic (fixed team width per size class in the batch lane, the same
    code as a lone adaptive solve on a solve lane), so the difference is 0 in practice;
    the bound is what the test requires;
  - overlap and coalescing: more than one request was running at once, and the small
    requests took fewer launches than requests;
  - admission: the admitted footprint never exceeded the budget, and a request that can
    never fit is refused at submit time with HAMLSS_ERR_BUDGET;
  - cancellation of a queued request and escalation of a batch failure to the ladder.
"""
import numpy as np
import pytest

from gpu_util import need_gpu
import hsps_b200 as H
from hsps_b200 import _abi
from hsps_b200 import problems as P
from hsps_b200._abi import default_params
from hsps_b200.serve import Server

pytestmark = pytest.mark.gpu

TOL = 1e-10


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    need_gpu()


def params(**over):
    kw = dict(tol=TOL, max_iter=4000, restart_size=30, drop_tol=0.0, precision=_abi.MIXED,
              amg_omega=2.0 / 3.0, amg_coarse_limit=512, amg_levels=25, amg_stall_ratio=0.75,
              ladder_mode=2)
    kw.update(over)
    return default_params(**kw)


def stream(count, seed, n_lo=400, n_hi=70000):
    """(rp, ci, v, b) requests of the serving mix (problems.serving_stream)."""
    return [r[:4] for r in P.serving_stream(count, seed, n_lo, n_hi)]


def rel_res(orc, rp, ci, v, b, x):
    return np.linalg.norm(b - orc.spmv(rp, ci, v, x)) / np.linalg.norm(b)


def test_mix_equals_alone(orc):
    reqs = stream(28, 7)
    with Server(slots=4, batch_max_rows=16384) as srv:
        handles = [srv.submit(rp, ci, v, b, params=params()) for rp, ci, v, b in reqs]
        mixed = [h.wait(timeout=600) for h in handles]
        rep = srv.report()
        alone = []
        for rp, ci, v, b in reqs:
            alone.append(srv.submit(rp, ci, v, b, params=params()).wait(timeout=600))
    assert rep["completed"] == len(reqs) and rep["failed"] == 0, rep
    assert rep["peak_running"] > 1, rep                      # requests overlapped
    assert 0 < rep["batches"] < rep["coalesced"], rep          # small ones were coalesced
    assert rep["peak_admitted_bytes"] <= 150e9
    assert rep["p99_latency_s"] >= rep["p50_latency_s"] > 0
    worst, same_bits = 0.0, 0
    for (rp, ci, v, b), (xm, sm), (xa, sa) in zip(reqs, mixed, alone):
        assert sm.converged and sa.converged
        assert rel_res(orc, rp, ci, v, b, xm) <= 1.5 * TOL
        assert rel_res(orc, rp, ci, v, b, xa) <= 1.5 * TOL
        d = np.max(np.abs(xm - xa)) / np.max(np.abs(xa))
        worst = max(worst, d)
        same_bits += int(np.array_equal(xm, xa))
        assert d <= 1e-9, (len(b), d)
    print(f"mix vs alone: worst rel diff {worst:.3e}, bit-identical {same_bits}/{len(reqs)}; "
          f"report {rep}")


def test_admission_budget(orc):
    big = stream(6, 11, n_lo=40000, n_hi=70000)
    # room for about one large request at a time
    with Server(slots=4, batch_max_rows=0, hbm_budget_bytes=120_000_000) as srv:
        hs = [srv.submit(rp, ci, v, b, params=params()) for rp, ci, v, b in big]
        for (rp, ci, v, b), h in zip(big, hs):
            x, st = h.wait(timeout=600)
            assert st.converged and rel_res(orc, rp, ci, v, b, x) <= 1.5 * TOL
        rep = srv.report()
        assert rep["peak_admitted_bytes"] <= 120_000_000, rep
        huge = P.poisson_2d(1500)
        with pytest.raises(H.HamlssError) as e:
            srv.submit(*huge, P.rhs(1500 * 1500, 1), params=params())
        assert e.value.code == _abi.ERR_BUDGET


def test_cancel_queued():
    first = P.varkappa_poisson_2d(400, 1.0, 3)
    second = P.poisson_2d(300)
    with Server(slots=1, batch_max_rows=0) as srv:
        h1 = srv.submit(*first, P.rhs(400 * 400, 3), params=params(precision=_abi.FP64))
        h2 = srv.submit(*second, P.rhs(300 * 300, 4), params=params())
        h2.cancel()
        with pytest.raises(H.HamlssError) as e:
            h2.wait(timeout=600)
        assert e.value.code == _abi.ERR_CANCELLED
        _, st = h1.wait(timeout=600)
        assert st.converged
        assert srv.report()["cancelled"] == 1


def test_batch_failure_escalates():
    # too few iterations for the batch lane's FGMRES + ILU(0): the request leaves the batch
    # lane and climbs the whole ladder on a solve lane (still not converging at this budget)
    side = 30
    A = P.convection_diffusion_2d(side, 1.0, *P.convdiff_wind(side, 300.0))
    b = P.rhs(side * side, 5)
    with Server(slots=2, batch_max_rows=16384) as srv:
        x, st = srv.submit(*A, b, params=params(max_iter=3, ir_max_outer=1,
                                                amg_stall_ratio=0.0)).wait(timeout=600)
        rep = srv.report()
    assert rep["escalated"] == 1 and rep["coalesced"] == 0, rep
    assert st.state_used == H.STATE_HARD and not st.converged


def test_fewest_nonzeros_first_order(orc):
    # order = 1 with one solve lane and no coalescing: while the first (largest) request
    # runs, the queued ones are admitted smallest first; results are those of the ladder
    reqs = [r for r in stream(12, 11, 2000, 40000)]
    reqs.sort(key=lambda r: -len(r[2]))
    with Server(slots=1, batch_max_rows=0, order=1) as srv:
        handles = [srv.submit(rp, ci, v, b, params=params()) for rp, ci, v, b in reqs]
        out = [h.wait(timeout=600) for h in handles]
        rep = srv.report()
    assert rep["completed"] == len(reqs) and rep["failed"] == 0 and rep["peak_running"] == 1, rep
    for (rp, ci, v, b), (x, st) in zip(reqs, out):
        assert st.converged and rel_res(orc, rp, ci, v, b, x) <= 1.5 * TOL
    with pytest.raises(Exception):
        Server(order=2)
