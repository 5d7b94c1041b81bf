"""Host logic of the multi-GPU path (CPU, no GPU): replicas only.

- bench.py's rank aggregation: every rank times its own solves; the job's time is the
  slowest rank's (max over ranks) and its throughput counts every rank's solves.  Run as
  two gloo ranks on CPU.
- serve.Router: least-loaded dispatch over one server per GPU, checked with fake servers.
"""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        local_ms = 100.0 + 50.0 * rank              # rank 1 is the slow replica
        m = bench.max_over_ranks(local_ms, "cpu")
        out[rank] = (m, bench.replica_throughput(4, world, m), bench.replica_seed(rank))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_rank_aggregation_gloo_two_ranks():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert out[0][0] == out[1][0] == 150.0          # slowest rank's time on every rank
    assert out[0][1] == pytest.approx(2 * 4 / 0.150)  # both ranks' solves over that time
    assert out[0][2] != out[1][2]                    # each replica has its own instance


def test_single_process_aggregation_is_identity():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(12.5, "cpu") == 12.5
    assert bench.replica_throughput(5, 1, 1000.0) == 5.0


class _FakeServer:
    def __init__(self, load):
        self.load = load
        self.got = []

    def report(self):
        return {"queued": self.load, "running": 0}

    def submit(self, *a, **k):
        self.got.append(a)
        self.load += 1
        return len(self.got)

    def close(self):
        pass


def test_router_least_loaded():
    from hsps_b200.serve import Router

    fakes = [_FakeServer(3), _FakeServer(0), _FakeServer(1)]
    r = Router(fakes)
    for i in range(5):
        r.submit([0], [], [], [], params=None)
    # loads 3,0,1: picks 1, 1 (tie with 2 -> lower index), 2, 1, 2; every load ends at 3
    assert [f.load for f in fakes] == [3, 3, 3]
    assert r.routed == [0, 3, 2]
    with pytest.raises(ValueError):
        Router([])
