"""bench.py's clock sampler, against a stand-in `nvidia-smi` on PATH (no GPU needed).

The sampler starts before the warm-up steps (the first `nvidia-smi` start on a fresh
machine initialises NVML and disturbs the GPU for about a second), so these tests check
that `ready()` waits for the first sample, that `mark()` keeps only what is sampled from
the timed region on, and that the summary reports the median clock and any throttle
reason seen.
"""
import os
import stat
import sys
import time

import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), ".."))


def fake_smi(tmp_path, lines, delay=0.02):
    """An executable `nvidia-smi` printing `lines` in order, `delay` seconds apart, then
    repeating the last one until it is terminated."""
    script = tmp_path / "nvidia-smi"
    body = "\n".join(f"echo '{ln}'; sleep {delay}" for ln in lines)
    script.write_text("#!/bin/sh\n" + body + f"\nwhile true; do echo '{lines[-1]}'; sleep {delay}; done\n")
    script.chmod(script.stat().st_mode | stat.S_IXUSR)
    return str(tmp_path)


def row(sm, mx=1965, reason="Not Active"):
    return f"0, {sm}, {mx}, 700.0, 0x0, Not Active, Not Active, Not Active, {reason}"


@pytest.fixture
def bench_mod(monkeypatch, tmp_path):
    import bench
    return bench


def test_ready_mark_and_summary(bench_mod, monkeypatch, tmp_path):
    warm = [row(1200, reason="Active")] * 5              # start-up samples, then dropped
    timed = [row(1965)] * 3
    monkeypatch.setenv("PATH", fake_smi(tmp_path, warm + timed) + os.pathsep + os.environ["PATH"])
    c = bench_mod.Clocks(0)
    c.start()
    try:
        c.ready(timeout=5.0)
        assert c.rows, "ready() returned before the first sample"
        time.sleep(0.3)                                   # past the start-up samples
        c.mark()
        time.sleep(0.2)
    finally:
        c.stop()
    s = c.summary()
    assert s["samples"] >= 1
    assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == []                             # the start-up throttle was marked away


def test_reasons_and_missing_tool(bench_mod, monkeypatch, tmp_path):
    monkeypatch.setenv("PATH", fake_smi(tmp_path, [row(1300, reason="Active")]) + os.pathsep
                       + os.environ["PATH"])
    c = bench_mod.Clocks(0)
    c.start()
    try:
        c.ready(timeout=5.0)
        c.mark()
        time.sleep(0.2)
    finally:
        c.stop()
    assert c.summary()["reasons"] == ["sw_power_cap"]
    # no nvidia-smi at all: the summary says so instead of failing
    empty = tmp_path / "empty"
    empty.mkdir()
    monkeypatch.setenv("PATH", str(empty))
    c2 = bench_mod.Clocks(0)
    c2.start()
    c2.ready(timeout=0.2)
    c2.stop()
    assert c2.summary()["reasons"] == ["unavailable"]
