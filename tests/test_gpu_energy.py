"""NVML energy counter (NVMLMonitor::read_energy_j, src/parallel/nvml_monitor.cpp:85-100 in
the reference): the raw reading through the C ABI, matched to the CUDA device by PCI bus
id, and the per-solve energy in SolverStats.energy_joules_hw (-m gpu).

NVML refreshes the counter every few tens of milliseconds, so the solves here run for
about half a second each (CG + Jacobi on Poisson 2048^2 with a tolerance it does not
reach within max_iter)."""
import ctypes as C

import numpy as np
import pytest

from gpu_util import need_gpu
import hsps_b200 as H
from hsps_b200 import _abi
from hsps_b200 import problems as P
from hsps_b200._abi import default_params

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    need_gpu()


def _read(device=0):
    j = C.c_double()
    rc = _abi.lib().hamlss_energy_read(device, C.byref(j))
    if rc == _abi.ERR_NOT_READY:
        pytest.skip("NVML energy counter not available on this device")
    assert rc == 0, _abi.lib().hamlss_last_error()
    return j.value


def test_counter_is_read_and_never_decreases():
    j0 = _read()
    assert j0 > 0.0
    A = P.poisson_2d(2048)
    n = len(A[0]) - 1
    M = H.SparseMatrix(n, n, *A)
    s, _ = H.SolverFactory.make("CG", "JACOBI", M, default_params(tol=1e-14, max_iter=3000))
    x = np.zeros(n)
    s.solve(M, np.ones(n), x, H.SolverStats())
    j1 = _read()
    assert j1 > j0, (j0, j1)


def test_solves_record_hardware_energy():
    A = P.poisson_2d(2048)
    n = len(A[0]) - 1
    M = H.SparseMatrix(n, n, *A)
    p = default_params(tol=1e-14, max_iter=3000, record_hw_energy=1)
    s, _ = H.SolverFactory.make("CG", "JACOBI", M, p)
    b = P.rhs(n, 3)
    readings, energies = [_read()], []
    for _ in range(2):
        st = H.SolverStats()
        x = np.zeros(n)
        s.solve(M, b, x, st)
        assert st.iterations == 3000
        energies.append(st.energy_joules_hw)
        readings.append(_read())
    assert all(e > 0.0 for e in energies), energies
    assert readings == sorted(readings), readings
    # each solve's energy lies within the counter's change across it
    for k, e in enumerate(energies):
        assert e <= readings[k + 1] - readings[k] + 1e-9, (e, readings)
