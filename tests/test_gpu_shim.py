"""The C++ drop-in shim (hybrid-sparse-pde-solver_b200/shim/hsps_device.hpp) driven the
way the project's own code drives its solvers: tests/shim/shim_test.cpp runs the
project's CPU classes and the device classes side by side (-m gpu)."""
import os
import subprocess

import pytest

from gpu_util import need_gpu

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "tests", "shim", "_build", "shim_test")


def test_shim_matches_project_classes():
    need_gpu()
    if not os.path.exists(BIN):
        pytest.skip("shim test not built (needs the project's headers: make -C "
                    "hybrid-sparse-pde-solver_b200 shim-test)")
    out = subprocess.run([BIN], capture_output=True, text=True, timeout=600)
    print(out.stdout)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "PASSED" in out.stdout
