"""Shared test setup: markers, paths and fixtures."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "hybrid-sparse-pde-solver_b200")
for p in (PKG, os.path.join(ROOT, "oracle"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: long-running case")


@pytest.fixture(scope="session")
def orc():
    import oracle

    return oracle.Oracle()


@pytest.fixture(scope="session")
def ref():
    import oracle

    if not oracle.reference_available():
        pytest.skip("reference not built from source here (oracle/_ref missing)")
    return oracle.Reference(threads=1)
