"""Helpers for the -m gpu tests."""
import numpy as np
import pytest


def need_gpu():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def csr_dense(rp, ci, v, m=None):
    n = len(rp) - 1
    d = np.zeros((n, m or n))
    d[np.repeat(np.arange(n), np.diff(rp)), ci] = v
    return d
