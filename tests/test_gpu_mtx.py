"""MatrixMarket files into the engine (-m gpu): hamlss_mat_load_mtx uploads what the reader
parses (SpMV bit for bit against the oracle on the same CSR), and the dataset runner solves
written problems to tolerance through the adaptive ladder."""
import ctypes as C
import os

import numpy as np
import pytest

from gpu_util import need_gpu
import hsps_b200 as H
from hsps_b200 import _abi
from hsps_b200 import problems as P
from hsps_b200.mtx import MatrixMarketIO as MM, run_dataset

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    need_gpu()


def test_load_mtx_to_device(orc, tmp_path):
    rp, ci, v = P.varkappa_poisson_2d(40, 1.0, 4)
    n = 40 * 40
    A = H.SparseMatrix(n, n, rp, ci, v)
    f = str(tmp_path / "k.mtx")
    MM.save_matrix(f, A)
    ctx = H.Context.default()
    h = C.c_void_p()
    assert H.lib().hamlss_mat_load_mtx(ctx.h, f.encode(), C.byref(h)) == 0
    rows, cols, rp2, ci2, v2 = MM.read_csr(f)
    x = P.rhs(n, 5, -1, 1)
    y = np.zeros(n)
    assert H.lib().hamlss_spmv(ctx.h, h, x.ctypes.data, y.ctypes.data, _abi.HOST) == 0
    assert np.array_equal(y, orc.spmv(rp2, ci2, v2, x))
    H.lib().hamlss_mat_release(h)


def test_run_dataset_solves_written_problems(orc, tmp_path):
    probs = {"poisson30": P.poisson_2d(30),
             "convdiff24": P.convection_diffusion_2d(24, 1.0, *P.convdiff_wind(24, 10.0))}
    for name, (rp, ci, v) in probs.items():
        n = len(rp) - 1
        MM.save_matrix(str(tmp_path / f"{name}.mtx"), H.SparseMatrix(n, n, rp, ci, v))
        MM.save_vector(str(tmp_path / f"{name}_rhs.mtx"), P.rhs(n, 3))
    rows = run_dataset(str(tmp_path), verbose=False)
    assert [r["name"] for r in rows] == sorted(probs)
    for r in rows:
        assert "error" not in r and r["converged"] and r["rel_res"] < 1e-7, r
