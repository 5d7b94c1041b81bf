"""MatrixMarket reading and writing (host code; CPU).

Each fixture (tests/golden/mtx, written by make_mtx.py) is parsed by the engine and by the
reference's MatrixMarketIO (compiled from its sources into oracle/_ref); the CSR arrays
and vectors must agree bit for bit.  Hand-computed expectations pin the small cases, and
the project's own data/*.mtx files are compared too when that checkout is present.
"""
import glob
import os

import numpy as np
import pytest

import oracle
from hsps_b200 import _abi
from hsps_b200.mtx import MatrixMarketIO as MM

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "mtx")
MATS = ["general", "symmetric", "skew", "pattern", "integer", "truncated"]
VECS = [("vec_array", 0), ("vec_coord", 0), ("vec_nobanner", 0), ("vec_array", 6),
        ("vec_array", 2), ("vec_coord", 3)]


def path(name):
    return os.path.join(HERE, name + ".mtx")


def dense(rows, cols, rp, ci, v):
    d = np.zeros((rows, cols))
    for i in range(rows):
        for k in range(rp[i], rp[i + 1]):
            d[i, ci[k]] += v[k]
    return d


def test_hand_expectations():
    rows, cols, rp, ci, v = MM.read_csr(path("general"))
    assert (rows, cols) == (4, 5)
    want = np.zeros((4, 5))
    want[0, 0], want[0, 3], want[1, 1], want[1, 2], want[2, 1], want[3, 4] = 2, -7, 3, 0.25, -1.0, 1e-3
    assert np.array_equal(dense(rows, cols, rp, ci, v), want)
    assert list(rp) == [0, 2, 4, 5, 6]              # duplicate (3,2) summed into one entry
    _, _, rp, ci, v = MM.read_csr(path("skew"))
    d = dense(3, 3, rp, ci, v)
    assert d[1, 0] == 1.5 and d[0, 1] == -1.5 and d[2, 0] == -2 and d[0, 2] == 2
    _, _, rp, ci, v = MM.read_csr(path("pattern"))
    assert np.all(v == 1.0) and len(v) == 4
    _, _, rp, ci, v = MM.read_csr(path("truncated"))
    assert len(v) == 2                              # stops at the header's count
    assert np.array_equal(MM.load_vector(path("vec_array")), [1.0, -2.5, 300.0, 0.125])
    assert np.array_equal(MM.load_vector(path("vec_coord")), [0, 1.5, 0, 0, -3])
    # another expected size: the reference's Vector::resize assigns, so all ones
    assert np.array_equal(MM.load_vector(path("vec_array"), 6), np.ones(6))
    h = MM.read_header(path("symmetric"))
    assert h["symmetry"] == "symmetric" and h["nnz"] == 4 and h["nnz_full"] == 5
    with pytest.raises(Exception):
        MM.read_csr(path("complex"))
    with pytest.raises(Exception):
        MM.read_csr(path("nobanner"))


@pytest.fixture(scope="module")
def refio():
    if not oracle.reference_available():
        pytest.skip("reference not built from source here (oracle/_ref missing)")
    return oracle.Reference(threads=1)


@pytest.mark.parametrize("name", MATS)
def test_matrix_matches_reference(refio, name):
    mine = MM.read_csr(path(name))
    ref = refio.mtx_load_matrix(path(name))
    assert ref is not None
    assert mine[:2] == ref[:2]
    for a, b in zip(mine[2:], ref[2:]):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("name,n", VECS)
def test_vector_matches_reference(refio, name, n):
    assert np.array_equal(MM.load_vector(path(name), n), refio.mtx_load_vector(path(name), n))


def test_refused_like_reference(refio):
    for name in ("complex", "nobanner"):
        assert refio.mtx_load_matrix(path(name)) is None
        with pytest.raises(Exception):
            MM.read_csr(path(name))


def test_write_read_round_trip(tmp_path):
    rows, cols, rp, ci, v = MM.read_csr(path("general"))

    class A:  # what save_matrix needs of a SparseMatrix
        def rows(self): return rows
        def cols(self): return cols
        def row_ptr(self): return rp
        def col_idx(self): return ci
        def values(self): return v

    f = str(tmp_path / "m.mtx")
    MM.save_matrix(f, A(), "round trip")
    r2 = MM.read_csr(f)
    assert r2[:2] == (rows, cols)
    assert np.array_equal(r2[2], rp) and np.array_equal(r2[3], ci) and np.array_equal(r2[4], v)
    x = np.array([np.pi, -1e-300, 12345.678901234567, 0.0])
    g = str(tmp_path / "x.mtx")
    MM.save_vector(g, x, "solution")
    # "%.15e" (the reference's format) keeps 16 significant digits
    assert np.allclose(MM.load_vector(g), x, rtol=1e-15, atol=0)
    assert open(g).read().startswith("%%MatrixMarket matrix array real general\n% solution\n4 1\n")


# the project checkout: HSPS_REFERENCE, else a `reference` directory beside this repository
DATA = os.path.join(os.environ.get("HSPS_REFERENCE") or
                    os.path.join(os.path.dirname(os.path.dirname(os.path.dirname(
                        os.path.abspath(__file__)))), "reference"), "data")


@pytest.mark.skipif(not os.path.isdir(DATA), reason="project data directory not present")
def test_project_data_files_match_reference(refio):
    files = sorted(glob.glob(os.path.join(DATA, "*.mtx")))
    assert files
    for f in files:
        stem = os.path.basename(f)[:-4]
        if stem.endswith("_rhs"):
            a, b = MM.load_vector(f), refio.mtx_load_vector(f)
            assert np.array_equal(a, b), f
            continue
        mine, ref = MM.read_csr(f), refio.mtx_load_matrix(f)
        assert mine[:2] == ref[:2], f
        for a, b in zip(mine[2:], ref[2:]):
            assert np.array_equal(a, b), f
