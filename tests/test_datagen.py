"""Seeded synthetic data: determinism, shapes, degree laws, split, transpose,
and the reference's raw binary CSR format."""
import os

import numpy as np
import pytest
import scipy.sparse as sp

import als_b200 as A


@pytest.fixture(scope="module")
def small():
    return A.synth(A.scaled_config("ml1m", 0.2), seed=11)


def test_same_seed_same_bytes_any_thread_count(small):
    again = A.synth(A.scaled_config("ml1m", 0.2), seed=11, threads=3)
    for k in ("csr_ptr", "csr_col", "csr_val", "csc_ptr", "csc_row", "csc_val", "test_u",
              "test_i", "test_r"):
        assert np.array_equal(getattr(small, k), getattr(again, k)), k


def test_different_seed_differs(small):
    other = A.synth(A.scaled_config("ml1m", 0.2), seed=12)
    assert not np.array_equal(other.csr_col[:1000], small.csr_col[:1000])


def test_csr_well_formed(small):
    r = small
    assert r.csr_ptr[0] == 0 and np.all(np.diff(r.csr_ptr) >= 0)
    assert r.csr_col.min() >= 0 and r.csr_col.max() < r.n
    for u in range(0, r.m, 37):  # sorted, no repeats within a row
        c = r.csr_col[r.csr_ptr[u]:r.csr_ptr[u + 1]]
        assert np.all(np.diff(c) > 0)
    assert set(np.unique(r.csr_val)) <= {1.0, 2.0, 3.0, 4.0, 5.0}


def test_degrees_hit_target():
    c = A.scaled_config("ml1m", 0.5)
    r = A.synth(c, seed=5)
    total = r.nnz + len(r.test_r)
    assert abs(total - c["target_nnz"]) / c["target_nnz"] < 0.01
    deg = np.diff(r.csr_ptr) + np.bincount(r.test_u, minlength=r.m)
    assert deg.min() >= min(c["degree_min"], r.n)


def test_split_fraction_and_disjoint(small):
    r = small
    frac = len(r.test_r) / (len(r.test_r) + r.nnz)
    assert abs(frac - 0.10) < 0.01
    train = set(zip(np.repeat(np.arange(r.m), np.diff(r.csr_ptr)).tolist(), r.csr_col.tolist()))
    test = set(zip(r.test_u.tolist(), r.test_i.tolist()))
    assert not (train & test)


def test_transpose_matches_scipy(small):
    r = small
    M = sp.csr_matrix((r.csr_val, r.csr_col, r.csr_ptr), shape=(r.m, r.n)).tocsc()
    assert np.array_equal(M.indptr, r.csc_ptr)
    assert np.array_equal(M.indices, r.csc_row)
    assert np.array_equal(M.data, r.csc_val)


def test_transpose_empty_rows_and_columns():
    ptr = np.array([0, 0, 2, 2, 3], np.int64)
    col = np.array([1, 3, 1], np.int32)
    val = np.array([1, 2, 3], np.float32)
    cp, rows, vals = A.transpose(4, 5, ptr, col, val)
    assert cp.tolist() == [0, 0, 2, 2, 3, 3]
    assert rows.tolist() == [1, 3, 1] and vals.tolist() == [1, 3, 2]


def test_zipf_popularity_is_skewed(small):
    deg = np.sort(np.diff(small.csc_ptr))[::-1]
    assert deg[0] > 10 * np.median(deg)


def test_powerlaw_degrees():
    c = A.scaled_config("yahoo", 0.01)
    r = A.synth(c, seed=2)
    deg = np.diff(r.csr_ptr) + np.bincount(r.test_u, minlength=r.m)
    assert deg.max() <= c["degree_max"]
    assert np.median(deg) < deg.mean()  # heavy tail
    assert r.csr_val.min() >= 0 and r.csr_val.max() <= 100


def test_tall_skinny_row_scaled():
    """The 3.1-billion-rating tall-skinny shape with a thousandth of its users:
    all 39,781 items kept, mean user degree ~62, float ratings in [0, 5], 1%
    held out, and the row and item sums of the two orientations agree."""
    c = A.row_scaled_config("hugewiki", 0.001)
    assert c["n"] == A.CONFIGS["hugewiki"]["n"] and c["m"] == 50_082
    r = A.synth(c, seed=3)
    assert r.n == 39_781 and r.m == 50_082
    total = r.nnz + len(r.test_r)
    assert 55 < total / r.m < 70
    assert 0.007 < len(r.test_r) / total < 0.013
    assert r.csr_val.min() >= 0.0 and r.csr_val.max() <= 5.0
    assert not np.all(r.csr_val == np.round(r.csr_val))  # float ratings
    assert r.csc_ptr[-1] == r.nnz
    assert np.array_equal(np.bincount(r.csc_row, minlength=r.m), np.diff(r.csr_ptr))


def test_init_factors_seeded():
    a = A.init_factors(100, 10, 3)
    b = A.init_factors(100, 10, 3, threads=2)
    assert np.array_equal(a, b)
    assert abs(a.std() - 10 ** -0.5) < 0.03


def test_binary_csr_roundtrip(tmp_path, small):
    """The raw format of the reference's loadCSRSparseMatrixBin
    (als/src/cuda/als.cu:914-933): int32 row pointers, int32 columns, float32 values."""
    r = small
    ptr32 = r.csr_ptr.astype(np.int32)
    files = [str(tmp_path / x).encode() for x in ("d.bin", "r.bin", "c.bin")]
    assert A.datalib.als_save_csr_bin(*files, A._ptr(r.csr_val), A._ptr(ptr32), A._ptr(r.csr_col),
                                      r.m, r.nnz) == 0
    assert os.path.getsize(files[1]) == 4 * (r.m + 1)
    d = np.empty(r.nnz, np.float32)
    rr = np.empty(r.m + 1, np.int32)
    cc = np.empty(r.nnz, np.int32)
    assert A.datalib.als_load_csr_bin(*files, A._ptr(d), A._ptr(rr), A._ptr(cc), r.m, r.nnz) == 0
    assert np.array_equal(d, r.csr_val) and np.array_equal(rr, ptr32) and np.array_equal(cc, r.csr_col)
    # a short file is reported instead of read past
    assert A.datalib.als_load_csr_bin(*files, A._ptr(d), A._ptr(rr), A._ptr(cc), r.m + 5, r.nnz) == -1
    missing = [b"/nonexistent/a", files[1], files[2]]
    assert A.datalib.als_load_csr_bin(*missing, A._ptr(d), A._ptr(rr), A._ptr(cc), r.m, r.nnz) == -1


def test_flop_formula_netflix_shape():
    """FLOP_iter at the Netflix shape (f=100) is 2.22e12 for ~99.1M training entries."""
    r = A.Ratings(480_189, 17_770, np.array([0, 99_100_000]), None, None, None, None, None,
                  None, None, None)
    assert abs(A.flop_per_iteration(r, 100) / 2.2174e12 - 1) < 1e-3
