"""Serving-side and data-format entry points on the GPU: top-k recommendation
against numpy (the k best items by x_u . theta_i, rated items left out), and
the device CSR -> CSC transpose against the host transpose (bit for bit).

Tolerance (top-k): scores within 1e-5 relative of numpy's FP64 dot products;
the item lists must agree except where numpy's scores tie within that
tolerance."""
import numpy as np
import pytest
import torch

import als_b200 as A

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("f,k,exclude", [(100, 10, True), (16, 100, True), (33, 256, False),
                                         (7, 1, True)])
def test_topk_matches_numpy(f, k, exclude):
    r = A.synth(A.scaled_config("ml1m", 0.3), seed=13)
    rng = np.random.default_rng(4)
    X = (rng.standard_normal((r.m, f)) * 0.3).astype(np.float32)
    T = (rng.standard_normal((r.n, f)) * 0.3).astype(np.float32)
    users = np.concatenate([rng.choice(r.m, 300, replace=False), [0, r.m - 1]]).astype(np.int32)
    dev = torch.device("cuda")
    seen = (torch.from_numpy(r.csr_ptr).to(dev), torch.from_numpy(r.csr_col).to(dev)) if exclude else (None, None)
    items, scores = A.topk(torch.from_numpy(users).to(dev), torch.from_numpy(X).to(dev),
                           torch.from_numpy(T).to(dev), k, *seen)
    items, scores = items.cpu().numpy(), scores.cpu().numpy()
    full = X[users].astype(np.float64) @ T.T.astype(np.float64)
    for q, u in enumerate(users):
        s = full[q].copy()
        if exclude:
            s[r.csr_col[r.csr_ptr[u]:r.csr_ptr[u + 1]]] = -np.inf
        order = np.lexsort((np.arange(r.n), -s))[:k]
        ref = s[order]
        valid = np.isfinite(ref)
        assert (items[q][~valid] == -1).all()
        got = items[q][valid]
        assert np.allclose(scores[q][valid], ref[valid], rtol=1e-5, atol=1e-5), q
        # same items, except where numpy's scores tie within the tolerance
        mismatch = got != order[valid]
        if mismatch.any():
            assert np.allclose(s[got[mismatch]], s[order[valid][mismatch]], rtol=1e-5, atol=1e-5), q
        assert not (exclude and np.isin(got, r.csr_col[r.csr_ptr[u]:r.csr_ptr[u + 1]]).any())


@pytest.mark.parametrize("cfg,scale", [("ml1m", 0.3), ("netflix", 0.05)])
def test_device_transpose_equals_host(cfg, scale):
    r = A.synth(A.scaled_config(cfg, scale), seed=17)
    dev = torch.device("cuda")
    cptr, rows, vals = A.csr_to_csc(r.m, r.n, torch.from_numpy(r.csr_ptr).to(dev),
                                    torch.from_numpy(r.csr_col).to(dev),
                                    torch.from_numpy(r.csr_val).to(dev))
    hp, hr, hv = A.transpose(r.m, r.n, r.csr_ptr, r.csr_col, r.csr_val)
    assert np.array_equal(cptr.cpu().numpy(), hp)
    assert np.array_equal(rows.cpu().numpy(), hr)
    assert np.array_equal(vals.cpu().numpy(), hv)


def test_device_transpose_edge_shapes():
    dev = torch.device("cuda")
    # empty rows and columns, one rating, and no ratings at all
    ptr = np.array([0, 0, 2, 2, 3], np.int64)
    col = np.array([4, 1, 4], np.int32)
    val = np.array([1.5, 2.5, 3.5], np.float32)
    cptr, rows, vals = A.csr_to_csc(4, 6, torch.from_numpy(ptr).to(dev),
                                    torch.from_numpy(col).to(dev), torch.from_numpy(val).to(dev))
    assert cptr.cpu().tolist() == [0, 0, 1, 1, 1, 3, 3]
    assert rows.cpu().tolist() == [1, 1, 3]
    assert vals.cpu().tolist() == [2.5, 1.5, 3.5]
    cptr, rows, vals = A.csr_to_csc(3, 2, torch.zeros(4, dtype=torch.int64, device=dev),
                                    torch.zeros(0, dtype=torch.int32, device=dev),
                                    torch.zeros(0, dtype=torch.float32, device=dev))
    assert cptr.cpu().tolist() == [0, 0, 0]
