"""The allocation-free FP32 half-step (als_half_step_static, scratch in a
file-scope device array) against the workspace entry point als_half_step on the
same seeded inputs, on two calls in a row, plus its size limit. The entry point
exists for callers that cannot call cudaMalloc (their GPU memory belongs to a
pooling allocator, or they must avoid the synchronisation an allocation can
cause); the second call checks that the shared array's leftover contents from
the first call do not leak into the result.

Tolerance: the FP32 form's, per-row relative L2 difference <= 1e-3 (both
entries run the same kernel, so the results normally agree exactly)."""
import ctypes

import numpy as np
import pytest
import torch

import als_b200 as A

pytestmark = pytest.mark.gpu
TOL = 1e-3
MAX_ROWS = 1048576  # ALS_STATIC_MAX_ROWS

c_i32, c_i64, c_f32, c_vp = ctypes.c_int32, ctypes.c_int64, ctypes.c_float, ctypes.c_void_p
_static = A.lib.als_half_step_static
_static.restype = c_i32
_static.argtypes = [c_i64, c_i64, c_i32, c_vp, c_vp, c_vp, c_vp, c_i32, c_vp, c_i32, c_f32, c_vp,
                    c_vp]


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _rel_rows(X, ref):
    den = np.maximum(np.linalg.norm(ref, axis=1), 1e-30)
    return np.linalg.norm(X - ref, axis=1) / den


def _static_call(ptr, col, val, src, dst, lam, opts):
    m = ptr.shape[0] - 1
    n, f = src.shape
    return _static(m, n, f, _p(ptr), _p(col), _p(val), _p(src), src.stride(0), _p(dst),
                   dst.stride(0), lam, ctypes.byref(opts), None)


@pytest.mark.parametrize("f", [10, 100])
def test_static_half_step_matches_workspace_entry(f):
    r = A.synth(A.scaled_config("ml1m", 0.15), seed=23)
    lam = 0.05
    opts = A.options()
    dev = torch.device("cuda")
    ptr = torch.from_numpy(r.csr_ptr).to(dev)
    col = torch.from_numpy(r.csr_col).to(dev)
    val = torch.from_numpy(r.csr_val).to(dev)
    src = torch.from_numpy(A.init_factors(r.n, f, 5).astype(np.float32)).to(dev)
    ref = torch.zeros(r.m, f, device=dev)
    A.half_step(ptr, col, val, src, ref, lam, opts)
    torch.cuda.synchronize()
    ref_h = ref.cpu().numpy().astype(np.float64)
    for call in range(2):
        out = torch.full((r.m, f), float("nan"), device=dev)
        rc = _static_call(ptr, col, val, src, out, lam, opts)
        assert rc == 0, A.lib.als_last_error()
        torch.cuda.synchronize()
        X = out.cpu().numpy().astype(np.float64)
        assert np.isfinite(X).all(), call
        assert _rel_rows(X, ref_h).max() < TOL, call


def test_static_half_step_matches_oracle():
    """The allocation-free entry against the FP64 oracle directly, at the FP32
    form's tolerance, on a case with empty and single-rating rows."""
    import oracle as O
    r = A.synth(A.scaled_config("ml1m", 0.1), seed=29)
    f, lam = 16, 0.05
    dev = torch.device("cuda")
    ptr = torch.from_numpy(r.csr_ptr).to(dev)
    col = torch.from_numpy(r.csr_col).to(dev)
    val = torch.from_numpy(r.csr_val).to(dev)
    th = A.init_factors(r.n, f, 9).astype(np.float32)
    src = torch.from_numpy(th).to(dev)
    out = torch.full((r.m, f), float("nan"), device=dev)
    assert _static_call(ptr, col, val, src, out, lam, A.options()) == 0, A.lib.als_last_error()
    torch.cuda.synchronize()
    ref, _ = O.half_step(r.csr_ptr, r.csr_col, r.csr_val, th, lam)
    keep = np.diff(r.csr_ptr) > 0
    X = out.cpu().numpy().astype(np.float64)
    assert _rel_rows(X[keep], ref[keep]).max() < TOL
    assert np.all(X[~keep] == 0)


def test_static_half_step_at_the_row_limit():
    """m equal to the limit: the visiting order fills its whole slot of the
    array, right up to the queue head and the counters behind it. Mostly empty
    rows with a few rated ones, two calls in a row, against als_half_step."""
    rng = np.random.default_rng(31)
    m, n, f, lam = MAX_ROWS, 64, 8, 0.05
    deg = np.zeros(m, np.int64)
    rated = rng.choice(m, 3000, replace=False)
    deg[rated] = rng.integers(1, 40, size=rated.size)
    deg[m - 1] = 5  # the last row of the order's slot carries ratings
    ptr_h = np.zeros(m + 1, np.int64)
    np.cumsum(deg, out=ptr_h[1:])
    nnz = int(ptr_h[-1])
    col_h = rng.integers(0, n, size=nnz).astype(np.int32)
    val_h = rng.integers(1, 6, size=nnz).astype(np.float32)
    dev = torch.device("cuda")
    ptr = torch.from_numpy(ptr_h).to(dev)
    col = torch.from_numpy(col_h).to(dev)
    val = torch.from_numpy(val_h).to(dev)
    src = torch.from_numpy(A.init_factors(n, f, 3).astype(np.float32)).to(dev)
    ref = torch.zeros(m, f, device=dev)
    A.half_step(ptr, col, val, src, ref, lam, A.options())
    torch.cuda.synchronize()
    ref_h = ref.cpu().numpy().astype(np.float64)
    for call in range(2):
        out = torch.full((m, f), float("nan"), device=dev)
        assert _static_call(ptr, col, val, src, out, lam, A.options()) == 0, A.lib.als_last_error()
        torch.cuda.synchronize()
        X = out.cpu().numpy().astype(np.float64)
        assert np.isfinite(X).all(), call
        keep = deg > 0
        assert _rel_rows(X[keep], ref_h[keep]).max() < TOL, call
        assert np.all(X[~keep] == 0), call


def test_static_half_step_rejects_too_many_rows():
    opts = A.options()
    # the size check comes before any pointer is used
    rc = _static(MAX_ROWS + 1, 10, 10, None, None, None, None, 10, None, 10, 0.05,
                 ctypes.byref(opts), None)
    assert rc == 1  # ALS_ERR_INVALID
    assert b"static scratch limit" in A.lib.als_last_error()
