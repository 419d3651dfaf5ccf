"""The pipelined host-buffer half-step (als_half_step_host, the path of the
Spark JNI call): ratings uploaded in row ranges, each range solved while the
next one is uploaded. Same inputs, options and result as doALSWithCSR: at this
size every split row is cut into 8192-rating pieces whatever the range, so the
result must be bit-identical to the one-shot call for every range count, for
pageable and pinned host memory, on both sides (the items side has rows of up
to 36k ratings, so split rows are among them)."""
import numpy as np
import pytest
import torch

import als_b200 as A

pytestmark = pytest.mark.gpu


def _pin(a):
    return torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()


@pytest.fixture(scope="module")
def ratings():
    return A.synth(A.scaled_config("netflix", 0.1), seed=5)


@pytest.mark.parametrize("form", ["fp32_cholesky", "bf16_cg"])
def test_host_half_step_equals_dropin(ratings, form):
    r = ratings
    f, lam = 32, 0.05
    old = A.get_dropin_options()
    try:
        if form == "bf16_cg":
            A.set_dropin_options(A.options(precision=A.PREC_BF16, solver=A.SOLVER_CG, solver_groups=3))
        else:
            A.set_dropin_options(A.options())
        th = A.init_factors(r.n, f, 3)
        sides = ((r.csr_ptr.astype(np.int32), r.csr_col, r.csr_val, r.m, r.n),
                 (r.csc_ptr.astype(np.int32), r.csc_row, r.csc_val, r.n, r.m))
        src = th
        for ptr, idx, val, rows, cols in sides:
            ref = A.do_als_with_csr(ptr, idx, val, src, rows, cols, f, lam)
            assert np.isfinite(ref).all()
            for chunks in (0, 1, 3, 8):
                X = A.half_step_host(ptr, idx, val, src, rows, cols, f, lam, chunks=chunks)
                assert np.array_equal(X, ref), (form, rows, chunks)
            # pinned inputs and a pinned X: uploads and per-range downloads go
            # directly on the streams
            Xp = _pin(np.zeros((rows, f), np.float32))
            out = A.half_step_host(_pin(ptr), _pin(idx), _pin(val), _pin(src), rows, cols, f, lam,
                                   out=Xp, chunks=5)
            assert out is Xp and np.array_equal(Xp, ref), (form, rows)
            src = ref
    finally:
        A.set_dropin_options(old)


def test_host_half_step_empty_rows_and_no_ratings():
    """Rows without ratings get x_u = 0; a matrix without ratings gives X = 0."""
    f = 16
    th = A.init_factors(5, f, 1)
    ptr = np.array([0, 0, 2, 2, 3], np.int32)
    col = np.array([0, 4, 2], np.int32)
    val = np.array([4.0, 3.0, 5.0], np.float32)
    X = A.half_step_host(ptr, col, val, th, 4, 5, f, 0.05, chunks=3)
    ref = A.do_als_with_csr(ptr, col, val, th, 4, 5, f, 0.05)
    assert np.array_equal(X, ref)
    assert not X[0].any() and not X[2].any() and X[1].any() and X[3].any()
    Z = A.half_step_host(np.zeros(4, np.int32), np.zeros(0, np.int32), np.zeros(0, np.float32),
                         th, 3, 5, f, 0.05, chunks=2)
    assert not Z.any()
