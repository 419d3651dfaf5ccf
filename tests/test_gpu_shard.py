"""The C++ shard driver (als_shard_*: nnz-balanced row ranges, one NCCL
all-gather per half-step, RMSE by an NCCL all-reduce) on the one GPU this run
has: with one rank the NCCL path runs end to end (communicator, all-gather of
the whole side, low-precision rebuild, all-reduce of the RMSE sum) and must
leave the iteration exactly as the unsharded model computes it. The exchange
logic for several ranks is covered on CPU (tests/test_dist.py)."""
import numpy as np
import pytest
import torch

import als_b200 as A

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [A.PREC_BF16, A.PREC_FP32])
def test_one_rank_shard_equals_unsharded(prec):
    r = A.synth(A.scaled_config("netflix", 0.05), seed=17)
    f, lam = 32, 0.05
    th = A.init_factors(r.n, f, 19)
    opts = A.options(precision=prec, solver=A.SOLVER_CG if prec != A.PREC_FP32 else A.SOLVER_CHOLESKY,
                     solver_groups=2)
    ref = A.Model(r, f, opts, theta0=th)
    ref.iterate(lam, 3)
    Xr, Tr = (t.cpu().numpy() for t in ref.factors())
    rm_ref = ref.rmse()
    ref.close()

    M = A.Model(r, f, opts, theta0=th)
    sh = A.Shard(M, r, 1, 0, A.shard_unique_id())
    assert np.array_equal(sh.bounds(A.SIDE_USERS), [0, r.m])
    assert np.array_equal(sh.bounds(A.SIDE_ITEMS), [0, r.n])
    sh.iterate(lam, 2)
    sh.half_step(A.SIDE_USERS, lam)
    sh.half_step(A.SIDE_ITEMS, lam)
    X, T = (t.cpu().numpy() for t in M.factors())
    rm = sh.rmse()
    st = M.stats()
    sh.close()
    M.close()
    assert st["kernel_errors"] == 0
    assert np.array_equal(X, Xr) and np.array_equal(T, Tr)
    assert abs(rm - rm_ref) <= 1e-12 * max(1.0, rm_ref), (rm, rm_ref)


def test_shard_rejects_dimensions_other_than_the_models():
    """m, n or f that differ from the model's are ALS_ERR_INVALID before any
    communicator is made."""
    import ctypes
    r = A.synth(A.scaled_config("ml1m", 0.05), seed=3)
    M = A.Model(r, 16, A.options(precision=A.PREC_BF16, solver=A.SOLVER_CG), theta0=A.init_factors(r.n, 16, 1))
    csr = np.ascontiguousarray(r.csr_ptr, np.int64)
    csc = np.ascontiguousarray(r.csc_ptr, np.int64)
    idbuf = ctypes.create_string_buffer(A.shard_unique_id(), 128)
    h = ctypes.c_void_p()
    for m, n, f in ((r.m + 1, r.n, 16), (r.m, r.n - 1, 16), (r.m, r.n, 32)):
        rc = A.lib.als_shard_create(ctypes.byref(h), M.handle, csr.ctypes.data, csc.ctypes.data,
                                    m, n, f, 1, 0, idbuf, M.stream)
        assert rc == 1 and not h.value and b"differ" in A.lib.als_last_error()
    M.close()
