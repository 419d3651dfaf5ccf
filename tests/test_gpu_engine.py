"""GPU parity of the engine's FP32 form against the FP64 oracle (same seeded
inputs): one half-step at several ranks, rows of edge degrees, both sides,
the stand-alone and drop-in entry points, RMSE/predict, and full training.

Tolerance (FP32 form): per-row relative L2 error <= 1e-3 against the FP64
oracle, test RMSE within 0.1%."""
import numpy as np
import pytest
import torch

import als_b200 as A
import oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-3


def rel_rows(X, ref):
    X = np.asarray(X, np.float64)
    den = np.maximum(np.linalg.norm(ref, axis=1), 1e-30)
    num = np.linalg.norm(X - ref, axis=1)
    num[np.linalg.norm(ref, axis=1) == 0] = np.linalg.norm(X, axis=1)[np.linalg.norm(ref, axis=1) == 0]
    return num / den


@pytest.fixture(scope="module")
def ml_small():
    return A.synth(A.scaled_config("ml1m", 0.15), seed=21)


@pytest.mark.parametrize("f", [1, 7, 10, 16, 20, 32, 50, 64, 100, 128])
def test_fp32_half_step_both_sides(ml_small, f):
    r = ml_small
    th0 = A.init_factors(r.n, f, 3)
    M = A.Model(r, f, A.options(), theta0=th0)
    M.half_step(A.SIDE_USERS, 0.05)
    X = M.factors()[0].cpu().numpy()
    X_ref, _ = O.half_step(r.csr_ptr, r.csr_col, r.csr_val, th0, 0.05)
    assert rel_rows(X, X_ref).max() < TOL
    M.half_step(A.SIDE_ITEMS, 0.05)
    T = M.factors()[1].cpu().numpy()
    T_ref, _ = O.half_step(r.csc_ptr, r.csc_row, r.csc_val, X.astype(np.float64), 0.05)
    assert rel_rows(T, T_ref).max() < TOL
    st = M.stats()
    assert st["rows_solved"] == r.m + r.n and st["rows_not_spd"] == 0
    M.close()


def _edge_csr(n, degrees, seed=0):
    rng = np.random.default_rng(seed)
    ptr = np.zeros(len(degrees) + 1, np.int64)
    ptr[1:] = np.cumsum(degrees)
    col = np.concatenate([np.sort(rng.choice(n, d, replace=False)) for d in degrees]
                         + [np.zeros(0, np.int64)]).astype(np.int32)
    val = rng.integers(1, 6, len(col)).astype(np.float32)
    return ptr, col, val


@pytest.mark.parametrize("f", [10, 100, 128])
def test_edge_degrees(f):
    """Rows with 0 ratings (x=0), with fewer ratings than f (regularisation
    carries the system), at staging-window edges, and very long rows."""
    n = 30000
    degrees = [0, 1, 2, 7, 8, 9, 23, 24, 25, 31, 32, 33, 63, 64, 65, 99, 100, 101, 1000, 20000, 0]
    ptr, col, val = _edge_csr(n, degrees, seed=f)
    th = A.init_factors(n, f, 9)
    dev = lambda a: torch.from_numpy(a).cuda()
    src = dev(th)
    dst = torch.full((len(degrees), f), float("nan"), device="cuda")
    A.half_step(dev(ptr), dev(col), dev(val), src, dst, 0.05)
    X = dst.cpu().numpy()
    X_ref, _ = O.half_step(ptr, col, val, th, 0.05)
    assert np.all(X[0] == 0) and np.all(X[-1] == 0)
    assert rel_rows(X, X_ref).max() < TOL


def test_strided_factors():
    """Caller factors with a row stride larger than f."""
    r = A.synth(A.scaled_config("ml1m", 0.08), seed=4)
    f = 12
    th = A.init_factors(r.n, f, 1)
    big = np.zeros((r.n, 20), np.float32)
    big[:, :f] = th
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    src = dev(big)[:, :f]
    out = torch.zeros((r.m, 17), device="cuda")
    A.half_step(dev(r.csr_ptr), dev(r.csr_col), dev(r.csr_val), src, out[:, :f], 0.05)
    X_ref, _ = O.half_step(r.csr_ptr, r.csr_col, r.csr_val, th, 0.05)
    assert rel_rows(out[:, :f].cpu().numpy(), X_ref).max() < TOL
    assert torch.all(out[:, f:] == 0)


@pytest.mark.parametrize("f", [10, 100])
def test_dropin_doALSWithCSR(ml_small, f):
    """The reference's entry point with int32 CSR on the device (freed by the
    callee) and host theta/X, as the Spark JNI drives it."""
    r = ml_small
    th = A.init_factors(r.n, f, 5)
    X = A.do_als_with_csr(r.csr_ptr.astype(np.int32), r.csr_col, r.csr_val, th, r.m, r.n, f, 0.05)
    X_ref, _ = O.half_step(r.csr_ptr, r.csr_col, r.csr_val, th, 0.05)
    assert rel_rows(X, X_ref).max() < TOL
    # repeated calls (each frees its CSR) keep working
    X2 = A.do_als_with_csr(r.csr_ptr.astype(np.int32), r.csr_col, r.csr_val, th, r.m, r.n, f, 0.05,
                           x_batch=3)
    assert np.array_equal(X, X2)


def test_dropin_staged_copies_match_pinned():
    """theta and X above 32 MB in pageable host memory travel through the
    drop-in's pinned staging (four host workers, two 8 MB halves each), in
    five chunks with a partial last one, so one worker reuses its first half;
    pinned host buffers are copied directly. Both give the same X,
    bit for bit, for the user side (X staged on the way down) and the item side
    (theta staged on the way up)."""
    r = A.synth(A.scaled_config("netflix", 0.2), seed=4)
    f, lam = 100, 0.05
    pin = lambda a: torch.from_numpy(a).pin_memory().numpy()
    th = A.init_factors(r.n, f, 5)
    ptr32, cptr32 = r.csr_ptr.astype(np.int32), r.csc_ptr.astype(np.int32)
    X_pg = A.do_als_with_csr(ptr32, r.csr_col, r.csr_val, th, r.m, r.n, f, lam)
    assert X_pg.nbytes > 32 << 20 and X_pg.nbytes % (16 << 20)
    X_pin = A.do_als_with_csr(ptr32, r.csr_col, r.csr_val, pin(th), r.m, r.n, f, lam,
                              out=pin(np.zeros((r.m, f), np.float32)))
    assert np.isfinite(X_pg).all() and np.array_equal(X_pg, X_pin)
    T_pg = A.do_als_with_csr(cptr32, r.csc_row, r.csc_val, X_pg, r.n, r.m, f, lam)
    T_pin = A.do_als_with_csr(cptr32, r.csc_row, r.csc_val, pin(X_pg), r.n, r.m, f, lam,
                              out=pin(np.zeros((r.n, f), np.float32)))
    assert np.isfinite(T_pg).all() and np.array_equal(T_pg, T_pin)
    X_ref, _ = O.half_step(r.csr_ptr[:2001], r.csr_col, r.csr_val, th, lam)
    assert rel_rows(X_pg[:2000], X_ref).max() < TOL


def test_rmse_and_predict(ml_small):
    r, f = ml_small, 16
    rng = np.random.default_rng(0)
    X = rng.standard_normal((r.m, f)).astype(np.float32)
    T = rng.standard_normal((r.n, f)).astype(np.float32)
    dev = lambda a: torch.from_numpy(a).cuda()
    got = A.rmse(dev(r.test_u), dev(r.test_i), dev(r.test_r), dev(X), dev(T))
    want = O.rmse(r.test_u, r.test_i, r.test_r, X, T)
    assert abs(got - want) <= 1e-6 * want
    p = A.predict(dev(r.test_u), dev(r.test_i), dev(X), dev(T)).cpu().numpy()
    np.testing.assert_allclose(p, np.einsum("ij,ij->i", X[r.test_u].astype(np.float64),
                                            T[r.test_i].astype(np.float64)), rtol=1e-4, atol=1e-4)
    assert A.rmse(dev(r.test_u[:0]), dev(r.test_i[:0]), dev(r.test_r[:0]), dev(X), dev(T)) == 0.0


def test_full_training_matches_oracle():
    """10 ALS iterations at the MovieLens-1M shape, f=10, lambda=0.05."""
    cfg = A.CONFIGS["ml1m"]
    r = A.synth(cfg, seed=1)
    f, lam, iters = cfg["f"], cfg["lam"], cfg["iters"]
    th0 = A.init_factors(r.n, f, 2)
    M = A.Model(r, f, A.options(), theta0=th0)
    M.iterate(lam, iters)
    X, T = (t.cpu().numpy() for t in M.factors())
    rm = M.rmse()
    Xr, Tr = O.train(r, f, lam, iters, th0)
    rm_ref = O.rmse(r.test_u, r.test_i, r.test_r, Xr, Tr)
    assert rel_rows(X, Xr).max() < TOL and rel_rows(T, Tr).max() < TOL
    assert abs(rm - rm_ref) / rm_ref < 1e-3
    # CUDA-graph replay and the host-buffer entry give the same bits
    M2 = A.Model(r, f, A.options(use_graph=1), theta0=th0, stream=torch.cuda.Stream())
    M2.iterate(lam, iters)
    torch.cuda.synchronize()
    assert np.array_equal(M2.factors()[0].cpu().numpy(), X)
    Xh, Th, st = A.train(r, f, lam, iters, th0)
    assert np.array_equal(Xh, X) and np.array_equal(Th, T)
    assert st["rows_solved"] == iters * (r.m + r.n)


def test_lambda_zero_rank_deficient_rows_flagged():
    """lambda = 0 and fewer ratings than f: A_u is singular; the row is
    flagged (not SPD) and its factor set to 0 instead of NaN."""
    n, f = 500, 16
    ptr, col, val = _edge_csr(n, [3, 40], seed=1)
    th = A.init_factors(n, f, 2)
    r = A.Ratings(2, n, ptr, col, val, *A.transpose(2, n, ptr, col, val),
                  np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros(0, np.float32))
    M = A.Model(r, f, A.options(), theta0=th)
    M.half_step(A.SIDE_USERS, 0.0)
    X = M.factors()[0].cpu().numpy()
    flags = M.row_flags(A.SIDE_USERS).cpu().numpy()
    assert np.all(np.isfinite(X))
    assert flags[0] & A.ROW_NOT_SPD and np.all(X[0] == 0)
    X_ref, _ = O.half_step(ptr, col, val, th, 0.0)
    assert rel_rows(X[1:], X_ref[1:]).max() < TOL


@pytest.mark.parametrize("prec", [A.PREC_FP32, A.PREC_BF16])
def test_row_ranges_compose(ml_small, prec):
    """Solving a side as two row ranges (what two ranks do) gives the same bits
    as solving it whole; sync_lp rebuilds the low-precision copy."""
    r, f = ml_small, 32
    th0 = A.init_factors(r.n, f, 3)
    solver = A.SOLVER_CHOLESKY
    full = A.Model(r, f, A.options(precision=prec, solver=solver), theta0=th0)
    full.half_step(A.SIDE_USERS, 0.05)
    X_full = full.factors()[0].clone()
    part = A.Model(r, f, A.options(precision=prec, solver=solver), theta0=th0)
    mid = r.m // 3
    part.set_row_range(A.SIDE_USERS, 0, mid)
    part.half_step(A.SIDE_USERS, 0.05)
    part.set_row_range(A.SIDE_USERS, mid, r.m)
    part.half_step(A.SIDE_USERS, 0.05)
    part.sync_lp(A.SIDE_USERS)
    assert torch.equal(part.factors()[0], X_full)
    full.half_step(A.SIDE_ITEMS, 0.05)
    part.set_row_range(A.SIDE_ITEMS, 0, r.n)
    part.half_step(A.SIDE_ITEMS, 0.05)
    assert torch.equal(part.factors()[1], full.factors()[1])
    with pytest.raises(A.AlsError):
        part.set_row_range(A.SIDE_USERS, 5, r.m + 1)


def test_dropin_tensor_core_form(ml_small):
    """doALSWithCSR switched to the tensor-core form (BF16 copy of theta, CG
    from zero) through the process-wide drop-in options; the FP32 default is
    restored afterwards."""
    import torch
    r, f = ml_small, 32
    th = A.init_factors(r.n, f, 5)
    old = A.get_dropin_options()
    try:
        A.set_dropin_options(A.options(precision=A.PREC_BF16, solver=A.SOLVER_CG))
        X = A.do_als_with_csr(r.csr_ptr.astype(np.int32), r.csr_col, r.csr_val, th, r.m, r.n, f,
                              0.05)
    finally:
        A.set_dropin_options(old)
    th_r = torch.from_numpy(th).to(torch.bfloat16).float().numpy().astype(np.float64)
    X_ref, _ = O.half_step(r.csr_ptr, r.csr_col, r.csr_val, th_r, 0.05)
    keep = np.diff(r.csr_ptr) > 0
    assert rel_rows(X, X_ref)[keep].max() < TOL
    assert A.get_dropin_options().precision == A.PREC_FP32
