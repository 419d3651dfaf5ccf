"""GPU parity of the tensor-core form (tcgen05 SYRK, BF16/FP16 factor copies,
FP32 accumulation) with CG or Cholesky solves.

Two comparisons per case:
  kernel parity    against the FP64 oracle run on the same rounded factors
                   (BF16/FP16 round-to-nearest of theta): the kernel must solve
                   that system; tolerance 1e-3 per-row relative L2 error
                   (Cholesky, and CG to relative residual 1e-5);
  precision effect against the FP64 oracle on the unrounded factors; stated
                   tolerance 3e-2 (BF16) / 5e-3 (FP16) per-row relative error
                   at the 99th percentile.
"""
import numpy as np
import pytest
import torch

import als_b200 as A
import oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-3
PREC_TOL = {A.PREC_BF16: 3e-2, A.PREC_FP16: 5e-3}


def rnd(x, prec):
    t = torch.from_numpy(np.ascontiguousarray(x, np.float32))
    dt = torch.bfloat16 if prec == A.PREC_BF16 else torch.float16
    return t.to(dt).to(torch.float32).numpy().astype(np.float64)


def rel_rows(X, ref):
    den = np.maximum(np.linalg.norm(ref, axis=1), 1e-30)
    return np.linalg.norm(np.asarray(X, np.float64) - ref, axis=1) / den


@pytest.fixture(scope="module")
def data():
    return A.synth(A.scaled_config("netflix", 0.03), seed=5)


@pytest.mark.parametrize("prec", [A.PREC_BF16, A.PREC_FP16])
@pytest.mark.parametrize("solver", [A.SOLVER_CHOLESKY, A.SOLVER_CG])
@pytest.mark.parametrize("f", [16, 20, 31, 32, 47, 64, 72, 96, 100, 104, 110, 120, 128])
def test_tc_half_step(data, f, prec, solver):
    r = data
    th0 = A.init_factors(r.n, f, 7)
    opts = A.options(precision=prec, solver=solver, warm_start=A.WARM_ZERO)
    M = A.Model(r, f, opts, theta0=th0)
    M.half_step(A.SIDE_USERS, 0.05)
    X = M.factors()[0].cpu().numpy()
    st = M.stats()
    assert st["kernel_errors"] == 0
    X_r, _ = O.half_step(r.csr_ptr, r.csr_col, r.csr_val, rnd(th0, prec), 0.05)
    err = rel_rows(X, X_r)
    keep = np.diff(r.csr_ptr) > 0
    assert err[keep].max() < TOL, (err.max(), st)
    assert np.all(X[~keep] == 0)
    X_e, _ = O.half_step(r.csr_ptr, r.csr_col, r.csr_val, th0, 0.05)
    assert np.quantile(rel_rows(X, X_e)[keep], 0.99) < PREC_TOL[prec]
    # items side from the new X (its low-precision copy)
    M.half_step(A.SIDE_ITEMS, 0.05)
    T = M.factors()[1].cpu().numpy()
    T_r, _ = O.half_step(r.csc_ptr, r.csc_row, r.csc_val, rnd(X, prec), 0.05)
    assert rel_rows(T, T_r).max() < TOL
    if solver == A.SOLVER_CG:
        st = M.stats()
        assert st["cg_steps"] > 0
    M.close()


@pytest.mark.parametrize("prec", [A.PREC_BF16, A.PREC_FP16])
def test_tc_edge_degrees(prec):
    n, f = 30000, 100
    rng = np.random.default_rng(3)
    degrees = [0, 1, 15, 16, 17, 63, 64, 65, 127, 128, 129, 20000, 0, 3]
    ptr = np.zeros(len(degrees) + 1, np.int64)
    ptr[1:] = np.cumsum(degrees)
    col = np.concatenate([np.sort(rng.choice(n, d, replace=False)) for d in degrees]).astype(np.int32)
    val = rng.integers(1, 6, len(col)).astype(np.float32)
    cp, cr, cv = A.transpose(len(degrees), n, ptr, col, val)
    r = A.Ratings(len(degrees), n, ptr, col, val, cp, cr, cv, np.zeros(0, np.int32),
                  np.zeros(0, np.int32), np.zeros(0, np.float32))
    th = A.init_factors(n, f, 2)
    for solver in (A.SOLVER_CHOLESKY, A.SOLVER_CG):
        M = A.Model(r, f, A.options(precision=prec, solver=solver, warm_start=A.WARM_ZERO),
                    theta0=th)
        M.half_step(A.SIDE_USERS, 0.05)
        X = M.factors()[0].cpu().numpy()
        X_r, _ = O.half_step(ptr, col, val, rnd(th, prec), 0.05)
        assert np.all(X[0] == 0) and np.all(X[12] == 0)
        keep = np.array(degrees) > 0
        assert rel_rows(X, X_r)[keep].max() < TOL
        M.close()


def test_tc_training_rmse_close_to_fp64():
    """Mixed-precision training (BF16 and FP16 factors, CG with the previous
    iterate as warm start) reaches a test RMSE within 0.1% of FP64 ALS."""
    cfg = A.scaled_config("netflix", 0.05)
    r = A.synth(cfg, seed=9)
    f, lam, iters = 100, 0.05, 6
    th0 = A.init_factors(r.n, f, 3)
    Xr, Tr = O.train(r, f, lam, iters, th0)
    rm_ref = O.rmse(r.test_u, r.test_i, r.test_r, Xr, Tr)
    for prec in (A.PREC_BF16, A.PREC_FP16):
        M = A.Model(r, f, A.options(precision=prec, solver=A.SOLVER_CG), theta0=th0)
        M.iterate(lam, iters)
        rm = M.rmse()
        st = M.stats()
        assert st["kernel_errors"] == 0
        assert abs(rm - rm_ref) / rm_ref < 1e-3, (prec, rm, rm_ref, st)
        M.close()


@pytest.mark.parametrize("f", [100, 48, 120, 128])
def test_solver_groups_agree_with_oracle(f):
    """The hot kernel with 1, 2 and 3 solver warpgroups (and the autotuner) on
    a matrix with multi-stage rows and item rows long enough to be split
    across CTAs: every configuration gives the same bits, and both sides match
    the FP64 oracle on the BF16-rounded factors (tolerance 1e-3). This covers
    the producers' alternate stages and the per-group row hand-over, and both
    placements of a row's system (registers with one or two warpgroups up to
    f = 112 and with one above it, TMEM otherwise), which must agree bit for
    bit. f = 120 and 128 use the three-atom stages and three accumulators."""
    r = A.synth(A.scaled_config("netflix", 0.1), seed=7)
    assert np.diff(r.csc_ptr).max() > 8192  # some item rows are split
    th = A.init_factors(r.n, f, 11)
    out = {}
    for ng in (1, 2, 3, 0):
        M = A.Model(r, f, A.options(precision=A.PREC_BF16, solver=A.SOLVER_CG,
                                    warm_start=A.WARM_ZERO, solver_groups=ng), theta0=th)
        M.half_step(A.SIDE_USERS, 0.05)
        M.half_step(A.SIDE_ITEMS, 0.05)
        X, T = (t.cpu().numpy() for t in M.factors())
        st = M.stats()
        M.close()
        assert st["kernel_errors"] == 0, (ng, st)
        assert st["rows_solved"] == r.m + r.n
        out[ng] = (X, T)
    for ng in (2, 3, 0):
        assert np.array_equal(out[ng][0], out[1][0]) and np.array_equal(out[ng][1], out[1][1]), ng
    X, T = out[1]
    Xr, _ = O.half_step(r.csr_ptr, r.csr_col, r.csr_val, rnd(th, A.PREC_BF16), 0.05)
    assert rel_rows(X, Xr).max() < TOL
    Tr, _ = O.half_step(r.csc_ptr, r.csc_row, r.csc_val, rnd(X, A.PREC_BF16), 0.05)
    assert rel_rows(T, Tr).max() < TOL


@pytest.mark.parametrize("f", [100, 128])
@pytest.mark.parametrize("ng", [1, 2, 3])
def test_cg_fallback_rows_match_oracle(f, ng):
    """CG limited to two steps, so most rows cannot finish: up to f = 112 they
    are solved by the kernel's own register-tile Cholesky (the system copied
    from registers or from TMEM into the tile), above it by the post-pass of
    the one-CTA-per-row kernel. Every row still matches the FP64 oracle on
    the BF16-rounded factors (1e-3) and carries the CG-fallback status bit;
    Jacobi-preconditioned CG (f = 100) takes the same fallback."""
    r = A.synth(A.scaled_config("netflix", 0.03), seed=17)
    th = A.init_factors(r.n, f, 19)
    Xr, _ = O.half_step(r.csr_ptr, r.csr_col, r.csr_val, rnd(th, A.PREC_BF16), 0.05)
    keep = np.diff(r.csr_ptr) > 0
    for jac in ((0, 1) if f <= 112 else (0,)):
        M = A.Model(r, f, A.options(precision=A.PREC_BF16, solver=A.SOLVER_CG, warm_start=A.WARM_ZERO,
                                    cg_max_steps=2, cg_jacobi=jac, solver_groups=ng), theta0=th)
        M.half_step(A.SIDE_USERS, 0.05)
        X = M.factors()[0].cpu().numpy()
        flags = M.row_flags(A.SIDE_USERS).cpu().numpy()
        st = M.stats()
        M.close()
        assert st["kernel_errors"] == 0 and st["rows_solved"] == r.m, st
        assert st["cg_fallbacks"] > r.m // 2, st
        fb = (flags & A.ROW_CG_FALLBACK) != 0
        assert fb.sum() == st["cg_fallbacks"]
        assert rel_rows(X, Xr)[keep].max() < TOL, (jac, rel_rows(X, Xr)[keep].max())


def test_wide_rank_runs_on_the_warp_specialised_kernel():
    """At f = 128 the CG form runs on the warp-specialised kernel: its
    autotuner (which only that kernel has) settles on a warpgroup count for
    each side after three half-steps, and the result matches the oracle."""
    r = A.synth(A.scaled_config("netflix", 0.05), seed=23)
    f = 128
    th = A.init_factors(r.n, f, 29)
    M = A.Model(r, f, A.options(precision=A.PREC_BF16, solver=A.SOLVER_CG, warm_start=A.WARM_ZERO),
                theta0=th)
    for _ in range(3):
        M.half_step(A.SIDE_USERS, 0.05)
    X = M.factors()[0].cpu().numpy()
    st = M.stats()
    M.close()
    assert st["solver_groups"][0] in (1, 2), st
    Xr, _ = O.half_step(r.csr_ptr, r.csr_col, r.csr_val, rnd(th, A.PREC_BF16), 0.05)
    keep = np.diff(r.csr_ptr) > 0
    assert rel_rows(X, Xr)[keep].max() < TOL


def test_bounded_wait_gives_up_and_the_next_half_step_is_clean():
    """The kernels' waits are bounded. A test switch makes the first CTA's MMA
    issuer stop after its first row without marking that row's accumulator
    complete (a flag that nothing sets): the solvers and producers waiting on
    it give up after their 2 s limit, every role leaves its loop, the kernel
    returns with the error word set, and the host reads kernel_errors == 1.
    No fault, no hang: the same model's next half-step runs normally and
    matches the oracle."""
    import time
    r = A.synth(A.scaled_config("netflix", 0.03), seed=41)
    f = 32
    th = A.init_factors(r.n, f, 43)
    M = A.Model(r, f, A.options(precision=A.PREC_BF16, solver=A.SOLVER_CG, warm_start=A.WARM_ZERO,
                                solver_groups=2), theta0=th)
    torch.cuda.synchronize()
    assert A.lib.als_debug_withhold_first_row(1) == 0
    t0 = time.time()
    M.half_step(A.SIDE_USERS, 0.05)
    torch.cuda.synchronize()
    dt = time.time() - t0
    st = M.stats(reset=True)
    assert st["kernel_errors"] == 1, st
    assert 1.5 < dt < 60, dt  # the wait ran to its limit, and no longer
    M.half_step(A.SIDE_USERS, 0.05)
    X = M.factors()[0].cpu().numpy()
    st = M.stats()
    M.close()
    assert st["kernel_errors"] == 0 and st["rows_solved"] == r.m, st
    Xr, _ = O.half_step(r.csr_ptr, r.csr_col, r.csr_val, rnd(th, A.PREC_BF16), 0.05)
    keep = np.diff(r.csr_ptr) > 0
    assert rel_rows(X, Xr)[keep].max() < TOL
