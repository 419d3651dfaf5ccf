"""The learned warm start on the GPU: the hand-written forward/backward
kernels against the CPU oracle (oracle/mlp.py, BF16 rounding emulated at the
same points), training that reduces the loss, and what the trained network
gains in an ALS run: fewer CG steps than starting from zero, with the test
RMSE still within 0.1% of FP64 ALS.

Tolerances: gradients and outputs 2e-2 relative Frobenius error (BF16
activations; one-ulp rounding flips between GPU and oracle are expected)."""
import numpy as np
import pytest
import torch

import als_b200 as A
from oracle import mlp as MO
import oracle as O

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30)


def _batch(f, B, ldf, seed):
    rng = np.random.default_rng(seed)
    F = np.zeros((B, ldf), np.float32)
    F[:, :2 * f + 1] = MO.bf16(rng.standard_normal((B, 2 * f + 1)) * 0.5)
    T = (rng.standard_normal((B, f)) * 0.3).astype(np.float32)
    Fd = torch.from_numpy(F).to(torch.bfloat16).cuda()
    return F[:, :2 * f + 1].astype(np.float64), T, Fd, torch.from_numpy(T).cuda()


@pytest.mark.parametrize("f", [16, 100, 128])
def test_gradients_match_cpu_oracle(f):
    net = A.Mlp(f, capacity=256, seed=3)
    params = [p.astype(np.float64) for p in net.get_params()]
    # non-zero biases so every term is exercised
    rng = np.random.default_rng(1)
    params[1] = rng.standard_normal(256) * 0.1
    params[3] = rng.standard_normal(256) * 0.1
    params[5] = rng.standard_normal(f) * 0.1
    net.set_params([p.astype(np.float32) for p in params])
    params = [p.astype(np.float32).astype(np.float64) for p in params]
    F, T, Fd, Td = _batch(f, 128, net.ldf, 2)
    grads, loss = net.gradients(Fd, Td)
    loss_ref, ref = MO.loss_and_grads(params, F, T, emulate=True)
    assert abs(loss - loss_ref) / loss_ref < 1e-3
    for k, (g, r) in enumerate(zip(grads, ref)):
        assert _rel(g, r) < 2e-2, (k, _rel(g, r))
    Y = net.forward(Fd).cpu().numpy()
    Y_ref, _ = MO.forward(params, F, emulate=True)
    assert _rel(Y, Y_ref) < 1e-2


def test_training_reduces_loss():
    f = 16
    net = A.Mlp(f, capacity=1024, seed=4)
    rng = np.random.default_rng(5)
    B = 1024
    F = np.zeros((B, net.ldf), np.float32)
    F[:, :2 * f + 1] = MO.bf16(rng.standard_normal((B, 2 * f + 1)))
    Wt = rng.standard_normal((2 * f + 1, f)) * 0.2
    T = (F[:, :2 * f + 1] @ Wt).astype(np.float32)
    Fd = torch.from_numpy(F).to(torch.bfloat16).cuda()
    Td = torch.from_numpy(T).cuda()
    _, l0 = net.gradients(Fd, Td)
    for _ in range(300):
        net.train_step(Fd, Td, 2e-3)
    _, l1 = net.gradients(Fd, Td)
    assert l1 < 0.1 * l0, (l0, l1)


@pytest.mark.parametrize("f", [100, 128])
def test_learned_warm_start_gain_in_als(f):
    """Iterations 1-3 train the net on the solved rows; in iterations 4-6 CG
    starts from the net's x0 (scaled optimally along its direction). Compared
    with starting from zero, the starting residual is far smaller; CG step
    counts and the previous-iterate start are reported alongside. f = 128 is
    the rank of the learned-warm-start workload (first-layer width 2f+1 = 257,
    so its weight gradient spans two accumulator blocks)."""
    cfg = A.scaled_config("netflix", 0.05)
    r = A.synth(cfg, seed=9)
    lam = 0.05
    th0 = A.init_factors(r.n, f, 3)
    steps, rmse, r0 = {}, {}, {}
    for name, warm in (("zero", A.WARM_ZERO), ("previous", A.WARM_PREVIOUS), ("mlp", A.WARM_MLP)):
        M = A.Model(r, f, A.options(precision=A.PREC_BF16, solver=A.SOLVER_CG, warm_start=warm,
                                    mlp_train_iters=3, mlp_steps=48, mlp_batch=4096),
                    theta0=th0)
        M.iterate(lam, 3)
        M.stats(reset=True)
        M.iterate(lam, 3)
        st = M.stats()
        assert st["kernel_errors"] == 0
        steps[name] = st["cg_steps"] / st["rows_solved"]
        r0[name] = st["cg_r0_micro"] / 1e6 / st["rows_solved"]
        rmse[name] = M.rmse()
        M.close()
    Xr, Tr = O.train(r, f, lam, 6, th0)
    rm_ref = O.rmse(r.test_u, r.test_i, r.test_r, Xr, Tr)
    print("mean CG steps per row, iterations 4-6:", steps, "mean starting relative residual:",
          r0, "rmse", rmse, "fp64", rm_ref)
    # what the trained network gains: a starting residual well below the zero
    # start's (1 for every row with a nonzero right-hand side)
    assert r0["zero"] > 0.99
    assert r0["mlp"] < 0.5 * r0["zero"]
    for v in rmse.values():
        assert abs(v - rm_ref) / rm_ref < 1e-3


@pytest.mark.parametrize("f,prec", [(100, A.PREC_BF16), (16, A.PREC_FP16), (33, A.PREC_BF16),
                                    (20, A.PREC_FP32), (128, A.PREC_BF16), (120, A.PREC_FP16)])
def test_features_match_numpy(f, prec):
    """Row features [b_u / n_u, diag(A_u) / n_u, log1p(n_u) / 8] against numpy
    on the same 16-bit (or FP32) factors: empty rows, short rows, rows long
    enough for several rounds of every warp, and a row long enough to be split
    across blocks (16-bit path). Tolerance 1e-2 relative (BF16 output)."""
    rng = np.random.default_rng(5)
    n = 300
    deg = np.array([0, 1, 3, 31, 32, 33, 200, 257, 1000, 2600, 0, 17, 20000])
    ptr = np.zeros(len(deg) + 1, np.int64)
    ptr[1:] = np.cumsum(deg)
    col = np.concatenate([rng.choice(n, d, replace=True) for d in deg]).astype(np.int32)
    val = rng.integers(1, 6, len(col)).astype(np.float32)
    ld = ((f + 1 + 7) // 8) * 8 if prec != A.PREC_FP32 else f
    th = np.zeros((n, ld), np.float32)
    th[:, :f] = rng.standard_normal((n, f)) * 0.3
    dt = {A.PREC_BF16: torch.bfloat16, A.PREC_FP16: torch.float16, A.PREC_FP32: torch.float32}[prec]
    src = torch.from_numpy(th).to(dt).cuda()
    thq = src.float().cpu().numpy().astype(np.float64)[:, :f]
    ldf = A.Mlp(f, capacity=64).ldf
    F = A.features(torch.from_numpy(ptr).cuda(), torch.from_numpy(col).cuda(),
                   torch.from_numpy(val).cuda(), src, f, prec, ldf).float().cpu().numpy()
    for u in range(len(deg)):
        s, e = ptr[u], ptr[u + 1]
        nu = e - s
        b = (val[s:e, None] * thq[col[s:e]]).sum(0) / max(nu, 1)
        d = (thq[col[s:e]] ** 2).sum(0) / max(nu, 1)
        ref = np.concatenate([b, d, [np.log1p(nu) / 8]])
        got = F[u, :2 * f + 1]
        assert np.abs(got - ref).max() <= 1e-2 * max(1.0, np.abs(ref).max()), (u, nu)
        assert not F[u, 2 * f + 1:].any()
