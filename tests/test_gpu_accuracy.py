"""Accuracy at the headline workload: every form trained for the workload's
10 iterations on the Netflix-shaped matrix (480,189 x 17,770, 99.1M training
ratings, 1.4M test, f = 100, lambda = 0.05) from the benchmark's seeded theta0,
against FP64 ALS (the oracle) run for the same 10 iterations from the same
theta0 (fixture tests/golden/netflix_f100_fp64.npz, made by
tests/golden/make_netflix_fp64.py).

Tolerances:
  test RMSE   within 0.1% (relative) of the FP64 run's, for every form;
  FP32 form   a seeded sample of 256 user rows of X and 256 item rows of
              theta within 1e-3 per-row relative L2 error of the FP64 rows
              (the FP32 port of the oracle itself lands within 4e-4).
"""
import numpy as np
import pytest
import torch

import als_b200 as A

pytestmark = pytest.mark.gpu

FIXTURE = __import__("os").path.join(__import__("os").path.dirname(__file__), "golden",
                                     "netflix_f100_fp64.npz")
RMSE_TOL = 1e-3   # relative
ROW_TOL = 1e-3    # FP32 form, per-row relative L2


@pytest.fixture(scope="module")
def golden():
    return np.load(FIXTURE)


@pytest.fixture(scope="module")
def netflix(golden):
    from golden.make_netflix_fp64 import checksums
    cfg = dict(A.CONFIGS["netflix"])
    r = A.synth(cfg, seed=int(golden["seed"]))
    th0 = A.init_factors(r.n, int(golden["f"]), int(golden["theta_seed"]))
    # the same matrix and theta0 as the FP64 run, or the comparison means nothing
    np.testing.assert_array_equal(checksums(r, th0), golden["checksums"])
    return r, th0


def rel_rows(X, ref):
    ref = np.asarray(ref, np.float64)
    return np.linalg.norm(np.asarray(X, np.float64) - ref, axis=1) / np.maximum(
        np.linalg.norm(ref, axis=1), 1e-30)


def train(r, th0, opts, iters, lam):
    M = A.Model(r, th0.shape[1], opts, theta0=th0)
    rm = []
    for _ in range(iters):
        M.half_step(A.SIDE_USERS, lam)
        M.half_step(A.SIDE_ITEMS, lam)
        rm.append(M.rmse())
    X, T = (t.cpu().numpy() for t in M.factors())
    st = M.stats()
    M.close()
    return X, T, rm, st


FORMS = {
    "fp32_cholesky": dict(precision=A.PREC_FP32, solver=A.SOLVER_CHOLESKY),
    "bf16_cg_previous": dict(precision=A.PREC_BF16, solver=A.SOLVER_CG, warm_start=A.WARM_PREVIOUS),
    "fp16_cg_previous": dict(precision=A.PREC_FP16, solver=A.SOLVER_CG, warm_start=A.WARM_PREVIOUS),
    "bf16_cg_mlp": dict(precision=A.PREC_BF16, solver=A.SOLVER_CG, warm_start=A.WARM_MLP),
    "bf16_cholesky": dict(precision=A.PREC_BF16, solver=A.SOLVER_CHOLESKY),
}


@pytest.mark.parametrize("form", list(FORMS))
def test_netflix_rmse_within_0p1_percent_of_fp64(netflix, golden, form):
    r, th0 = netflix
    iters, lam = int(golden["iters"]), float(golden["lam"])
    X, T, rm, st = train(r, th0, A.options(**FORMS[form]), iters, lam)
    assert st["kernel_errors"] == 0 and st["rows_not_spd"] == 0, st
    ref = golden["rmse_fp64"]
    gap = abs(rm[-1] - ref[-1]) / ref[-1]
    print(f"{form}: rmse {rm[-1]:.6f} fp64 {ref[-1]:.6f} gap {gap:.2e}; per iteration",
          [f"{(a - b) / b:+.1e}" for a, b in zip(rm, ref)])
    assert gap < RMSE_TOL, (form, rm[-1], float(ref[-1]))
    ex = rel_rows(X[golden["users"]], golden["x_users"])
    et = rel_rows(T[golden["items"]], golden["theta_items"])
    print(f"{form}: sampled rows vs fp64: X median {np.median(ex):.2e} max {ex.max():.2e}, "
          f"theta median {np.median(et):.2e} max {et.max():.2e}")
    if form == "fp32_cholesky":
        assert ex.max() < ROW_TOL and et.max() < ROW_TOL, (ex.max(), et.max())
