"""The CPU oracle itself: exact mode against numpy, the emulation of the
reference's store defect, the FP32 port, RMSE and the objective."""
import numpy as np
import pytest

import als_b200 as A
import oracle as O


def _case(f, scale=0.15, seed=3):
    c = A.scaled_config("ml1m", scale)
    r = A.synth(c, seed=seed)
    th = A.init_factors(r.n, f, seed + 1).astype(np.float64)
    return r, th


def _numpy_half(ptr, col, val, src, lam):
    m, f = len(ptr) - 1, src.shape[1]
    X = np.zeros((m, f))
    for u in range(m):
        s, e = ptr[u], ptr[u + 1]
        if e == s:
            continue
        T = src[col[s:e]]
        X[u] = np.linalg.solve(T.T @ T + lam * (e - s) * np.eye(f), T.T @ val[s:e].astype(np.float64))
    return X


@pytest.mark.parametrize("f", [1, 10, 16, 100])
def test_exact_matches_numpy(f):
    r, th = _case(f)
    X, fails = O.half_step(r.csr_ptr, r.csr_col, r.csr_val, th, 0.05)
    assert fails == 0
    ref = _numpy_half(r.csr_ptr, r.csr_col, r.csr_val, th, 0.05)
    np.testing.assert_allclose(X, ref, rtol=1e-9, atol=1e-12)


def test_exact_thread_count_independent():
    r, th = _case(20)
    a, _ = O.half_step(r.csr_ptr, r.csr_col, r.csr_val, th, 0.05, threads=1)
    b, _ = O.half_step(r.csr_ptr, r.csr_col, r.csr_val, th, 0.05, threads=5)
    assert np.array_equal(a, b)


def test_empty_rows_give_zero():
    ptr = np.array([0, 0, 2, 2], np.int64)
    col = np.array([0, 1], np.int32)
    val = np.array([3.0, 4.0], np.float32)
    th = np.random.default_rng(0).standard_normal((2, 4))
    X, fails = O.half_step(ptr, col, val, th, 0.1)
    assert fails == 0
    assert np.all(X[0] == 0) and np.all(X[2] == 0) and np.any(X[1] != 0)


def test_non_spd_row_reported():
    # lambda = 0 with one rating at f = 3: rank-1 system, not positive definite
    ptr = np.array([0, 1], np.int64)
    X, fails = O.half_step(ptr, np.array([0], np.int32), np.array([1.0], np.float32),
                           np.ones((1, 3)), 0.0)
    assert fails == 1 and np.all(X == 0)


@pytest.mark.parametrize("f", [10, 20, 100])
def test_reference_store_defect_map(f):
    """The emulated reference system differs from the symmetric A_u exactly at
    (10*ti + 4, 10*tj), ti <= tj, where it holds A(10*ti, 10*tj): N(N+1)/2
    entries for N = f/10 (55 at f=100, 1 at f=10)."""
    rng = np.random.default_rng(1)
    rows = rng.standard_normal((37, f)).astype(np.float32).astype(np.float64)
    lam = 0.05
    tt = O.refemu_system(rows, lam)
    exact = rows.T @ rows + lam * 37 * np.eye(f)
    diff = np.abs(tt - exact) > 1e-3 * np.abs(exact).max()
    N = f // 10
    want = np.zeros((f, f), bool)
    for ti in range(N):
        for tj in range(ti, N):
            want[10 * ti + 4, 10 * tj] = True
    assert diff.sum() == N * (N + 1) // 2
    assert np.array_equal(diff, want)
    for ti in range(N):
        for tj in range(ti, N):
            raw = (rows.T @ rows)[10 * ti, 10 * tj]
            assert abs(tt[10 * ti + 4, 10 * tj] - raw) < 1e-4 * max(1.0, abs(raw))
    # mirrored lower triangle is correct: tt is not symmetric only at the defects
    asym = np.abs(tt - tt.T) > 1e-3 * np.abs(exact).max()
    assert asym.sum() == 2 * (N * (N + 1) // 2)  # each defect and its correct transpose


def test_refemu_differs_from_exact_only_by_the_defect():
    """Rebuilding the emulated solve with the defect-free system recovers the
    exact solution: the emulation changes nothing but the defective entries."""
    r, th = _case(10)
    Xe, _ = O.half_step(r.csr_ptr, r.csr_col, r.csr_val, th, 0.05, mode=O.REFEMU)
    X, _ = O.half_step(r.csr_ptr, r.csr_col, r.csr_val, th, 0.05)
    # Recompute the emulated solution in numpy from refemu_system for a few rows
    for u in range(0, r.m, max(1, r.m // 25)):
        s, e = r.csr_ptr[u], r.csr_ptr[u + 1]
        if e == s:
            continue
        rows = th[r.csr_col[s:e]]
        tt = O.refemu_system(rows, 0.05)
        b = rows.astype(np.float32).T @ r.csr_val[s:e]
        np.testing.assert_allclose(Xe[u], np.linalg.solve(tt, b), rtol=2e-3, atol=1e-5)
    assert np.abs(Xe - X).max() > 1e-3  # the defect is visible


def test_fp32_port_close_to_fp64():
    r, th = _case(32)
    X, _ = O.half_step(r.csr_ptr, r.csr_col, r.csr_val, th, 0.05)
    Xf, fails = O.half_step_f32(r.csr_ptr, r.csr_col, r.csr_val, th.astype(np.float32), 0.05)
    assert fails == 0
    rel = np.linalg.norm(Xf - X, axis=1) / np.maximum(np.linalg.norm(X, axis=1), 1e-30)
    assert rel.max() < 1e-4


def test_rmse_and_objective():
    r, th = _case(8)
    X, _ = O.half_step(r.csr_ptr, r.csr_col, r.csr_val, th, 0.05)
    pred = np.einsum("ij,ij->i", X[r.test_u], th[r.test_i])
    assert abs(O.rmse(r.test_u, r.test_i, r.test_r, X, th) -
               np.sqrt(np.mean((r.test_r - pred) ** 2))) < 1e-12
    # ALS never increases the objective: each half-step is an exact minimisation
    obj = [O.objective(r.csr_ptr, r.csr_col, r.csr_val, X, th, 0.05)]
    T = th
    for _ in range(3):
        T, _ = O.half_step(r.csc_ptr, r.csc_row, r.csc_val, X, 0.05)
        obj.append(O.objective(r.csr_ptr, r.csr_col, r.csr_val, X, T, 0.05))
        X, _ = O.half_step(r.csr_ptr, r.csr_col, r.csr_val, T, 0.05)
        obj.append(O.objective(r.csr_ptr, r.csr_col, r.csr_val, X, T, 0.05))
    assert all(b <= a * (1 + 1e-12) for a, b in zip(obj, obj[1:]))
