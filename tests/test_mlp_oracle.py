"""The MLP oracle's FP64 backward against central finite differences."""
import numpy as np

from oracle import mlp as M


def test_oracle_gradients_match_finite_differences():
    f, hidden, B = 3, 8, 5
    rng = np.random.default_rng(0)
    params = M.init(f, hidden, seed=1)
    params = [p + 0.1 * rng.standard_normal(p.shape) for p in params]
    F = rng.standard_normal((B, 2 * f + 1))
    T = rng.standard_normal((B, f))
    _, grads = M.loss_and_grads(params, F, T, emulate=False)
    h = 1e-6
    for k, p in enumerate(params):
        num = np.zeros_like(p)
        flat = p.reshape(-1)
        for i in range(flat.size):
            old = flat[i]
            flat[i] = old + h
            lp, _ = M.loss_and_grads(params, F, T, emulate=False)
            flat[i] = old - h
            lm, _ = M.loss_and_grads(params, F, T, emulate=False)
            flat[i] = old
            num.reshape(-1)[i] = (lp - lm) / (2 * h)
        np.testing.assert_allclose(grads[k], num, rtol=1e-5, atol=1e-8)


def test_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 1e-3])
    r = M.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0  # tie -> even
    assert r[2] == 1.0 + 2 ** -7        # above the midpoint rounds up
    assert r[3] == -2.5
    assert abs(r[4] - 1e-3) / 1e-3 < 2 ** -8
