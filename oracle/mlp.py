"""CPU oracle of the warm-start MLP -- TEST INFRASTRUCTURE ONLY.

FP64 forward and backward of x0 = W3 g(W2 g(W1 F + b1) + b2) + b3 with
g = GELU (erf form), loss mean_b |Y_b - T_b|^2 / f. With `emulate=True` the
values the GPU kernels hold in BF16 are rounded to BF16 at the same points
(weights, the features, H1, H2, dY, dZ2, dZ1); the bias gradients use the
unrounded FP32 values, as the GPU does. With `emulate=False` it is plain FP64
(used for the finite-difference check of this oracle itself).
"""
import numpy as np
from scipy.special import erf


def bf16(x):
    """Round to the nearest BF16 value (ties to even); returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, np.float64).astype(np.float32))
    b = a.view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(z):
    return 0.5 * z * (1.0 + erf(z / np.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + erf(z / np.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / np.sqrt(2 * np.pi)


def forward(params, F, emulate=True):
    W1, b1, W2, b2, W3, b3 = (np.asarray(p, np.float64) for p in params)
    rnd = bf16 if emulate else (lambda v: v)
    F = rnd(F)
    Z1 = F @ rnd(W1).T + b1
    H1 = rnd(gelu(Z1))
    Z2 = H1 @ rnd(W2).T + b2
    H2 = rnd(gelu(Z2))
    Y = H2 @ rnd(W3).T + b3
    return Y, (F, Z1, H1, Z2, H2)


def loss_and_grads(params, F, T, emulate=True):
    W1, b1, W2, b2, W3, b3 = (np.asarray(p, np.float64) for p in params)
    rnd = bf16 if emulate else (lambda v: v)
    Y, (Fr, Z1, H1, Z2, H2) = forward(params, F, emulate)
    B, f = Y.shape
    E = Y - np.asarray(T, np.float64)
    loss = float(np.sum(E * E) / (B * f))
    dY = 2.0 * E / (B * f)
    dYb = rnd(dY)
    G3 = dYb.T @ H2
    gb3 = dY.sum(0)
    dZ2 = (dYb @ rnd(W3)) * gelu_grad(Z2)
    dZ2b = rnd(dZ2)
    G2 = dZ2b.T @ H1
    gb2 = dZ2.sum(0)
    dZ1 = (dZ2b @ rnd(W2)) * gelu_grad(Z1)
    dZ1b = rnd(dZ1)
    G1 = dZ1b.T @ Fr
    gb1 = dZ1.sum(0)
    return loss, [G1, gb1, G2, gb2, G3, gb3]


def init(f, hidden=256, seed=0):
    rng = np.random.default_rng(seed)
    din = 2 * f + 1
    return [rng.standard_normal((hidden, din)) * np.sqrt(2.0 / din), np.zeros(hidden),
            rng.standard_normal((hidden, hidden)) * np.sqrt(2.0 / hidden), np.zeros(hidden),
            rng.standard_normal((f, hidden)) * np.sqrt(2.0 / hidden), np.zeros(f)]
