"""Generate the FP64 accuracy fixture of the Netflix-shaped workload.

FP64 ALS (the oracle's exact mode: symmetric A_u, Cholesky, x_u = 0 for empty
rows) for the full 10 iterations of the 480,189 x 17,770, 99.1M-rating
synthetic matrix at f = 100, lambda = 0.05, started from the same seeded
theta0 the benchmark uses. The FP32 port of the same half-step is run beside
it for the same iterations, to record how far a correct FP32 solver drifts
from FP64 after 10 iterations.

Stored in netflix_f100_fp64.npz:
  checksums of the generated matrix and of theta0 (so a GPU test can tell a
  different matrix from a wrong result), the FP64 test RMSE after every
  iteration, the FP32 port's, and a seeded sample of 256 user rows of X and
  256 item rows of theta after the last iteration (float32).

CPU only; about 6 minutes on 8 cores for the FP64 run.

    python tests/golden/make_netflix_fp64.py [outdir]
"""
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [ROOT, os.path.join(ROOT, "cuda-mllib_b200")]

import als_b200 as A  # noqa: E402
import oracle as O  # noqa: E402

SEED = 1          # matrix seed of the benchmark
THETA_SEED = 101  # the benchmark's theta0 seed (matrix seed + 100)
N_SAMPLE = 256


def checksums(r, th0):
    """Order-sensitive checksums of the generated inputs: the sum, modulo 2^64,
    of each array's bit patterns weighted by position. Integer arithmetic, so
    every machine gets the same value for the same bytes."""
    def wsum(a):
        a = np.ascontiguousarray(a)
        bits = a.view(np.uint64 if a.itemsize == 8 else np.uint32).ravel().astype(np.uint64)
        w = (np.arange(bits.size, dtype=np.uint64) % np.uint64(1009)) + np.uint64(1)
        with np.errstate(over="ignore"):
            return int(np.sum(bits * w, dtype=np.uint64))
    return np.array([r.m, r.n, r.nnz, len(r.test_r), wsum(r.csr_ptr), wsum(r.csr_col),
                     wsum(r.csr_val), wsum(r.test_u), wsum(r.test_i), wsum(r.test_r),
                     wsum(th0)], np.uint64)


def main(outdir):
    cfg = dict(A.CONFIGS["netflix"])
    f, lam, iters = cfg["f"], cfg["lam"], cfg["iters"]
    t0 = time.time()
    r = A.synth(cfg, seed=SEED)
    th0 = A.init_factors(r.n, f, THETA_SEED)
    print(f"generated {r.m} x {r.n}, {r.nnz} train, {len(r.test_r)} test in {time.time() - t0:.1f} s",
          flush=True)
    rng = np.random.default_rng(20261203)
    users = np.sort(rng.choice(r.m, N_SAMPLE, replace=False)).astype(np.int64)
    items = np.sort(rng.choice(r.n, N_SAMPLE, replace=False)).astype(np.int64)

    T64 = th0.astype(np.float64)
    T32 = th0.astype(np.float32)
    rmse64, rmse32 = [], []
    for it in range(iters):
        t1 = time.time()
        X64, b1 = O.half_step(r.csr_ptr, r.csr_col, r.csr_val, T64, lam)
        T64, b2 = O.half_step(r.csc_ptr, r.csc_row, r.csc_val, X64, lam)
        X32, _ = O.half_step_f32(r.csr_ptr, r.csr_col, r.csr_val, T32, lam)
        T32, _ = O.half_step_f32(r.csc_ptr, r.csc_row, r.csc_val, X32, lam)
        rmse64.append(O.rmse(r.test_u, r.test_i, r.test_r, X64, T64))
        rmse32.append(O.rmse(r.test_u, r.test_i, r.test_r, X32.astype(np.float64),
                             T32.astype(np.float64)))
        print(f"iteration {it + 1}: fp64 rmse {rmse64[-1]:.8f}  fp32 port {rmse32[-1]:.8f}  "
              f"non-SPD {b1 + b2}  {time.time() - t1:.1f} s", flush=True)

    def rel(a, b):
        return np.linalg.norm(a - b, axis=1) / np.maximum(np.linalg.norm(b, axis=1), 1e-30)

    ex, et = rel(X32[users], X64[users]), rel(T32[items], T64[items])
    print(f"fp32 port vs fp64 after {iters} iterations: X median {np.median(ex):.2e} "
          f"max {ex.max():.2e}; theta median {np.median(et):.2e} max {et.max():.2e}")
    out = os.path.join(outdir, "netflix_f100_fp64.npz")
    np.savez_compressed(out, checksums=checksums(r, th0), f=f, lam=np.float64(lam), iters=iters,
                        seed=SEED, theta_seed=THETA_SEED, rmse_fp64=np.array(rmse64),
                        rmse_fp32_port=np.array(rmse32), users=users, items=items,
                        x_users=X64[users].astype(np.float32),
                        theta_items=T64[items].astype(np.float32),
                        x_users_fp32_port=X32[users], theta_items_fp32_port=T32[items])
    print("wrote", out)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.abspath(__file__)))
