"""Time the reference's own GPU half-step (doALSWithCSR from
als/src/cuda/als.cu, built for sm_100a into oracle/_ref) at a benchmark shape.

Checker tooling: it runs the reference, not the engine. One full iteration =
the user half-step (CSR, X from theta) plus the item half-step (CSC, theta
from X). X_BATCH is chosen as the reference needs (batch * f * f < 2^31, its
int indexing; als.cu:1069). Times are CUDA events around each doALSWithCSR
call, which include its own theta upload and X download (its API does both).

    python oracle/time_reference.py [--config netflix] [--iters 2] [--out file.json]
"""
import argparse
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path[:0] = [ROOT, os.path.join(ROOT, "cuda-mllib_b200")]

import als_b200 as A  # noqa: E402
import oracle as O  # noqa: E402


def x_batch(m, f):
    lim = (2 ** 31 - 1) // (f * f)
    return max(1, -(-m // lim))


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--config", default="netflix")
    p.add_argument("--scale", type=float, default=1.0)
    p.add_argument("--iters", type=int, default=2)
    p.add_argument("--seed", type=int, default=1)
    p.add_argument("--out", default=None)
    a = p.parse_args()
    cfg = A.scaled_config(a.config, a.scale) if a.scale != 1.0 else dict(A.CONFIGS[a.config])
    f, lam = cfg["f"], cfg["lam"]
    r = A.synth(cfg, seed=a.seed)
    T = A.init_factors(r.n, f, a.seed + 100)
    ptr32, cptr32 = r.csr_ptr.astype(np.int32), r.csc_ptr.astype(np.int32)
    rows = []
    for it in range(a.iters):
        t0 = time.perf_counter()
        X, ms_u = O.ref_half_step(ptr32, r.csr_col, r.csr_val, T, lam, x_batch(r.m, f))
        Tn, ms_i = O.ref_half_step(cptr32, r.csc_row, r.csc_val, X, lam, x_batch(r.n, f))
        wall = time.perf_counter() - t0
        T = np.nan_to_num(Tn)  # the reference leaves NaN in rows without ratings
        rows.append({"iter": it, "users_ms": ms_u, "items_ms": ms_i, "wall_s": wall})
        print(json.dumps(rows[-1]), flush=True)
    best = min(rows[1:] or rows, key=lambda d: d["users_ms"] + d["items_ms"])
    sec = (best["users_ms"] + best["items_ms"]) / 1e3
    res = {"config": a.config, "scale": a.scale, "m": r.m, "n": r.n, "nnz_train": r.nnz, "f": f,
           "sec_per_iter": sec, "gflops": A.flop_per_iteration(r, f) / sec / 1e9,
           "x_batch_users": x_batch(r.m, f), "x_batch_items": x_batch(r.n, f), "iters": rows}
    print(json.dumps(res), flush=True)
    if a.out:
        with open(a.out, "w") as fh:
            json.dump(res, fh, indent=1)


if __name__ == "__main__":
    main()
