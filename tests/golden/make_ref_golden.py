"""Generate the golden fixtures of the reference's own half-step.

Runs doALSWithCSR from the reference's als/src/cuda/als.cu (compiled for
sm_100a into oracle/_ref by oracle/Makefile) on small seeded inputs and stores
inputs and outputs here as ref_<case>.npz. Needs a GPU and the reference
checker build; the CPU test tests/test_golden.py then pins the oracle's
reference-emulation mode against these files without a GPU.

    python tests/golden/make_ref_golden.py [outdir]
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [ROOT, os.path.join(ROOT, "cuda-mllib_b200")]

import als_b200 as A  # noqa: E402
import oracle as O  # noqa: E402

CASES = [("ml1m_f10", "ml1m", 0.1, 10, 51), ("ml1m_f20", "ml1m", 0.1, 20, 52),
         ("ml1m_f100", "ml1m", 0.1, 100, 53)]
LAMBDA = 0.05


def main(outdir):
    os.makedirs(outdir, exist_ok=True)
    for tag, name, scale, f, seed in CASES:
        r = A.synth(A.scaled_config(name, scale), seed=seed)
        th = A.init_factors(r.n, f, seed + 1)
        ptr32 = r.csr_ptr.astype(np.int32)
        X, ms = O.ref_half_step(ptr32, r.csr_col, r.csr_val, th, LAMBDA)
        np.savez_compressed(os.path.join(outdir, f"ref_{tag}.npz"), ptr=ptr32, col=r.csr_col,
                            val=r.csr_val, theta=th, x_ref=X, lam=np.float32(LAMBDA),
                            name=name, scale=scale, f=f, seed=seed)
        print(tag, r.m, r.n, r.nnz, "ms", ms)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.abspath(__file__)))
