"""Row sharding of the ALS half-step across ranks, restated over
torch.distributed for the multi-rank tests.

The engine's shard driver (als_shard_* in csrc/als_shard.cu, bound as
als_b200.Shard; bench.py uses it under torchrun) is C++ over the C ABI with NCCL:
every rank keeps the whole CSR/CSC and both factor matrices, solves an
nnz-balanced contiguous row range of each side, and after each half-step the
ranges are exchanged by ONE all-gather and the low-precision copy is rebuilt
from the FP32 rows. NCCL needs one GPU per rank, so the exchange with several
ranks is tested here instead: the same partition and blocks (checked equal to
the engine's by tests/test_dist.py) and the same all-gather over gloo, with a
CPU stand-in for the model.

The ranges are nnz-balanced, so their row counts differ; the all-gather moves
equal blocks of `span` = the largest range's row count. Each rank sends the
`span` contiguous rows of its factor matrix that start at its range (shifted
back to stay inside the matrix for the last ranges), so the send needs no
staging copy; after the collective each rank copies the other ranks' ranges
out of the gathered blocks into place.
"""
from __future__ import annotations

import numpy as np

SIDE_USERS, SIDE_ITEMS = 0, 1


def partition(ptr: np.ndarray, world: int, f: int) -> np.ndarray:
    """Contiguous row ranges [b[r], b[r+1]) with balanced cost, where a row's
    cost is its nnz * f^2 (hermitian) plus f^3 / 3 (solve)."""
    ptr = np.asarray(ptr, np.int64)
    rows = len(ptr) - 1
    cost = np.diff(ptr).astype(np.float64) * f * f + f ** 3 / 3.0
    cum = np.concatenate([[0.0], np.cumsum(cost)])
    targets = cum[-1] * np.arange(1, world) / world
    cuts = np.searchsorted(cum, targets, side="left")
    b = np.concatenate([[0], np.clip(cuts, 0, rows), [rows]]).astype(np.int64)
    return np.maximum.accumulate(b)


def gather_blocks(b: np.ndarray):
    """(span, start): the all-gather block size in rows and, per rank, the
    first row of the block it sends. start[r] = min(b[r], rows - span), so the
    block [start[r], start[r] + span) lies inside the matrix and covers the
    range [b[r], b[r+1])."""
    b = np.asarray(b, np.int64)
    rows = int(b[-1])
    span = int(np.diff(b).max()) if len(b) > 1 else 0
    start = np.minimum(b[:-1], rows - span)
    return span, start


class ShardedIteration:
    """Drives a model's half-steps on this rank's rows and exchanges rows.

    model: exposes set_row_range(side, b, e), half_step(side, lam),
           factors() -> (X, theta) tensors over the model's storage, and
           sync_lp(side).
    """

    def __init__(self, model, ratings, world: int, rank: int, stream=None):
        self.model, self.world, self.rank, self.stream = model, world, rank, stream
        f = model.f
        self.bounds = {SIDE_USERS: partition(ratings.csr_ptr, world, f),
                       SIDE_ITEMS: partition(ratings.csc_ptr, world, f)}
        self.blocks = {side: gather_blocks(b) for side, b in self.bounds.items()}
        self.stage = {}

    def apply(self):
        for side, b in self.bounds.items():
            self.model.set_row_range(side, int(b[self.rank]), int(b[self.rank + 1]))

    def gather(self, side: int):
        import torch
        import torch.distributed as dist
        X, T = self.model.factors()
        target = X if side == SIDE_USERS else T
        b = self.bounds[side]
        span, start = self.blocks[side]
        if span == 0:
            self.model.sync_lp(side)
            return
        ctx = torch.cuda.stream(self.stream) if self.stream is not None else _null()
        with ctx:
            stage = self.stage.get(side)
            if stage is None or stage.dtype != target.dtype or stage.device != target.device:
                stage = torch.empty((self.world * span,) + tuple(target.shape[1:]),
                                    dtype=target.dtype, device=target.device)
                self.stage[side] = stage
            s0 = int(start[self.rank])
            dist.all_gather_into_tensor(stage, target[s0:s0 + span])
            for r in range(self.world):
                lo, hi = int(b[r]), int(b[r + 1])
                if r == self.rank or hi == lo:
                    continue
                off = r * span + lo - int(start[r])
                target[lo:hi].copy_(stage[off:off + hi - lo])
        self.model.sync_lp(side)

    def half_step(self, side: int, lam: float):
        self.model.half_step(side, lam)
        self.gather(side)

    def iterate(self, lam: float, iters: int = 1):
        for _ in range(iters):
            self.half_step(SIDE_USERS, lam)
            self.half_step(SIDE_ITEMS, lam)


class _null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False
