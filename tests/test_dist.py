"""Row sharding across ranks: partition balance, and a 2-rank gloo run of the
sharded iteration (each rank solves its rows, then the rows are exchanged by
one all-gather per half-step) that must equal the unsharded ALS. The per-rank solver here is a CPU stand-in
built on the oracle; the exchange logic is the one the GPU ranks use."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import als_b200 as A
import als_dist as D
import oracle as O


def test_partition_balanced_and_contiguous():
    r = A.synth(A.scaled_config("netflix", 0.05), seed=2)
    for world in (1, 2, 3, 8):
        for ptr in (r.csr_ptr, r.csc_ptr):
            b = D.partition(ptr, world, 100)
            assert b[0] == 0 and b[-1] == len(ptr) - 1 and np.all(np.diff(b) >= 0)
            cost = np.diff(ptr) * 1e4 + 1e6 / 3
            shares = [cost[b[k]:b[k + 1]].sum() for k in range(world)]
            assert max(shares) <= cost.sum() / world + cost.max() + 1


def test_gather_blocks_cover_every_range():
    rng = np.random.default_rng(3)
    cases = [np.array([0, 5, 5, 12]), np.array([0, 0, 7]), np.array([0, 9]),
             np.array([0, 1, 2, 3, 40])]
    for _ in range(50):
        world = int(rng.integers(1, 9))
        cuts = np.sort(rng.integers(0, 200, world - 1))
        cases.append(np.concatenate([[0], cuts, [int(rng.integers(max(cuts.max(initial=0), 1), 300))]]))
    for b in cases:
        span, start = D.gather_blocks(b)
        rows = b[-1]
        assert span == np.diff(b).max()
        for r in range(len(b) - 1):
            assert 0 <= start[r] <= b[r] and b[r + 1] <= start[r] + span <= rows


def test_engine_partition_and_blocks_match():
    """The C++ shard driver's partition and all-gather blocks
    (als_shard_partition, als_shard_blocks; host code, no GPU) equal the
    Python ones the gloo test drives, including empty and single-row ranges."""
    r = A.synth(A.scaled_config("netflix", 0.05), seed=2)
    rng = np.random.default_rng(8)
    cases = [r.csr_ptr, r.csc_ptr, np.array([0, 0, 0, 5]), np.array([0, 7]),
             np.concatenate([[0], np.cumsum(rng.integers(0, 50, 300))])]
    for ptr in cases:
        for world in (1, 2, 3, 5, 8):
            for f in (10, 100, 128):
                b = A.shard_partition(ptr, world, f)
                assert np.array_equal(b, D.partition(ptr, world, f)), (world, f)
                span, start = A.shard_blocks(b)
                span_p, start_p = D.gather_blocks(b)
                assert span == span_p and np.array_equal(start, start_p)


def test_engine_shard_rejects_bad_arguments():
    """The shard entry points check their arguments before touching a GPU or
    NCCL: null pointers, world < 1 and a rank outside [0, world) are
    ALS_ERR_INVALID with a message."""
    import ctypes
    lib = A.lib
    ptr = np.array([0, 3, 5], np.int64)
    b = np.zeros(3, np.int64)
    assert lib.als_shard_partition(None, 2, 2, 10, b.ctypes.data) == 1
    assert lib.als_shard_partition(ptr.ctypes.data, 2, 0, 10, b.ctypes.data) == 1
    assert b"bad arguments" in lib.als_last_error()
    h = ctypes.c_void_p()
    idbuf = ctypes.create_string_buffer(128)
    for world, rank in ((0, 0), (2, 2), (2, -1)):
        rc = lib.als_shard_create(ctypes.byref(h), ctypes.c_void_p(1), ptr.ctypes.data, ptr.ctypes.data,
                                  2, 2, 10, world, rank, idbuf, None)
        assert rc == 1 and not h.value, (world, rank)
    span = ctypes.c_int64()
    assert lib.als_shard_blocks(None, 2, ctypes.byref(span), b.ctypes.data) == 1


class CpuModel:
    """CPU stand-in with the engine model's interface (FP64 oracle solves)."""

    def __init__(self, r, f, theta0, lam):
        self.r, self.f = r, f
        self.X = torch.zeros((r.m, f), dtype=torch.float64)
        self.T = torch.from_numpy(np.asarray(theta0, np.float64).copy())
        self.range = {0: (0, r.m), 1: (0, r.n)}
        self.synced = []

    def set_row_range(self, side, b, e):
        self.range[side] = (b, e)

    def half_step(self, side, lam):
        r = self.r
        b, e = self.range[side]
        if side == 0:
            ptr, idx, val, src, dst = r.csr_ptr, r.csr_col, r.csr_val, self.T, self.X
        else:
            ptr, idx, val, src, dst = r.csc_ptr, r.csc_row, r.csc_val, self.X, self.T
        sub = ptr[b:e + 1] - ptr[b]
        out, _ = O.half_step(sub, idx[ptr[b]:ptr[e]], val[ptr[b]:ptr[e]], src.numpy(), lam)
        dst[b:e] = torch.from_numpy(out)

    def factors(self):
        return self.X, self.T

    def sync_lp(self, side):
        self.synced.append(side)


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    r = A.synth(A.scaled_config("ml1m", 0.1), seed=4)
    f, lam = 8, 0.05
    th0 = A.init_factors(r.n, f, 5)
    model = CpuModel(r, f, th0, lam)
    sh = D.ShardedIteration(model, r, world, rank)
    sh.apply()
    sh.iterate(lam, 3)
    if rank == 0:
        np.save(out, np.concatenate([model.X.numpy().ravel(), model.T.numpy().ravel()]))
    assert model.synced == [0, 1] * 3
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_sharded_iteration_equals_unsharded(tmp_path, world):
    out = str(tmp_path / "xt.npy")
    mp.start_processes(_worker, args=(world, _free_port(), out), nprocs=world, join=True,
                       start_method="spawn")
    got = np.load(out)
    r = A.synth(A.scaled_config("ml1m", 0.1), seed=4)
    f, lam = 8, 0.05
    Xr, Tr = O.train(r, f, lam, 3, A.init_factors(r.n, f, 5))
    want = np.concatenate([Xr.ravel(), Tr.ravel()])
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-14)
