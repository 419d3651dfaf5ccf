"""Python host layer of the B200 ALS engine.

Thin ctypes bindings over the C ABI in ``include/als_b200.h`` (``libGPUALS.so``)
and ``include/als_data.h`` (``libalsdata.so``). All computation happens in those
libraries; PyTorch is used only to hold device memory and streams.

The drop-in path mirrors the reference's Spark JNI flow
(als/src/CuMFJNIInterface.cpp:93-109): CSR copied into ``mallocBest`` memory,
``doALSWithCSR`` called, the callee frees the CSR. The engine path keeps both
sides of the rating matrix and both factor matrices resident in HBM.

There is no CPU fallback: if the libraries are missing the import fails, and
if no GPU is present every compute call fails with the CUDA error.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))

# Synthetic data, CSR utilities and the configurations live in als_data
# (host-only libalsdata.so); they are re-exported here.
from als_data import (CONFIGS, Ratings, SynthSpec, datalib, flop_per_iteration,  # noqa: E402,F401
                      init_factors, row_scaled_config, scaled_config, synth, transpose)

ALS_OK, ALS_ERR_INVALID, ALS_ERR_CUDA, ALS_ERR_UNSUPPORTED = 0, 1, 2, 3
PREC_FP32, PREC_BF16, PREC_FP16 = 0, 1, 2
SOLVER_CHOLESKY, SOLVER_CG = 0, 1
WARM_ZERO, WARM_PREVIOUS, WARM_MLP = 0, 1, 2
SIDE_USERS, SIDE_ITEMS = 0, 1
ROW_EMPTY, ROW_NOT_SPD, ROW_REFINED_F64, ROW_CG_FALLBACK = 1, 2, 4, 8


class AlsError(RuntimeError):
    """A non-zero status from the C ABI."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def _load(name: str) -> ctypes.CDLL:
    path = os.path.join(_HERE, name)
    if not os.path.exists(path):
        raise ImportError(f"{path} is not built (run `make` in {_HERE})")
    return ctypes.CDLL(path)


lib = _load("libGPUALS.so")

c_i32, c_i64, c_u64, c_f32, c_f64 = (ctypes.c_int32, ctypes.c_int64, ctypes.c_uint64,
                                     ctypes.c_float, ctypes.c_double)
c_vp, c_sz = ctypes.c_void_p, ctypes.c_size_t


class Options(ctypes.Structure):
    _fields_ = [("precision", c_i32), ("solver", c_i32), ("warm_start", c_i32),
                ("cg_max_steps", c_i32), ("cg_tol", c_f32), ("refine_tol", c_f32),
                ("use_graph", c_i32), ("mlp_train_iters", c_i32), ("mlp_steps", c_i32),
                ("mlp_batch", c_i32), ("mlp_lr", c_f32), ("cg_jacobi", c_i32),
                ("solver_groups", c_i32), ("reserved", c_i32 * 3)]


class Stats(ctypes.Structure):
    _fields_ = [("rows_solved", c_u64), ("rows_refined", c_u64), ("rows_not_spd", c_u64),
                ("cg_steps", c_u64), ("cg_fallbacks", c_u64), ("kernel_errors", c_u64),
                ("cg_r0_micro", c_u64), ("solver_groups", ctypes.c_uint32 * 2)]

    def as_dict(self) -> dict:
        out = {}
        for k, _ in self._fields_:
            v = getattr(self, k)
            out[k] = list(v) if k == "solver_groups" else int(v)
        return out


def _sig(fn, restype, *argtypes):
    fn.restype = restype
    fn.argtypes = list(argtypes)
    return fn


_sig(lib.als_default_options, None, c_vp)
_sig(lib.als_last_error, ctypes.c_char_p)
_sig(lib.als_version, ctypes.c_char_p)
_sig(lib.als_model_create, c_i32, c_vp, c_i64, c_i64, c_i32, c_i64, c_vp, c_vp, c_vp, c_vp, c_vp,
     c_vp, c_vp, c_vp)
_sig(lib.als_model_destroy, None, c_vp)
_sig(lib.als_model_set_theta, c_i32, c_vp, c_vp, c_i32, c_vp)
_sig(lib.als_model_set_x, c_i32, c_vp, c_vp, c_i32, c_vp)
_sig(lib.als_model_half_step, c_i32, c_vp, c_i32, c_f32, c_vp)
_sig(lib.als_model_iterate, c_i32, c_vp, c_f32, c_i32, c_vp)
_sig(lib.als_model_set_row_range, c_i32, c_vp, c_i32, c_i64, c_i64, c_vp)
_sig(lib.als_model_sync_lp, c_i32, c_vp, c_i32, c_vp)
_sig(lib.als_model_factors, c_i32, c_vp, c_vp, c_vp)
_sig(lib.als_model_row_flags, c_i32, c_vp, c_i32, c_vp)
_sig(lib.als_model_stats, c_i32, c_vp, c_vp, c_i32)
_sig(lib.als_model_rmse, c_i32, c_vp, c_i64, c_vp, c_vp, c_vp, c_vp, c_vp)
_sig(lib.als_half_step_work_bytes, c_sz, c_i64)
_sig(lib.als_half_step, c_i32, c_i64, c_i64, c_i32, c_vp, c_vp, c_vp, c_vp, c_i32, c_vp, c_i32,
     c_f32, c_vp, c_vp, c_sz, c_vp)
_sig(lib.als_rmse_work_bytes, c_sz)
_sig(lib.als_rmse, c_i32, c_i64, c_vp, c_vp, c_vp, c_vp, c_i32, c_vp, c_i32, c_i32, c_vp, c_vp,
     c_sz, c_vp)
_sig(lib.als_predict, c_i32, c_i64, c_vp, c_vp, c_vp, c_i32, c_vp, c_i32, c_i32, c_vp, c_vp)
_sig(lib.als_topk, c_i32, c_i64, c_vp, c_vp, c_i32, c_vp, c_i32, c_i64, c_i32, c_i32, c_vp, c_vp,
     c_vp, c_vp, c_vp)
_sig(lib.als_csr_to_csc, c_i32, c_i64, c_i64, c_i64, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp)
_sig(lib.als_train, c_i32, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_i64, c_i64, c_i32, c_i64, c_f32,
     c_i32, c_vp, c_vp, c_vp, c_vp)
_sig(lib.doALSWithCSR, None, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, ctypes.c_int, ctypes.c_int,
     ctypes.c_int, ctypes.c_long, c_f32, ctypes.c_int)
_sig(lib.als_half_step_host, c_i32, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, ctypes.c_int,
     ctypes.c_int, ctypes.c_int, ctypes.c_long, c_f32, ctypes.c_int)
_sig(lib.als_set_dropin_options, c_i32, c_vp)
_sig(lib.als_debug_withhold_first_row, c_i32, c_i32)
_sig(lib.als_get_dropin_options, c_i32, c_vp)
# mallocBest / freeBest keep the reference's C++ linkage; these are their C names
_sig(lib.als_shard_unique_id, c_i32, c_vp)
_sig(lib.als_shard_partition, c_i32, c_vp, c_i64, c_i32, c_i32, c_vp)
_sig(lib.als_shard_blocks, c_i32, c_vp, c_i32, c_vp, c_vp)
_sig(lib.als_shard_create, c_i32, c_vp, c_vp, c_vp, c_vp, c_i64, c_i64, c_i32, c_i32, c_i32, c_vp,
     c_vp)
_sig(lib.als_shard_bounds, c_i32, c_vp, c_i32, c_vp)
_sig(lib.als_shard_exchange, c_i32, c_vp, c_i32, c_vp)
_sig(lib.als_shard_half_step, c_i32, c_vp, c_i32, c_f32, c_vp)
_sig(lib.als_shard_iterate, c_i32, c_vp, c_f32, c_i32, c_vp)
_sig(lib.als_shard_rmse, c_i32, c_vp, c_i64, c_vp, c_vp, c_vp, c_vp, c_vp)
_sig(lib.als_shard_destroy, None, c_vp)
_sig(lib.als_malloc_best, ctypes.c_int, c_vp, c_sz)
_sig(lib.als_free_best, ctypes.c_int, c_vp)
_sig(lib.get_gpu, ctypes.c_int)

_sig(lib.als_mlp_create, c_i32, c_vp, c_i32, c_i64, c_u64, c_vp)
_sig(lib.als_mlp_destroy, None, c_vp)
_sig(lib.als_mlp_feature_stride, c_i32, c_vp)
_sig(lib.als_mlp_param_count, c_i64, c_i32)
_sig(lib.als_mlp_get_params, c_i32, c_vp, c_vp, c_vp)
_sig(lib.als_mlp_set_params, c_i32, c_vp, c_vp, c_vp)
_sig(lib.als_mlp_gradients, c_i32, c_vp, c_i64, c_vp, c_vp, c_i32, c_vp, c_vp, c_vp)
_sig(lib.als_mlp_train_step, c_i32, c_vp, c_i64, c_vp, c_vp, c_i32, c_f32, c_vp)
_sig(lib.als_mlp_forward, c_i32, c_vp, c_i64, c_vp, c_vp, c_i32, c_vp)
_sig(lib.als_features, c_i32, c_i64, c_i32, c_vp, c_vp, c_vp, c_vp, c_i32, c_i32, c_vp, c_i32, c_vp)

def _check(rc: int) -> None:
    if rc != ALS_OK:
        raise AlsError(rc, lib.als_last_error().decode(errors="replace"))


def _ptr(a) -> int:
    """Raw address of a numpy array or torch tensor (None -> 0)."""
    if a is None:
        return 0
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()


def options(**kw) -> Options:
    o = Options()
    lib.als_default_options(ctypes.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise KeyError(k)
        setattr(o, k, v)
    return o


def version() -> str:
    return lib.als_version().decode()


# ---------------------------------------------------------------------------
# engine on device memory
# ---------------------------------------------------------------------------

def _stream_handle(stream) -> int:
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    return int(getattr(stream, "cuda_stream", stream))


class Model:
    """A resident ALS model: both sides of R and both factor matrices in HBM.

    Construct from a ``Ratings`` (uploaded once) or from device tensors.
    """

    def __init__(self, ratings: Ratings, f: int, opts: Options | None = None, stream=None,
                 theta0: np.ndarray | None = None, seed: int = 2):
        import torch
        self.torch = torch
        self.m, self.n, self.f = ratings.m, ratings.n, f
        dev = torch.device("cuda")
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        self._dev = [t(ratings.csr_ptr), t(ratings.csr_col), t(ratings.csr_val),
                     t(ratings.csc_ptr), t(ratings.csc_row), t(ratings.csc_val)]
        self.test = [t(ratings.test_u), t(ratings.test_i), t(ratings.test_r)]
        self.opts = opts or options()
        self.stream = _stream_handle(stream)
        h = c_vp()
        _check(lib.als_model_create(ctypes.byref(h), self.m, self.n, f, ratings.nnz,
                                    *[_ptr(x) for x in self._dev], ctypes.byref(self.opts),
                                    self.stream))
        self.handle = h
        if theta0 is None:
            theta0 = init_factors(self.n, f, seed)
        self.set_theta(torch.from_numpy(np.ascontiguousarray(theta0, np.float32)).to(dev))

    @classmethod
    def from_device(cls, m: int, n: int, f: int, nnz: int, arrays, test, opts=None,
                    stream=None, theta0: np.ndarray | None = None, seed: int = 2):
        """A model over rating arrays already on the device: ``arrays`` is
        (csr_ptr, csr_col, csr_val, csc_ptr, csc_row, csc_val) as CUDA tensors
        (int64 pointers, which may start at any offset into col/val), ``test``
        is (u, i, r). The tensors stay borrowed for the model's lifetime."""
        import torch
        self = cls.__new__(cls)
        self.torch = torch
        self.m, self.n, self.f = m, n, f
        self._dev = list(arrays)
        self.test = list(test)
        self.opts = opts or options()
        self.stream = _stream_handle(stream)
        h = c_vp()
        _check(lib.als_model_create(ctypes.byref(h), m, n, f, nnz, *[_ptr(x) for x in self._dev],
                                    ctypes.byref(self.opts), self.stream))
        self.handle = h
        if theta0 is None:
            theta0 = init_factors(n, f, seed)
        self.set_theta(torch.from_numpy(np.ascontiguousarray(theta0, np.float32)).cuda())
        return self

    def close(self):
        if getattr(self, "handle", None):
            lib.als_model_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_theta(self, theta_dev):
        _check(lib.als_model_set_theta(self.handle, _ptr(theta_dev), theta_dev.shape[1],
                                       self.stream))

    def set_x(self, x_dev):
        _check(lib.als_model_set_x(self.handle, _ptr(x_dev), x_dev.shape[1], self.stream))

    def half_step(self, side: int, lam: float):
        _check(lib.als_model_half_step(self.handle, side, lam, self.stream))

    def set_row_range(self, side: int, begin: int, end: int):
        _check(lib.als_model_set_row_range(self.handle, side, begin, end, self.stream))

    def sync_lp(self, side: int):
        _check(lib.als_model_sync_lp(self.handle, side, self.stream))

    def iterate(self, lam: float, iters: int = 1):
        _check(lib.als_model_iterate(self.handle, lam, iters, self.stream))

    def factors(self):
        """(X, theta) as torch tensors viewing the model's device memory."""
        torch = self.torch
        x, t = c_vp(), c_vp()
        _check(lib.als_model_factors(self.handle, ctypes.byref(x), ctypes.byref(t)))
        return (_wrap_device(x.value, (self.m, self.f), torch.float32),
                _wrap_device(t.value, (self.n, self.f), torch.float32))

    def row_flags(self, side: int):
        p = c_vp()
        _check(lib.als_model_row_flags(self.handle, side, ctypes.byref(p)))
        rows = self.m if side == SIDE_USERS else self.n
        return _wrap_device(p.value, (rows,), self.torch.int32)

    def stats(self, reset: bool = False) -> dict:
        s = Stats()
        _check(lib.als_model_stats(self.handle, ctypes.byref(s), int(reset)))
        return s.as_dict()

    def rmse(self, test=None) -> float:
        u, i, r = test if test is not None else self.test
        out = c_f64()
        _check(lib.als_model_rmse(self.handle, len(u), _ptr(u), _ptr(i), _ptr(r),
                                  ctypes.byref(out), self.stream))
        return float(out.value)


def shard_partition(ptr, world: int, f: int) -> np.ndarray:
    """The engine's nnz-balanced row ranges of a side (host row pointers):
    world + 1 bounds, a row costing nnz * f^2 + f^3 / 3."""
    ptr = np.ascontiguousarray(ptr, np.int64)
    b = np.zeros(world + 1, np.int64)
    _check(lib.als_shard_partition(_ptr(ptr), len(ptr) - 1, world, f, _ptr(b)))
    return b


def shard_blocks(bounds):
    """(span, start): the all-gather's block size in rows and each rank's
    first row of the block it sends."""
    bounds = np.ascontiguousarray(bounds, np.int64)
    world = len(bounds) - 1
    span = c_i64()
    start = np.zeros(world, np.int64)
    _check(lib.als_shard_blocks(_ptr(bounds), world, ctypes.byref(span), _ptr(start)))
    return int(span.value), start


def shard_unique_id() -> bytes:
    """A 128-byte NCCL unique id for Shard (made on rank 0, copied to all)."""
    buf = ctypes.create_string_buffer(128)
    _check(lib.als_shard_unique_id(buf))
    return buf.raw


class Shard:
    """Row sharding of a Model across GPUs through the engine's C ABI (one
    process per GPU): als_shard_create partitions both sides, restricts the
    model to this rank's rows and creates the NCCL communicator; every call
    below is collective."""

    def __init__(self, model: "Model", ratings, world: int, rank: int, nccl_id: bytes):
        self.model = model
        csr = np.ascontiguousarray(ratings.csr_ptr, np.int64)
        csc = np.ascontiguousarray(ratings.csc_ptr, np.int64)
        idbuf = ctypes.create_string_buffer(bytes(nccl_id), 128)
        h = c_vp()
        _check(lib.als_shard_create(ctypes.byref(h), model.handle, _ptr(csr), _ptr(csc),
                                    len(csr) - 1, len(csc) - 1, model.f, world, rank, idbuf,
                                    model.stream))
        self.handle, self.world, self.rank = h, world, rank

    def bounds(self, side: int) -> np.ndarray:
        b = np.zeros(self.world + 1, np.int64)
        _check(lib.als_shard_bounds(self.handle, side, _ptr(b)))
        return b

    def exchange(self, side: int):
        _check(lib.als_shard_exchange(self.handle, side, self.model.stream))

    def half_step(self, side: int, lam: float):
        _check(lib.als_shard_half_step(self.handle, side, lam, self.model.stream))

    def iterate(self, lam: float, iters: int = 1):
        _check(lib.als_shard_iterate(self.handle, lam, iters, self.model.stream))

    def rmse(self, test=None) -> float:
        u, i, r = test if test is not None else self.model.test
        out = c_f64()
        _check(lib.als_shard_rmse(self.handle, len(u), _ptr(u), _ptr(i), _ptr(r),
                                  ctypes.byref(out), self.model.stream))
        return float(out.value)

    def close(self):
        if getattr(self, "handle", None):
            lib.als_shard_destroy(self.handle)
            self.handle = None


def _wrap_device(addr: int, shape, dtype):
    """A torch tensor over device memory owned by the library (no copy)."""
    import torch
    typestr = {torch.float32: "<f4", torch.int32: "<i4", torch.int64: "<i8"}[dtype]

    class _Iface:
        __cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr,
                                    "data": (addr, False), "version": 3, "strides": None}
    return torch.as_tensor(_Iface(), device="cuda")


class Mlp:
    """The learned warm-start network (see als_mlp_* in include/als_b200.h)."""

    def __init__(self, f: int, capacity: int = 8192, seed: int = 1, stream=None):
        self.f = f
        self.stream = _stream_handle(stream)
        h = c_vp()
        _check(lib.als_mlp_create(ctypes.byref(h), f, capacity, seed, self.stream))
        self.handle = h
        self.ldf = int(lib.als_mlp_feature_stride(h))
        self.nparam = int(lib.als_mlp_param_count(f))

    def __del__(self):
        if getattr(self, "handle", None):
            lib.als_mlp_destroy(self.handle)
            self.handle = None

    def shapes(self):
        f, H = self.f, 256
        return [(H, 2 * f + 1), (H,), (H, H), (H,), (f, H), (f,)]

    def _split(self, flat):
        out, off = [], 0
        for sh in self.shapes():
            k = int(np.prod(sh))
            out.append(flat[off:off + k].reshape(sh))
            off += k
        return out

    def get_params(self):
        flat = np.empty(self.nparam, np.float32)
        _check(lib.als_mlp_get_params(self.handle, _ptr(flat), self.stream))
        return self._split(flat)

    def set_params(self, params):
        flat = np.concatenate([np.asarray(p, np.float32).ravel() for p in params])
        _check(lib.als_mlp_set_params(self.handle, _ptr(flat), self.stream))

    def gradients(self, F, T):
        flat = np.empty(self.nparam, np.float32)
        loss = c_f64()
        _check(lib.als_mlp_gradients(self.handle, F.shape[0], _ptr(F), _ptr(T), T.stride(0),
                                     _ptr(flat), ctypes.byref(loss), self.stream))
        return self._split(flat), float(loss.value)

    def train_step(self, F, T, lr: float):
        _check(lib.als_mlp_train_step(self.handle, F.shape[0], _ptr(F), _ptr(T), T.stride(0), lr,
                                      self.stream))

    def forward(self, F):
        import torch
        out = torch.empty((F.shape[0], self.f), dtype=torch.float32, device="cuda")
        _check(lib.als_mlp_forward(self.handle, F.shape[0], _ptr(F), _ptr(out), self.f,
                                   self.stream))
        return out


def features(row_ptr, col, val, src, f: int, precision: int, ldf: int, stream=None):
    """BF16 features [b/n, diag/n, log1p(n)/8] of each CSR row (device tensors);
    src holds the fixed factors (FP32, BF16 or FP16 per `precision`, row stride
    src.stride(0) >= f)."""
    import torch
    m = row_ptr.shape[0] - 1
    F = torch.zeros((m, ldf), dtype=torch.bfloat16, device="cuda")
    _check(lib.als_features(m, f, _ptr(row_ptr), _ptr(col), _ptr(val), _ptr(src), src.stride(0),
                            precision, _ptr(F), ldf, _stream_handle(stream)))
    return F


def half_step(row_ptr, col, val, src, dst, lam: float, opts: Options | None = None, stream=None):
    """Stand-alone FP32 half-step on caller device tensors (no model)."""
    import torch
    m = row_ptr.shape[0] - 1
    n, f = src.shape
    work = torch.empty(int(lib.als_half_step_work_bytes(m)), dtype=torch.uint8, device="cuda")
    _check(lib.als_half_step(m, n, f, _ptr(row_ptr), _ptr(col), _ptr(val), _ptr(src),
                             src.stride(0), _ptr(dst), dst.stride(0), lam,
                             ctypes.byref(opts or options()), _ptr(work), work.numel(),
                             _stream_handle(stream)))


def topk(users, x, theta, k: int, seen_ptr=None, seen_col=None, stream=None):
    """Top-k items per user (device tensors): returns (items int32 [nq, k],
    scores float32 [nq, k]), leaving out the items in each user's row of the
    (seen_ptr, seen_col) CSR when given."""
    import torch
    nq = users.shape[0]
    n, f = theta.shape
    items = torch.empty((nq, k), dtype=torch.int32, device="cuda")
    scores = torch.empty((nq, k), dtype=torch.float32, device="cuda")
    _check(lib.als_topk(nq, _ptr(users), _ptr(x), x.stride(0), _ptr(theta), theta.stride(0), n, f,
                        k, _ptr(seen_ptr) if seen_ptr is not None else None,
                        _ptr(seen_col) if seen_col is not None else None, _ptr(items),
                        _ptr(scores), _stream_handle(stream)))
    return items, scores


def csr_to_csc(m: int, n: int, ptr, col, val, stream=None):
    """Device CSR (int64 pointers) -> device CSC (col_ptr int64, rows int32, vals)."""
    import torch
    nnz = col.shape[0]
    cptr = torch.empty(n + 1, dtype=torch.int64, device="cuda")
    rows = torch.empty(max(nnz, 1), dtype=torch.int32, device="cuda")
    vals = torch.empty(max(nnz, 1), dtype=torch.float32, device="cuda")
    _check(lib.als_csr_to_csc(m, n, nnz, _ptr(ptr), _ptr(col), _ptr(val), _ptr(cptr), _ptr(rows),
                              _ptr(vals), _stream_handle(stream)))
    return cptr, rows[:nnz], vals[:nnz]


def rmse(u, i, r, x, theta, stream=None) -> float:
    import torch
    work = torch.empty(int(lib.als_rmse_work_bytes()), dtype=torch.uint8, device="cuda")
    out = c_f64()
    _check(lib.als_rmse(len(u), _ptr(u), _ptr(i), _ptr(r), _ptr(x), x.stride(0), _ptr(theta),
                        theta.stride(0), x.shape[1], ctypes.byref(out), _ptr(work), work.numel(),
                        _stream_handle(stream)))
    return float(out.value)


def predict(u, i, x, theta, stream=None):
    import torch
    out = torch.empty(len(u), dtype=torch.float32, device="cuda")
    _check(lib.als_predict(len(u), _ptr(u), _ptr(i), _ptr(x), x.stride(0), _ptr(theta),
                           theta.stride(0), x.shape[1], _ptr(out), _stream_handle(stream)))
    return out


def train(r: Ratings, f: int, lam: float, iters: int, theta0: np.ndarray,
          opts: Options | None = None):
    """Host-buffer full training through ``als_train`` (cuMF-standalone style)."""
    X = np.empty((r.m, f), np.float32)
    T = np.array(theta0, np.float32, copy=True, order="C")
    st = Stats()
    _check(lib.als_train(_ptr(r.csr_ptr), _ptr(r.csr_col), _ptr(r.csr_val), _ptr(r.csc_ptr),
                         _ptr(r.csc_row), _ptr(r.csc_val), r.m, r.n, f, r.nnz, lam, iters,
                         ctypes.byref(opts or options()), _ptr(X), _ptr(T), ctypes.byref(st)))
    return X, T, st.as_dict()


# ---------------------------------------------------------------------------
# drop-in path (the reference's JNI flow, without the JVM)
# ---------------------------------------------------------------------------

_cudart = None


def _rt():
    global _cudart
    if _cudart is None:
        for name in ("libcudart.so.12", "/usr/local/cuda/lib64/libcudart.so.12"):
            try:
                _cudart = ctypes.CDLL(name)
                break
            except OSError:
                continue
        if _cudart is None:
            raise ImportError("libcudart.so.12 not found")
        _sig(_cudart.cudaMemcpy, ctypes.c_int, c_vp, c_vp, c_sz, ctypes.c_int)
    return _cudart


def set_dropin_options(opts: Options) -> None:
    """Form used by the drop-in doALSWithCSR (process-wide)."""
    _check(lib.als_set_dropin_options(ctypes.byref(opts)))


def get_dropin_options() -> Options:
    o = Options()
    _check(lib.als_get_dropin_options(ctypes.byref(o)))
    return o


def do_als_with_csr(row_ptr32: np.ndarray, col: np.ndarray, val: np.ndarray, theta: np.ndarray,
                    m: int, n: int, f: int, lam: float, x_batch: int = 1,
                    out: np.ndarray | None = None) -> np.ndarray:
    """Run the drop-in ``doALSWithCSR``: CSR into mallocBest memory (freed by the
    callee), theta and X in host memory; returns X (m x f), written into ``out``
    (C-contiguous float32, pageable or pinned) when it is given."""
    rt = _rt()
    nnz = len(col)
    ptrs = []
    for arr in (np.ascontiguousarray(row_ptr32, np.int32), np.ascontiguousarray(col, np.int32),
                np.ascontiguousarray(val, np.float32)):
        p = c_vp()
        if lib.als_malloc_best(ctypes.byref(p), max(arr.nbytes, 4)) != 0:
            for q in ptrs:
                lib.als_free_best(q)
            raise AlsError(ALS_ERR_CUDA, "mallocBest failed")
        ptrs.append(p)
        if arr.nbytes and rt.cudaMemcpy(p, arr.ctypes.data, arr.nbytes, 1) != 0:
            for q in ptrs:
                lib.als_free_best(q)
            raise AlsError(ALS_ERR_CUDA, "cudaMemcpy failed")
    th = np.ascontiguousarray(theta, np.float32)
    if out is None:
        X = np.zeros((m, f), np.float32)
    else:
        if out.dtype != np.float32 or out.shape != (m, f) or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous float32 array of shape (m, f)")
        X = out
    lib.doALSWithCSR(None, ptrs[0], ptrs[1], ptrs[2], _ptr(th), _ptr(X), m, n, f, nnz, lam, x_batch)
    return X


def half_step_host(row_ptr32: np.ndarray, col: np.ndarray, val: np.ndarray, theta: np.ndarray,
                   m: int, n: int, f: int, lam: float, out: np.ndarray | None = None,
                   chunks: int = 0) -> np.ndarray:
    """The drop-in half-step on host CSR arrays (``als_half_step_host``, the
    path of the Spark JNI call): the ratings are uploaded in ``chunks`` row
    ranges (0: chosen from the rating count), each solved while the next one
    is uploaded. Same options and result as ``do_als_with_csr``; the arrays
    stay the caller's. Returns X (m x f), written into ``out`` when given."""
    ptr = np.ascontiguousarray(row_ptr32, np.int32)
    c = np.ascontiguousarray(col, np.int32)
    v = np.ascontiguousarray(val, np.float32)
    th = np.ascontiguousarray(theta, np.float32)
    if out is None:
        X = np.zeros((m, f), np.float32)
    else:
        if out.dtype != np.float32 or out.shape != (m, f) or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous float32 array of shape (m, f)")
        X = out
    _check(lib.als_half_step_host(None, _ptr(ptr), _ptr(c), _ptr(v), _ptr(th), _ptr(X), m, n, f,
                                  len(c), lam, chunks))
    return X
