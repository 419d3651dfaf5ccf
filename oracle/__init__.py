"""CPU oracle for the ALS half-step -- TEST INFRASTRUCTURE ONLY.

Bindings for ``liboracle.so`` (the C restatement in ``als_oracle.c``) and, when
it was built, ``_ref/libcumf_ref.so`` (the reference's own ``doALSWithCSR``
compiled from its sources). Only tests, the smoke check and the benchmark's
CPU-baseline leg use this package; the engine never does.

Parity is pinned two ways: the FP64 restatement is checked against numpy's
dense solver in the CPU tests, and its reference-emulation mode against the
reference's own kernels run on the GPU (the committed fixtures under
tests/golden were produced that way by tests/golden/make_ref_golden.py).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
EXACT, REFEMU = 0, 1

_lib = None
_ref = None


def build() -> None:
    """Build liboracle.so (and _ref/ when the reference sources are present)."""
    subprocess.run(["make", "-C", HERE, "-s"], check=True)


def _load():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        lib = ctypes.CDLL(path)
        vp, i64, i32, f64, f32 = (ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32,
                                  ctypes.c_double, ctypes.c_float)
        lib.orc_half_step_f64.restype = i64
        lib.orc_half_step_f64.argtypes = [i64, i32, vp, vp, vp, vp, f64, vp, i32, i32]
        lib.orc_half_step_f32.restype = i64
        lib.orc_half_step_f32.argtypes = [i64, i32, vp, vp, vp, vp, f32, vp, i32]
        lib.orc_rmse.restype = f64
        lib.orc_rmse.argtypes = [i64, vp, vp, vp, vp, vp, i32]
        lib.orc_objective.restype = f64
        lib.orc_objective.argtypes = [i64, i64, i32, vp, vp, vp, vp, vp, f64]
        lib.orc_refemu_system.restype = ctypes.c_int
        lib.orc_refemu_system.argtypes = [i32, i64, vp, f64, vp]
        _lib = lib
    return _lib


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


def half_step(ptr, col, val, src, lam: float, mode: int = EXACT, threads: int = 0):
    """FP64 half-step: rows of the CSR solved against src (n x f). Returns
    (dst m x f float64, number of non-SPD rows)."""
    lib = _load()
    ptr = np.ascontiguousarray(ptr, np.int64)
    col = np.ascontiguousarray(col, np.int32)
    val = np.ascontiguousarray(val, np.float32)
    src = np.ascontiguousarray(src, np.float64)
    m, f = len(ptr) - 1, src.shape[1]
    dst = np.zeros((m, f), np.float64)
    fails = lib.orc_half_step_f64(m, f, _p(ptr), _p(col), _p(val), _p(src), lam, _p(dst), mode,
                                  threads)
    if fails < 0:
        raise ValueError("oracle rejected the arguments")
    return dst, int(fails)


def half_step_f32(ptr, col, val, src, lam: float, threads: int = 0):
    """The same algorithm in FP32 (the timed CPU baseline)."""
    lib = _load()
    ptr = np.ascontiguousarray(ptr, np.int64)
    col = np.ascontiguousarray(col, np.int32)
    val = np.ascontiguousarray(val, np.float32)
    src = np.ascontiguousarray(src, np.float32)
    m, f = len(ptr) - 1, src.shape[1]
    dst = np.zeros((m, f), np.float32)
    fails = lib.orc_half_step_f32(m, f, _p(ptr), _p(col), _p(val), _p(src), lam, _p(dst), threads)
    if fails < 0:
        raise ValueError("oracle rejected the arguments")
    return dst, int(fails)


def refemu_system(rows, lam: float):
    """The column-major system the reference forms for one row whose gathered
    factor rows are `rows` (d x f); returned as a row-major (f, f) array
    A[r, c] (the reference's tt[r + c*f])."""
    lib = _load()
    rows = np.ascontiguousarray(rows, np.float64)
    d, f = rows.shape
    tt = np.zeros(f * f, np.float64)
    if lib.orc_refemu_system(f, d, _p(rows), lam, _p(tt)) != 0:
        raise ValueError("f must be a multiple of 10")
    return tt.reshape(f, f).T.copy()


def rmse(u, i, r, X, T) -> float:
    lib = _load()
    u = np.ascontiguousarray(u, np.int32)
    i = np.ascontiguousarray(i, np.int32)
    r = np.ascontiguousarray(r, np.float32)
    X = np.ascontiguousarray(X, np.float64)
    T = np.ascontiguousarray(T, np.float64)
    return float(lib.orc_rmse(len(u), _p(u), _p(i), _p(r), _p(X), _p(T), X.shape[1]))


def objective(ptr, col, val, X, T, lam: float) -> float:
    lib = _load()
    ptr = np.ascontiguousarray(ptr, np.int64)
    col = np.ascontiguousarray(col, np.int32)
    val = np.ascontiguousarray(val, np.float32)
    X = np.ascontiguousarray(X, np.float64)
    T = np.ascontiguousarray(T, np.float64)
    return float(lib.orc_objective(len(ptr) - 1, T.shape[0], X.shape[1], _p(ptr), _p(col),
                                   _p(val), _p(X), _p(T), lam))


def train(r, f: int, lam: float, iters: int, theta0, threads: int = 0):
    """FP64 ALS: users from theta, then items from X, `iters` times."""
    T = np.asarray(theta0, np.float64)
    X = None
    for _ in range(iters):
        X, _ = half_step(r.csr_ptr, r.csr_col, r.csr_val, T, lam, EXACT, threads)
        T, _ = half_step(r.csc_ptr, r.csc_row, r.csc_val, X, lam, EXACT, threads)
    return X, T


# ---------------------------------------------------------------- reference

def ref_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libcumf_ref.so"))


def _load_ref():
    global _ref
    if _ref is None:
        path = os.path.join(HERE, "_ref", "libcumf_ref.so")
        if not os.path.exists(path):
            raise FileNotFoundError("reference checker not built (needs the reference sources)")
        lib = ctypes.CDLL(path)
        vp = ctypes.c_void_p
        lib.ref_half_step.restype = ctypes.c_int
        lib.ref_half_step.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_long, vp,
                                      vp, vp, vp, ctypes.c_float, ctypes.c_int, vp, vp]
        _ref = lib
    return _ref


def ref_half_step(ptr32, col, val, theta, lam: float, x_batch: int = 1):
    """Run the reference's doALSWithCSR on the GPU. Returns (X float32, ms)."""
    lib = _load_ref()
    ptr32 = np.ascontiguousarray(ptr32, np.int32)
    col = np.ascontiguousarray(col, np.int32)
    val = np.ascontiguousarray(val, np.float32)
    theta = np.ascontiguousarray(theta, np.float32)
    m, (n, f) = len(ptr32) - 1, theta.shape
    X = np.zeros((m, f), np.float32)
    ms = ctypes.c_float(0.0)
    rc = lib.ref_half_step(m, n, f, len(col), _p(ptr32), _p(col), _p(val), _p(theta), lam,
                           x_batch, _p(X), ctypes.byref(ms))
    if rc != 0:
        raise RuntimeError(f"reference half-step failed ({rc})")
    return X, float(ms.value)
