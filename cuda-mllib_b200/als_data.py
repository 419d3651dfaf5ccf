"""Host-side synthetic data and CSR utilities of the B200 ALS engine.

ctypes bindings over ``include/als_data.h`` (``libalsdata.so``, host code
only): seeded generators with the shapes of the benchmark rating matrices,
the train/test split, the CSR transpose and the initial factors. Loading this
module loads no GPU code, so a CPU-only process (the CPU baseline) can
generate the same inputs as the engine.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))


def _load(name: str) -> ctypes.CDLL:
    path = os.path.join(_HERE, name)
    if not os.path.exists(path):
        raise ImportError(f"{path} is not built (run `make` in {_HERE})")
    return ctypes.CDLL(path)


datalib = _load("libalsdata.so")

c_i32, c_i64, c_u64, c_f32, c_f64 = (ctypes.c_int32, ctypes.c_int64, ctypes.c_uint64,
                                     ctypes.c_float, ctypes.c_double)
c_vp = ctypes.c_void_p


def _sig(fn, restype, *argtypes):
    fn.restype = restype
    fn.argtypes = list(argtypes)
    return fn


def _check(rc: int) -> None:
    if rc != 0:
        raise RuntimeError(f"libalsdata call failed ({rc})")


def _ptr(a) -> int:
    return 0 if a is None else a.ctypes.data


class SynthSpec(ctypes.Structure):
    _fields_ = [("m", c_i64), ("n", c_i64), ("planted_rank", c_i32), ("integer_ratings", c_i32),
                ("factor_sigma", c_f64), ("noise_sigma", c_f64), ("mu", c_f64),
                ("rating_min", c_f64), ("rating_max", c_f64), ("degree_law", c_i32),
                ("threads", c_i32), ("degree_p1", c_f64), ("degree_min", c_i64),
                ("degree_max", c_i64), ("item_zipf_s", c_f64), ("target_nnz", c_i64),
                ("seed", c_u64)]


_sig(datalib.als_synth_degrees, c_i32, c_vp, c_vp, c_vp)
_sig(datalib.als_synth_fill, c_i32, c_vp, c_vp, c_vp, c_vp)
_sig(datalib.als_split, c_i32, c_i64, c_vp, c_vp, c_vp, c_f64, c_u64, c_vp, c_vp, c_vp, c_vp,
     c_vp, c_vp, c_vp, c_vp, c_i32)
_sig(datalib.als_csr_transpose, c_i32, c_i64, c_i64, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_i32)
_sig(datalib.als_init_factors, c_i32, c_i64, c_i32, c_f64, c_u64, c_vp, c_i32)
_sig(datalib.als_load_csr_bin, c_i32, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, c_vp,
     c_vp, c_vp, c_i64, c_i64)
_sig(datalib.als_save_csr_bin, c_i32, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, c_vp,
     c_vp, c_vp, c_i64, c_i64)



# ---------------------------------------------------------------------------
# synthetic data
# ---------------------------------------------------------------------------

@dataclass
class Ratings:
    m: int
    n: int
    csr_ptr: np.ndarray   # int64 [m+1]  train, users x items
    csr_col: np.ndarray   # int32 [nnz]
    csr_val: np.ndarray   # float32 [nnz]
    csc_ptr: np.ndarray   # int64 [n+1]  train, items x users
    csc_row: np.ndarray   # int32 [nnz]
    csc_val: np.ndarray   # float32 [nnz]
    test_u: np.ndarray    # int32 [nt]
    test_i: np.ndarray    # int32 [nt]
    test_r: np.ndarray    # float32 [nt]
    seed: int = 0

    @property
    def nnz(self) -> int:
        return int(self.csr_ptr[-1])


# Synthetic stand-ins with the published shapes of the rating matrices the
# reference is run on (no dataset records are reproduced). Sizes, value ranges
# and degree laws follow the benchmark configurations; mu is the centre of the
# rating range, factor_sigma gives <u,v> unit variance where the configuration
# does not state it.
CONFIGS = {
    # MovieLens-1M shape: plain FP32, f=10
    "ml1m": dict(m=6040, n=3706, target_nnz=1_000_000, planted_rank=10, factor_sigma=10 ** -0.5,
                 noise_sigma=0.5, mu=3.0, rating_min=1, rating_max=5, integer_ratings=1,
                 degree_law=0, degree_p1=1.0, degree_min=20, degree_max=0, item_zipf_s=1.0,
                 test_fraction=0.10, f=10, lam=0.05, iters=10),
    # Netflix shape: f=100, the headline workload
    "netflix": dict(m=480_189, n=17_770, target_nnz=100_500_000, planted_rank=100,
                    factor_sigma=100 ** -0.25, noise_sigma=0.8, mu=3.0, rating_min=1,
                    rating_max=5, integer_ratings=1, degree_law=0, degree_p1=1.2, degree_min=1,
                    degree_max=0, item_zipf_s=1.1, test_fraction=1.4e6 / 100.5e6, f=100,
                    lam=0.05, iters=10),
    # Yahoo!-Music shape: power-law users, 0..100 ratings
    "yahoo": dict(m=1_000_990, n=624_961, target_nnz=252_800_000, planted_rank=64,
                  factor_sigma=64 ** -0.25, noise_sigma=8.0, mu=50.0, rating_min=0,
                  rating_max=100, integer_ratings=1, degree_law=1, degree_p1=1.8, degree_min=1,
                  degree_max=100_000, item_zipf_s=1.2, test_fraction=0.01, f=100, lam=1.0,
                  iters=10),
}
CONFIGS["netflix128"] = dict(CONFIGS["netflix"], f=128)
# Tall-skinny shape with ~3.1 billion ratings (int64 row pointers): lognormal
# users (mean ~62), Zipf s=1.05 items, float ratings in [0, 5]; 1% held out
CONFIGS["hugewiki"] = dict(m=50_082_604, n=39_781, target_nnz=3_100_000_000, planted_rank=100,
                           factor_sigma=100 ** -0.25, noise_sigma=0.5, mu=2.5, rating_min=0,
                           rating_max=5, integer_ratings=0, degree_law=0, degree_p1=1.2,
                           degree_min=1, degree_max=0, item_zipf_s=1.05, test_fraction=0.01,
                           f=100, lam=0.05, iters=10)


def scaled_config(name: str, scale: float) -> dict:
    """A configuration with m, n and nnz scaled down (degree laws kept)."""
    c = dict(CONFIGS[name])
    c["m"] = max(8, int(c["m"] * scale))
    c["n"] = max(8, int(c["n"] * scale))
    c["target_nnz"] = max(16, int(c["target_nnz"] * scale * scale))
    if c["degree_max"]:
        c["degree_max"] = max(1, int(c["degree_max"] * scale))
    return c


def row_scaled_config(name: str, scale: float) -> dict:
    """A configuration with m and nnz scaled (n and the degree laws kept)."""
    c = dict(CONFIGS[name])
    c["m"] = max(8, int(c["m"] * scale))
    c["target_nnz"] = max(16, int(c["target_nnz"] * scale))
    return c


def synth(cfg: dict, seed: int = 1, threads: int = 0) -> Ratings:
    """Generate a seeded rating matrix, split it, and build both sides."""
    s = SynthSpec()
    for k, _ in SynthSpec._fields_:
        if k in cfg:
            setattr(s, k, cfg[k])
    s.seed, s.threads = seed, threads
    m, n = int(s.m), int(s.n)
    deg = np.zeros(m, np.int64)
    tot = c_i64(0)
    _check(datalib.als_synth_degrees(ctypes.byref(s), _ptr(deg), ctypes.byref(tot)))
    ptr = np.zeros(m + 1, np.int64)
    np.cumsum(deg, out=ptr[1:])
    col = np.empty(int(tot.value), np.int32)
    val = np.empty(int(tot.value), np.float32)
    _check(datalib.als_synth_fill(ctypes.byref(s), _ptr(ptr), _ptr(col), _ptr(val)))
    del deg
    frac = float(cfg.get("test_fraction", 0.0))
    trc = np.empty(m, np.int64)
    tec = np.empty(m, np.int64)
    _check(datalib.als_split(m, _ptr(ptr), _ptr(col), _ptr(val), frac, seed + 7919, _ptr(trc),
                             _ptr(tec), 0, 0, 0, 0, 0, 0, threads))
    tr_ptr = np.zeros(m + 1, np.int64)
    np.cumsum(trc, out=tr_ptr[1:])
    te_ptr = np.zeros(m + 1, np.int64)
    np.cumsum(tec, out=te_ptr[1:])
    tr_col = np.empty(int(tr_ptr[-1]), np.int32)
    tr_val = np.empty(int(tr_ptr[-1]), np.float32)
    te_col = np.empty(int(te_ptr[-1]), np.int32)
    te_val = np.empty(int(te_ptr[-1]), np.float32)
    _check(datalib.als_split(m, _ptr(ptr), _ptr(col), _ptr(val), frac, seed + 7919, 0, 0,
                             _ptr(tr_ptr), _ptr(tr_col), _ptr(tr_val), _ptr(te_ptr),
                             _ptr(te_col), _ptr(te_val), threads))
    del col, val
    csc_ptr, csc_row, csc_val = transpose(m, n, tr_ptr, tr_col, tr_val, threads)
    test_u = np.repeat(np.arange(m, dtype=np.int32), np.diff(te_ptr))
    return Ratings(m, n, tr_ptr, tr_col, tr_val, csc_ptr, csc_row, csc_val, test_u, te_col,
                   te_val, seed)


def transpose(m, n, ptr, col, val, threads: int = 0):
    """CSR (m x n) -> CSC (the CSR of the transpose), rows ascending per column."""
    cptr = np.zeros(n + 1, np.int64)
    rows = np.empty(len(col), np.int32)
    vals = np.empty(len(col), np.float32)
    _check(datalib.als_csr_transpose(m, n, _ptr(ptr), _ptr(col), _ptr(val), _ptr(cptr),
                                     _ptr(rows), _ptr(vals), threads))
    return cptr, rows, vals


def init_factors(rows: int, f: int, seed: int, sigma: float | None = None,
                 threads: int = 0) -> np.ndarray:
    """Seeded N(0, 1/f) initial factors (rows x f, float32)."""
    out = np.empty((rows, f), np.float32)
    sig = (1.0 / f) ** 0.5 if sigma is None else sigma
    _check(datalib.als_init_factors(rows, f, sig, seed, _ptr(out), threads))
    return out


def flop_per_iteration(r: Ratings, f: int) -> float:
    """Algorithmic FLOPs of one full iteration (both sides), solver-independent:
    sum over sides of nnz*f*(f+1) + 2*nnz*f + rows*(f^3/3 + 2 f^2)."""
    per_side = r.nnz * f * (f + 1) + 2 * r.nnz * f
    return 2 * per_side + (r.m + r.n) * (f ** 3 / 3 + 2 * f * f)
