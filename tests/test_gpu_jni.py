"""The Spark JNI entry point, driven through a fake JNIEnv (no JVM here).

tests/jni_fake.c implements the JNI functions the shim uses, at the slots of
the JNI specification's function table, over plain C arrays. The call must
return float[m][f] equal to the drop-in doALSWithCSR result."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import als_b200 as A
import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))


def _fake():
    so = os.path.join(HERE, "_build", "libjni_fake.so")
    src = os.path.join(HERE, "jni_fake.c")
    if not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(src):
        os.makedirs(os.path.dirname(so), exist_ok=True)
        subprocess.run(["gcc", "-O2", "-fPIC", "-shared", "-o", so, src], check=True)
    lib = ctypes.CDLL(so)
    vp = ctypes.c_void_p
    lib.fake_env.restype = vp
    lib.fake_float_array.restype = vp
    lib.fake_float_array.argtypes = [ctypes.c_int, vp]
    lib.fake_int_array.restype = vp
    lib.fake_int_array.argtypes = [ctypes.c_int, vp]
    lib.fake_object_array.restype = vp
    lib.fake_object_array.argtypes = [ctypes.c_int]
    lib.fake_set.argtypes = [vp, ctypes.c_int, vp]
    lib.fake_length.restype = ctypes.c_int
    lib.fake_length.argtypes = [vp]
    lib.fake_get.restype = vp
    lib.fake_get.argtypes = [vp, ctypes.c_int]
    lib.fake_float_data.restype = ctypes.POINTER(ctypes.c_float)
    lib.fake_float_data.argtypes = [vp]
    lib.fake_live_critical.restype = ctypes.c_int
    lib.fake_open_frames.restype = ctypes.c_int
    lib.fake_max_frames.restype = ctypes.c_int
    return lib


def test_fake_env_builds():
    lib = _fake()
    assert lib.fake_env()


@pytest.mark.gpu
def test_jni_doALSWithCSR_through_fake_env():
    fk = _fake()
    r = A.synth(A.scaled_config("ml1m", 0.1), seed=8)
    f = 10
    th = A.init_factors(r.n, f, 1)
    # Spark passes the source factors as blocks: float[blocks][factors][f]
    blocks = np.array_split(np.arange(r.n), 3)
    outer = fk.fake_object_array(len(blocks))
    keep = []
    for b, idx in enumerate(blocks):
        blk = fk.fake_object_array(len(idx))
        for j, i in enumerate(idx):
            row = np.ascontiguousarray(th[i])
            keep.append(row)
            fk.fake_set(blk, j, fk.fake_float_array(f, row.ctypes.data))
        fk.fake_set(outer, b, blk)
    ptr32 = r.csr_ptr.astype(np.int32)
    jrow = fk.fake_int_array(len(ptr32), ptr32.ctypes.data)
    jcol = fk.fake_int_array(len(r.csr_col), r.csr_col.ctypes.data)
    jval = fk.fake_float_array(len(r.csr_val), r.csr_val.ctypes.data)
    fn = A.lib.Java_org_apache_spark_ml_recommendation_CuMFJNIInterface_doALSWithCSR
    fn.restype = ctypes.c_void_p
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                   ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p,
                   ctypes.c_void_p, ctypes.c_void_p]
    out = fn(fk.fake_env(), None, r.m, r.n, f, r.nnz, 0.05, outer, jrow, jcol, jval)
    assert out and fk.fake_length(out) == r.m
    X = np.array([np.ctypeslib.as_array(fk.fake_float_data(fk.fake_get(out, i)), (f,))
                  for i in range(r.m)])
    assert fk.fake_live_critical() == 0  # every critical section was released
    assert fk.fake_open_frames() == 0 and fk.fake_max_frames() >= 1  # local frames balanced
    X_ref, _ = O.half_step(r.csr_ptr, r.csr_col, r.csr_val, th, 0.05)
    err = np.linalg.norm(X - X_ref, axis=1) / np.maximum(np.linalg.norm(X_ref, axis=1), 1e-30)
    assert err.max() < 1e-3
    X2 = A.do_als_with_csr(ptr32, r.csr_col, r.csr_val, th, r.m, r.n, f, 0.05)
    assert np.array_equal(X, X2)
    # a second call reuses the shim's pooled pinned buffers and stream
    jrow = fk.fake_int_array(len(ptr32), ptr32.ctypes.data)
    jcol = fk.fake_int_array(len(r.csr_col), r.csr_col.ctypes.data)
    jval = fk.fake_float_array(len(r.csr_val), r.csr_val.ctypes.data)
    out2 = fn(fk.fake_env(), None, r.m, r.n, f, r.nnz, 0.05, outer, jrow, jcol, jval)
    assert out2 and fk.fake_open_frames() == 0
    X3 = np.array([np.ctypeslib.as_array(fk.fake_float_data(fk.fake_get(out2, i)), (f,))
                   for i in range(r.m)])
    assert np.array_equal(X, X3)


def _no_gpu():
    try:
        import torch
        return not torch.cuda.is_available()
    except Exception:
        return True


@pytest.mark.skipif(not _no_gpu(), reason="checks the path taken when no GPU is present")
def test_jni_without_gpu_returns_null():
    """Without a usable GPU the entry point reports the CUDA error and returns
    null, as the reference's catch block does (CuMFJNIInterface.cpp:129-131),
    instead of ending the executor process."""
    fk = _fake()
    f, n, m = 4, 3, 2
    th = np.arange(n * f, dtype=np.float32).reshape(n, f)
    outer = fk.fake_object_array(1)
    blk = fk.fake_object_array(n)
    keep = [np.ascontiguousarray(th[i]) for i in range(n)]
    for i, row in enumerate(keep):
        fk.fake_set(blk, i, fk.fake_float_array(f, row.ctypes.data))
    fk.fake_set(outer, 0, blk)
    ptr = np.array([0, 1, 2], np.int32)
    col = np.array([0, 2], np.int32)
    val = np.array([4.0, 5.0], np.float32)
    fn = A.lib.Java_org_apache_spark_ml_recommendation_CuMFJNIInterface_doALSWithCSR
    fn.restype = ctypes.c_void_p
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                   ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p,
                   ctypes.c_void_p, ctypes.c_void_p]
    out = fn(fk.fake_env(), None, m, n, f, 2, 0.05, outer,
             fk.fake_int_array(3, ptr.ctypes.data), fk.fake_int_array(2, col.ctypes.data),
             fk.fake_float_array(2, val.ctypes.data))
    assert not out
    assert fk.fake_live_critical() == 0


@pytest.mark.gpu
def test_jni_error_inside_dropin_returns_null():
    """A failure inside the half-step (here: a rank the FP32 form does not
    take, f = 129) reaches the shim's catch block, which reports it and
    returns null instead of letting the exception end the executor process
    (reference CuMFJNIInterface.cpp:129-131). The Java arrays' critical
    sections are released on that path too."""
    fk = _fake()
    f, n, m = 129, 3, 2
    th = np.arange(n * f, dtype=np.float32).reshape(n, f)
    outer = fk.fake_object_array(1)
    blk = fk.fake_object_array(n)
    keep = [np.ascontiguousarray(th[i]) for i in range(n)]
    for i, row in enumerate(keep):
        fk.fake_set(blk, i, fk.fake_float_array(f, row.ctypes.data))
    fk.fake_set(outer, 0, blk)
    ptr = np.array([0, 1, 2], np.int32)
    col = np.array([0, 2], np.int32)
    val = np.array([4.0, 5.0], np.float32)
    fn = A.lib.Java_org_apache_spark_ml_recommendation_CuMFJNIInterface_doALSWithCSR
    fn.restype = ctypes.c_void_p
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                   ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p,
                   ctypes.c_void_p, ctypes.c_void_p]
    for _ in range(3):  # repeated failures leave the process and the library usable
        out = fn(fk.fake_env(), None, m, n, f, 2, 0.05, outer,
                 fk.fake_int_array(3, ptr.ctypes.data), fk.fake_int_array(2, col.ctypes.data),
                 fk.fake_float_array(2, val.ctypes.data))
        assert not out
        assert fk.fake_live_critical() == 0
    # a valid call afterwards still works
    X = A.do_als_with_csr(ptr, col, val, th[:, :16].copy(), m, n, 16, 0.05)
    assert np.isfinite(X).all()


@pytest.mark.gpu
def test_jni_kernel_timeout_returns_null():
    """A half-step whose kernel gives up a bounded wait (forced by the test
    switch) fails instead of returning incomplete rows; the Spark shim reports
    it and returns null, and the next call is correct."""
    fk = _fake()
    r = A.synth(A.scaled_config("ml1m", 0.1), seed=8)
    f = 32
    th = A.init_factors(r.n, f, 1)
    outer = fk.fake_object_array(1)
    blk = fk.fake_object_array(r.n)
    keep = [np.ascontiguousarray(th[i]) for i in range(r.n)]
    for i, row in enumerate(keep):
        fk.fake_set(blk, i, fk.fake_float_array(f, row.ctypes.data))
    fk.fake_set(outer, 0, blk)
    ptr32 = r.csr_ptr.astype(np.int32)
    fn = A.lib.Java_org_apache_spark_ml_recommendation_CuMFJNIInterface_doALSWithCSR
    fn.restype = ctypes.c_void_p
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                   ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p,
                   ctypes.c_void_p, ctypes.c_void_p]
    old = A.get_dropin_options()
    try:
        A.set_dropin_options(A.options(precision=A.PREC_BF16, solver=A.SOLVER_CG))
        outs = []
        for withhold in (1, 0):
            A.lib.als_debug_withhold_first_row(withhold)
            jrow = fk.fake_int_array(len(ptr32), ptr32.ctypes.data)
            jcol = fk.fake_int_array(len(r.csr_col), r.csr_col.ctypes.data)
            jval = fk.fake_float_array(len(r.csr_val), r.csr_val.ctypes.data)
            outs.append(fn(fk.fake_env(), None, r.m, r.n, f, r.nnz, 0.05, outer, jrow, jcol, jval))
            assert fk.fake_live_critical() == 0 and fk.fake_open_frames() == 0
    finally:
        A.lib.als_debug_withhold_first_row(0)
        A.set_dropin_options(old)
    assert not outs[0]
    assert outs[1] and fk.fake_length(outs[1]) == r.m
