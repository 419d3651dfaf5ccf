"""The C ABI: every entry point declared in include/*.h is exported by the
library that implements it, and argument errors come back as status codes
without touching a GPU."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import als_b200 as A

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")


# Declared with C++ linkage, as the reference's utilities.h:36-41 does; their
# exported names are mangled (checked by test_cxx_linkage_names).
CXX_LINKAGE = {"mallocBest": "_Z10mallocBestPPvm", "freeBest": "_Z8freeBestPv"}


def _declared(header):
    text = open(os.path.join(INC, header)).read()
    # the block of C++-linkage declarations
    text = re.sub(r"#ifdef __cplusplus\n\} /\* extern \"C\" \*/.*?#endif", "", text, flags=re.S)
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = set()
    for m in re.finditer(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", text):
        name = m.group(1)
        prev = text[:m.start()].rstrip()
        if name in {"if", "sizeof", "defined"} or prev.endswith("#define"):
            continue
        # a declaration: preceded by a type token and followed by a ';' after the ')'
        tail = text[m.end():]
        depth, j = 1, 0
        while depth and j < len(tail):
            depth += {"(": 1, ")": -1}.get(tail[j], 0)
            j += 1
        if tail[j:].lstrip().startswith(";") and re.search(r"[A-Za-z_*]\s*$", prev):
            names.add(name)
    return names


@pytest.mark.parametrize("header,libattr", [("als_b200.h", "lib"), ("cumf_jni.h", "lib"),
                                            ("als_data.h", "datalib")])
def test_every_declared_symbol_is_exported(header, libattr):
    names = _declared(header)
    assert len(names) >= 2
    lib = getattr(A, libattr)
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_dropin_symbols_match_reference_names():
    for n in ("doALSWithCSR", "get_gpu", "als_malloc_best", "als_free_best",
              "Java_org_apache_spark_ml_recommendation_CuMFJNIInterface_doALSWithCSR",
              "Java_org_apache_spark_ml_recommendation_CuMFJNIInterface_testjni"):
        assert hasattr(A.lib, n)
    for n in CXX_LINKAGE:  # C++ linkage only: no C name
        assert not hasattr(A.lib, n)


def _dynsyms(path):
    out = subprocess.run(["nm", "-D", "--defined-only", path], check=True, capture_output=True,
                         text=True).stdout
    return {line.split()[-1] for line in out.splitlines() if line.strip()}


def test_cxx_linkage_names():
    syms = _dynsyms(os.path.join(ROOT, "cuda-mllib_b200", "libGPUALS.so"))
    for mangled in CXX_LINKAGE.values():
        assert mangled in syms
    assert "doALSWithCSR" in syms and "get_gpu" in syms


def test_reference_style_cxx_caller_links_and_runs(tmp_path):
    """A C++ translation unit written against the reference's declarations
    (utilities.h:36-41, als.h:96-103) links against libGPUALS.so with every
    symbol resolved, and the drop-in's kernel-error check throws
    thrust::system_error across the library boundary (no GPU needed)."""
    pkg = os.path.join(ROOT, "cuda-mllib_b200")
    exe = str(tmp_path / "cxx_caller")
    # built for sm_100a like the library (and like the reference's JNI, which its
    # build compiles in one nvcc command with als.cu): the inline namespace of
    # thrust::system_error follows the target architecture
    subprocess.run(["nvcc", "-std=c++17", "-O1", "-gencode", "arch=compute_100a,code=sm_100a",
                    os.path.join(ROOT, "tests", "cxx_caller.cpp"),
                    "-o", exe, "-L" + pkg, "-lGPUALS", "-Xlinker", "-rpath," + pkg],
                   check=True, capture_output=True)
    run = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0, (run.stdout, run.stderr)
    assert "checks 7" in run.stdout
    assert "bounded wait timed out" in run.stderr


def test_default_options():
    o = A.options()
    assert o.precision == A.PREC_FP32 and o.solver == A.SOLVER_CHOLESKY
    assert o.cg_max_steps == 16 and abs(o.cg_tol - 1e-5) < 1e-12 and abs(o.refine_tol - 1e-5) < 1e-12
    with pytest.raises(KeyError):
        A.options(nonexistent=1)


def test_argument_errors_without_gpu():
    h = ctypes.c_void_p()
    rc = A.lib.als_model_create(ctypes.byref(h), 0, 10, 8, 0, None, None, None, None, None, None,
                                None, None)
    assert rc == A.ALS_ERR_INVALID and not h.value
    assert b"size" in A.lib.als_last_error()
    rc = A.lib.als_model_create(None, 1, 1, 1, 0, None, None, None, None, None, None, None, None)
    assert rc == A.ALS_ERR_INVALID
    rc = A.lib.als_half_step(-1, 1, 1, None, None, None, None, 1, None, 1, 0.1, None, None, 0, None)
    assert rc == A.ALS_ERR_INVALID
    o = A.options(precision=7)
    ptr = (ctypes.c_int64 * 2)(0, 0)
    rc = A.lib.als_model_create(ctypes.byref(h), 1, 1, 4, 0, ctypes.addressof(ptr), None, None,
                                ctypes.addressof(ptr), None, None, ctypes.byref(o), None)
    assert rc == A.ALS_ERR_INVALID and b"precision" in A.lib.als_last_error()
    o = A.options(precision=A.PREC_FP32)
    rc = A.lib.als_model_create(ctypes.byref(h), 1, 1, 129, 0, ctypes.addressof(ptr), None, None,
                                ctypes.addressof(ptr), None, None, ctypes.byref(o), None)
    assert rc == A.ALS_ERR_UNSUPPORTED
    rc = A.lib.als_train(None, None, None, None, None, None, 1, 1, 1, 0, 0.1, 1, None, None, None, None)
    assert rc == A.ALS_ERR_INVALID


def test_host_half_step_argument_errors_without_gpu():
    """als_half_step_host checks sizes and the host row pointers before any
    CUDA call: decreasing pointers, pointers that do not start at 0 or end at
    nnz, and range counts above 16 are ALS_ERR_INVALID; m = 0 has nothing to
    solve and returns ALS_OK."""
    f, n = 4, 3
    th = np.zeros((n, f), np.float32)
    X = np.zeros((2, f), np.float32)
    col = np.array([0, 1, 2], np.int32)
    val = np.ones(3, np.float32)
    fn = A.lib.als_half_step_host

    def call(ptr, m=2, nnz=3, chunks=0, theta=th):
        p = np.ascontiguousarray(ptr, np.int32)
        return fn(None, p.ctypes.data, col.ctypes.data, val.ctypes.data,
                  theta.ctypes.data if theta is not None else None, X.ctypes.data, m, n, f, nnz,
                  0.05, chunks)

    assert call([0, 2, 1]) == A.ALS_ERR_INVALID and b"span" in A.lib.als_last_error()
    assert call([0, 2, 1, 3], m=3) == A.ALS_ERR_INVALID and b"decreasing" in A.lib.als_last_error()
    assert call([1, 2, 3]) == A.ALS_ERR_INVALID
    assert call([0, 1, 3], chunks=17) == A.ALS_ERR_INVALID
    assert call([0, 1, 3], chunks=-1) == A.ALS_ERR_INVALID
    assert call([0, 1, 3], theta=None) == A.ALS_ERR_INVALID
    assert call([0, 1, 3], m=-1) == A.ALS_ERR_INVALID
    assert call([0], m=0, nnz=0) == A.ALS_OK


def test_version_string():
    assert "sm_100a" in A.version()
