"""The C ABI: every entry point declared in include/*.h is exported by the
library that implements it, and argument errors come back as status codes
without touching a GPU."""
import ctypes
import os
import re

import pytest

import als_b200 as A

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")


def _declared(header):
    text = open(os.path.join(INC, header)).read()
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
    for n in ("doALSWithCSR", "get_gpu", "mallocBest", "freeBest",
              "Java_org_apache_spark_ml_recommendation_CuMFJNIInterface_doALSWithCSR",
              "Java_org_apache_spark_ml_recommendation_CuMFJNIInterface_testjni"):
        assert hasattr(A.lib, n)


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


def test_version_string():
    assert "sm_100a" in A.version()
