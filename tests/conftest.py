"""Shared test set-up: import paths, the `gpu` marker, and in-tree builds.

Tests marked `gpu` need a B200; everything else runs on CPU. The engine and
checker libraries are built in-tree on first use if they are missing.
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "cuda-mllib_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def _ensure_built():
    need = [os.path.join(PKG, "libGPUALS.so"), os.path.join(PKG, "libalsdata.so"),
            os.path.join(ROOT, "oracle", "liboracle.so")]
    if not all(os.path.exists(p) for p in need):
        subprocess.run(["make", "-C", PKG, "-j8", "-s"], check=True)
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "-s"], check=True)


_ensure_built()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def pytest_collection_modifyitems(config, items):
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)
