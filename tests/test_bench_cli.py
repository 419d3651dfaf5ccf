"""Host-side pieces of bench.py that need no GPU: the workload each flag set
selects and the name the JSON line gives it."""
import sys

import bench


def _args(monkeypatch, *argv):
    monkeypatch.setattr(sys, "argv", ["bench.py", *argv])
    return bench.parse()


def test_default_is_the_netflix_shape(monkeypatch):
    a = _args(monkeypatch)
    c = bench.cfg_of(a)
    assert (c["m"], c["n"], c["f"]) == (480_189, 17_770, 100)
    assert bench.workload_name(a) == bench.WORKLOAD
    assert (a.gpus, a.precision, a.solver, a.warm, a.graph) == (1, "bf16", "cg", "previous", False)
    assert a.warmup >= 3


def test_row_scale_keeps_the_items(monkeypatch):
    a = _args(monkeypatch, "--config", "hugewiki", "--row-scale", "0.1")
    c = bench.cfg_of(a)
    assert c["n"] == 39_781 and c["m"] == 5_008_260
    assert c["target_nnz"] == 310_000_000
    assert bench.workload_name(a) == "hugewiki rows x0.1"


def test_scale_shrinks_both_sides(monkeypatch):
    a = _args(monkeypatch, "--config", "yahoo", "--scale", "0.5", "--graph", "--precision", "fp16")
    c = bench.cfg_of(a)
    assert c["m"] == 500_495 and c["n"] == 312_480
    assert bench.workload_name(a) == "yahoo x0.5" and a.graph


def test_full_size_configs(monkeypatch):
    a = _args(monkeypatch, "--config", "hugewiki")
    c = bench.cfg_of(a)
    assert c["target_nnz"] == 3_100_000_000 and c["f"] == 100
    assert bench.workload_name(a) == "hugewiki"
    assert bench.cfg_of(_args(monkeypatch, "--config", "netflix128"))["f"] == 128
