"""The batched kernel's autotuner (rwig_b200/autotune.py) on the GPU: it
times a mixed batch under a coordinate search of the batch.* options, keeps
a setting no slower than the one it started from, leaves it set, and the
batched results under the tuned setting still match the CPU oracle
(Sinkhorn::compute_log restated) at the parity tolerance."""
import ctypes
import math

import pytest

import rwig_b200 as rw
from rwig_b200 import _lib
from rwig_b200.autotune import OPTIONS
from tests.test_gpu_batch import _check, _problem

pytestmark = pytest.mark.gpu

SIZES = [(64, 64, 0.05, 2), (300, 200, 0.1, 3), (1024, 700, 0.05, 2), (2500, 300, 0.1, 64), (700, 3000, 0.05, 2),
         (4096, 128, 0.1, 3), (150, 150, 0.01, 2), (2048, 2048, 0.05, 2)]


def _clear():
    L = _lib.load()
    for n in OPTIONS:
        L.rwig_set_option(n.encode(), float("nan"))


def test_autotune_keeps_results_and_sets_options():
    probs = [_problem(m, n, reg, dim, salt=i + 3, tol=1e-7) for i, (m, n, reg, dim) in enumerate(SIZES)]
    space = {"batch.max_team": [29.0, 59.0, 88.0], "batch.resident_team": [16.0, 64.0],
             "batch.stream_strip_kb": [512.0, 2048.0]}
    try:
        r = rw.autotune_batch(probs, space=space, reps=2)
        assert set(r) == {"options", "ms", "start_ms", "speedup", "trials", "rejected"}
        assert r["ms"] <= r["start_ms"] and r["speedup"] >= 1.0
        assert len(r["trials"]) >= 1 + 3 + 2 + 2 - 3  # the start plus every candidate not equal to it
        assert not r["rejected"], r["rejected"]
        L = _lib.load()
        v = ctypes.c_double()
        for name, val in r["options"].items():
            assert L.rwig_get_option(name.encode(), ctypes.byref(v)) == 0 and v.value == val, name
        out = rw.batch_sinkhorn_log(probs)
        assert all(o["path"] == 0 for o in out)
        for q, o in zip(probs, out):
            _check(q, o)
    finally:
        _clear()


def test_autotune_without_apply_restores_options():
    probs = [_problem(m, n, reg, dim, salt=i + 40, tol=1e-7) for i, (m, n, reg, dim) in enumerate(SIZES[:4])]
    L = _lib.load()
    try:
        assert L.rwig_set_option(b"batch.resident_team", 48.0) == 0
        r = rw.autotune_batch(probs, space={"batch.resident_team": [16.0, 64.0]}, reps=1, apply=False)
        assert r["trials"][0][0] == {"batch.resident_team": 48.0}
        v = ctypes.c_double()
        assert L.rwig_get_option(b"batch.resident_team", ctypes.byref(v)) == 0 and v.value == 48.0
        assert L.rwig_get_option(b"batch.max_team", ctypes.byref(v)) == 1
        assert math.isfinite(r["ms"])
    finally:
        _clear()
