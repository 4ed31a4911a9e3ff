"""Host logic of the batched kernel's autotuner (rwig_b200/autotune.py) and
the option calls it rests on (rwig_set_option / rwig_get_option), without a
GPU: the coordinate search against synthetic costs."""
import ctypes
import math

import pytest

from rwig_b200 import _lib
from rwig_b200.autotune import coordinate_search, default_space, defaults


def _cost(target):
    """Synthetic time in ms: 10 plus a separable penalty away from target
    (each step towards it gains more than the 2 % noise threshold)."""
    def measure(opts):
        return 10.0 + sum((math.log2(opts[k]) - math.log2(v)) ** 2 for k, v in target.items())
    return measure


def test_search_finds_separable_optimum():
    space = {"x": [1.0, 2.0, 4.0, 8.0], "y": [16.0, 32.0, 64.0]}
    best, ms, trials = coordinate_search(_cost({"x": 4.0, "y": 64.0}), space, {"x": 1.0, "y": 16.0})
    assert best == {"x": 4.0, "y": 64.0} and ms == 10.0
    assert trials[0] == ({"x": 1.0, "y": 16.0}, 10.0 + 4.0 + 4.0)
    assert len(trials) == 1 + 3 + 2  # the start, then every other candidate once


def test_search_never_worse_than_start_and_ignores_noise():
    space = {"x": [1.0, 2.0]}
    # a 1 % gain is below min_gain (2 %): the start stays
    best, ms, _ = coordinate_search(lambda o: 100.0 if o["x"] == 1.0 else 99.0, space, {"x": 1.0})
    assert best == {"x": 1.0} and ms == 100.0
    best, ms, _ = coordinate_search(lambda o: 100.0 if o["x"] == 1.0 else 90.0, space, {"x": 1.0})
    assert best == {"x": 2.0} and ms == 90.0


def test_rejected_trials_are_skipped():
    space = {"x": [1.0, 2.0, 3.0]}
    best, ms, trials = coordinate_search(lambda o: None if o["x"] == 2.0 else (50.0 if o["x"] == 3.0 else 80.0),
                                         space, {"x": 1.0})
    assert best == {"x": 3.0} and ms == 50.0 and ({"x": 2.0}, None) in trials
    with pytest.raises(RuntimeError):
        coordinate_search(lambda o: None, space, {"x": 1.0})


def test_default_space_contains_defaults():
    for sm in (132, 148):
        d, sp = defaults(sm), default_space(sm)
        assert set(d) == set(sp)
        for k, v in d.items():
            assert v in sp[k], (k, v, sp[k])


def test_get_set_clear_option():
    L = _lib.load()
    v = ctypes.c_double()
    try:
        assert L.rwig_set_option(b"batch.resident_team", 48.0) == 0
        assert L.rwig_get_option(b"batch.resident_team", ctypes.byref(v)) == 0 and v.value == 48.0
        assert L.rwig_set_option(b"batch.resident_team", float("nan")) == 0
        assert L.rwig_get_option(b"batch.resident_team", ctypes.byref(v)) == 1
    finally:
        L.rwig_set_option(b"batch.resident_team", float("nan"))
    assert L.rwig_get_option(b"no.such.option", ctypes.byref(v)) < 0
    assert L.rwig_set_option(b"no.such.option", 1.0) < 0
