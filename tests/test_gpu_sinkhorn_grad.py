"""Gradient of the Sinkhorn loss w.r.t. a on the GPU (rwig_sinkhorn_vanilla /
rwig_sinkhorn_log with withgrad = 1) against the CPU oracle's unrolled
backward (Sinkhorn::_bwd_vanilla, src/sinkhorn_impl_vanilla.cpp:169-213, and
Sinkhorn::_bwd_log, src/sinkhorn_impl_log.cpp:379-520, restated) and rwig's
known-answer vectors (inst/tinytest/test_sinkhorn.R)."""
import numpy as np
import pytest

import oracle
import rwig_b200 as rw
from rwig_b200 import synth
from tests.util import GOLDEN_TOL, PARITY_TOL, mean_rel_diff, rel_err

pytestmark = pytest.mark.gpu

ORACLE = {"vanilla": oracle.sinkhorn_vanilla, "log": oracle.sinkhorn_log}


def _compare(method, a, b, C, reg, max_iter=1000, zero_tol=1e-9):
    ref = ORACLE[method](a, b, C, reg, with_grad=True, max_iter=max_iter, zero_tol=zero_tol)
    got = rw.sinkhorn(a, b, C, {"reg": reg, "method": method, "with_grad": True, "max_iter": max_iter,
                                "zero_tol": zero_tol})
    assert got["iter"] == ref["iter"], (got["iter"], ref["iter"])
    assert got["return_status"] == ref["return_status"]
    # normwise against max|grad_a|; a gradient that is zero in exact arithmetic
    # (one row of support: a = [1] cannot move) leaves rounding residue of the
    # size of the loss's terms, so the loss bounds the scale from below
    sc = max(float(np.abs(ref["grad_a"]).max()), abs(ref["loss"]))
    e = rel_err(got["grad_a"], ref["grad_a"], sc)
    assert e <= PARITY_TOL, e
    assert abs(got["loss"] - ref["loss"]) <= PARITY_TOL * abs(ref["loss"])
    return got, ref


@pytest.mark.parametrize("method", ["vanilla", "log"])
def test_golden_vectors(golden, method):
    g = golden["sinkhorn"]
    a, b, C = np.array(g["inputs"]["a"]), np.array(g["inputs"]["b"]), np.array(g["inputs"]["C"])
    reg = g["inputs"]["reg"]
    r = rw.sinkhorn(a, b, C, {"reg": reg, "method": method, "with_grad": True})
    assert mean_rel_diff(g[method]["grad_a"], r["grad_a"]) <= GOLDEN_TOL
    assert mean_rel_diff(g[method]["loss"], r["loss"]) <= GOLDEN_TOL
    _compare(method, a, b, C, reg, zero_tol=1e-6)


@pytest.mark.parametrize("method", ["vanilla", "log"])
@pytest.mark.parametrize("m,n,reg", [
    (64, 64, 0.1), (100, 37, 0.2), (37, 100, 0.2), (513, 300, 0.1), (1500, 700, 0.05),
    (2048, 900, 0.1), (4096, 256, 0.1), (6000, 300, 0.1), (1, 5, 0.1), (5, 1, 0.1), (2, 2, 0.5),
])
def test_parity_shapes(method, m, n, reg):
    a, b, C = synth.sinkhorn_problem(m, n, 1.0, salt=m * 17 + n)
    _compare(method, a, b, C, reg)


@pytest.mark.parametrize("method", ["vanilla", "log"])
@pytest.mark.parametrize("iters", [0, 1, 2, 15, 200])
def test_pinned_iterations(method, iters):
    """Fixed unroll depth L: every step of the backward is exercised, the
    first and last steps alone at L = 1, 2; L = 0 gives a zero gradient."""
    a, b, C = synth.sinkhorn_problem(300, 200, 1.0, salt=7)
    got, _ = _compare(method, a, b, C, 0.05, max_iter=iters, zero_tol=0.0)
    assert got["iter"] == iters
    if iters == 0:
        assert not got["grad_a"].any()


@pytest.mark.parametrize("method", ["vanilla", "log"])
def test_support_reduction(method):
    """Zero masses drop out of the problem; the gradient is zero there."""
    a, b, C = synth.sinkhorn_problem(120, 90, 1.0, salt=11)
    a[[0, 5, 119]] = 0.0
    b[[3, 89]] = 0.0
    a /= a.sum()
    b /= b.sum()
    got, _ = _compare(method, a, b, C, 0.1)
    assert not got["grad_a"][[0, 5, 119]].any()


def test_log_small_reg():
    """The log form at a regularisation where K = exp(-C/eps) underflows."""
    a, b, C = synth.sinkhorn_problem(400, 300, 1.0, salt=13)
    _compare("log", a, b, C, 0.002, max_iter=300, zero_tol=1e-9)


def test_grad_is_deterministic():
    a, b, C = synth.sinkhorn_problem(700, 500, 1.0, salt=19)
    ctrl = {"reg": 0.05, "method": "log", "with_grad": True, "max_iter": 100, "zero_tol": 0.0}
    g1 = rw.sinkhorn(a, b, C, ctrl)["grad_a"]
    g2 = rw.sinkhorn(a, b, C, ctrl)["grad_a"]
    assert np.array_equal(g1, g2)


def test_rows_beyond_limit_rejected():
    a, b, C = synth.sinkhorn_problem(8193, 8, 1.0, salt=23)
    with pytest.raises(rw.RwigError):
        rw.sinkhorn(a, b, C, {"reg": 0.1, "method": "log", "with_grad": True, "max_iter": 5})
