"""Pins the CPU oracle against rwig's own known-answer vectors.

The expected values come from inst/tinytest/test_sinkhorn.R and
inst/tinytest/test_barycenter.R (Julia/ForwardDiff restatements), extracted into
tests/golden/tinytest_golden.json by tests/golden/make_golden.py.  The
tolerance and statistic are the reference's: all.equal's mean relative
difference at 10*sqrt(eps).
"""
import numpy as np
import pytest

import oracle
from tests.util import GOLDEN_TOL, mean_rel_diff


def _sk_inputs(golden):
    g = golden["sinkhorn"]["inputs"]
    return np.array(g["a"]), np.array(g["b"]), np.array(g["C"]), g["reg"]


def _bc_inputs(golden):
    g = golden["barycenter"]["inputs"]
    return np.array(g["A"]), np.array(g["C"]), np.array(g["w"]), np.array(g["b"]), g["reg"]


def test_vanilla_sinkhorn_golden(golden):
    a, b, C, reg = _sk_inputs(golden)
    r = oracle.sinkhorn_vanilla(a, b, C, reg, with_grad=True)
    exp = golden["sinkhorn"]["vanilla"]
    for k in ("loss", "P", "u", "v", "grad_a"):
        assert mean_rel_diff(exp[k], r[k]) <= GOLDEN_TOL, k
    assert r["return_status"] == 0


@pytest.mark.parametrize("n_threads", [0, 4])
def test_log_sinkhorn_golden(golden, n_threads):
    a, b, C, reg = _sk_inputs(golden)
    r = oracle.sinkhorn_log(a, b, C, reg, with_grad=True, n_threads=n_threads)
    exp = golden["sinkhorn"]["log"]
    for k in ("loss", "P", "f", "g", "grad_a"):
        assert mean_rel_diff(exp[k], r[k]) <= GOLDEN_TOL, k


def test_parallel_barycenter_golden(golden):
    A, C, w, b, reg = _bc_inputs(golden)
    r = oracle.barycenter_parallel(A, C, w, b, reg, with_grad=True)
    exp = golden["barycenter"]["parallel"]
    for k in ("loss", "U", "V", "grad_A", "grad_w", "b"):
        assert mean_rel_diff(exp[k], r[k]) <= GOLDEN_TOL, k


@pytest.mark.parametrize("n_threads", [0, 4])
def test_log_barycenter_golden(golden, n_threads):
    A, C, w, b, reg = _bc_inputs(golden)
    r = oracle.barycenter_log(A, C, w, b, reg, with_grad=True, n_threads=n_threads)
    exp = golden["barycenter"]["log"]
    # F and G are printed by the generator but never checked by the R tests;
    # they are pinned here as well.
    for k in ("loss", "grad_A", "grad_w", "F", "G", "b"):
        assert mean_rel_diff(exp[k], r[k]) <= GOLDEN_TOL, k


def test_threaded_equals_serial():
    from rwig_b200 import synth
    a, b, C = synth.sinkhorn_problem(37, 29, 0.5)
    s = oracle.sinkhorn_log(a, b, C, 0.05, n_threads=0, max_iter=50, zero_tol=0)
    t = oracle.sinkhorn_log(a, b, C, 0.05, n_threads=3, max_iter=50, zero_tol=0)
    assert np.array_equal(s["f"], t["f"]) and np.array_equal(s["g"], t["g"])


def _fd(fun, x, h=1e-6, mask=None):
    g = np.zeros_like(x)
    for k in range(x.size):
        if mask is not None and not mask.flat[k]:
            continue
        xp, xm = x.copy(), x.copy()
        xp.flat[k] += h
        xm.flat[k] -= h
        g.flat[k] = (fun(xp) - fun(xm)) / (2 * h)
    return g


def _fd_check(fun, x, grad, tol=1e-6, mask=None):
    """Central differences with h = 1e-6 over the entries selected by mask."""
    g = _fd(fun, x, mask=mask)
    sel = np.ones(x.shape, bool) if mask is None else mask
    assert sel.any()
    assert np.abs(g[sel] - np.asarray(grad)[sel]).max() <= tol * max(1.0, np.abs(g[sel]).max())


def test_log_barycenter_gradient_fd():
    """Central finite differences (h=1e-6) of the oracle's unrolled gradient.

    The reference seeds the adjoint with 2 (b - b_ext) o b for the normalised b
    (barycenter_impl_log.cpp:324), i.e. it differentiates ||exp(logb)/Z0 - b_ext||^2
    with the normaliser Z0 held at its value; that is the objective checked here."""
    from rwig_b200 import synth
    A, C, w, be = synth.barycenter_config(n=12, S=3, dim=4)
    L, reg = 15, 0.1
    r = oracle.barycenter_log(A, C, w, be, reg, with_grad=True, max_iter=L, zero_tol=0)
    Z0 = r["b_raw"].sum()

    def obj(A_, w_):
        q = oracle.barycenter_log(A_, C, w_, be, reg, True, max_iter=L, zero_tol=0)
        return float(((q["b_raw"] / Z0 - be) ** 2).sum())

    # log(A) needs A +- h > 0: differentiate the entries well above h
    _fd_check(lambda X: obj(X, w), A, r["grad_A"], mask=A > 1e-3)
    _fd_check(lambda x: obj(A, x), w, r["grad_w"])


def test_parallel_barycenter_gradient_fd():
    """The parallel adjoint differentiates ||b - b_ext||^2 with the un-normalised
    b (barycenter_impl_parallel.cpp:180)."""
    from rwig_b200 import synth
    A, C, w, be = synth.barycenter_config(n=10, S=3, dim=3)
    L, reg = 12, 0.2
    r = oracle.barycenter_parallel(A, C, w, be, reg, with_grad=True, max_iter=L, zero_tol=0)

    def obj(A_, w_):
        q = oracle.barycenter_parallel(A_, C, w_, be, reg, True, max_iter=L, zero_tol=0)
        return float(((q["b_raw"] - be) ** 2).sum())

    _fd_check(lambda X: obj(X, w), A, r["grad_A"])
    _fd_check(lambda x: obj(A, x), w, r["grad_w"])


@pytest.mark.parametrize("kind", ["vanilla", "log"])
def test_sinkhorn_gradient_fd(kind):
    """grad_a of the regularised loss, checked by central differences."""
    from rwig_b200 import synth
    a, b, C = synth.sinkhorn_problem(9, 7, 1.0)
    reg, L = 0.2, 30
    f = oracle.sinkhorn_vanilla if kind == "vanilla" else oracle.sinkhorn_log
    r = f(a, b, C, reg, True, max_iter=L, zero_tol=0)
    _fd_check(lambda x: f(x, b, C, reg, False, max_iter=L, zero_tol=0)["loss"], a, r["grad_a"])


def test_wdl_batch_grad_fd():
    """WDL batched gradient (softmax-parametrised) against central differences of
    the summed un-normalised barycenter loss, averaged over the batch."""
    from rwig_b200 import synth
    N, S, D, L, reg = 8, 3, 2, 6, 0.2
    g = synth.rng(7)
    x = g.standard_normal((N, 3))
    C = synth.sq_euclid_cost(x, x)
    K = np.exp(-C / reg)
    Alpha = g.standard_normal((N, S))
    Lam = g.standard_normal((S, D))
    YB = synth.dirichlet(g, 1.0, N, D)
    A = oracle.col_softmax(Alpha)
    W = oracle.col_softmax(Lam)
    gA, gl = oracle.wdl_batch_grad(A, W, YB, K, L)

    def loss_alpha(Al):
        A_ = oracle.col_softmax(Al)
        tot = 0.0
        for d in range(D):
            q = oracle.barycenter_parallel(A_, C, W[:, d], YB[:, d], reg, True, max_iter=L, zero_tol=0)
            tot += float(((q["b_raw"] - YB[:, d]) ** 2).sum())
        return tot / D

    _fd_check(loss_alpha, Alpha, gA, tol=1e-5)
