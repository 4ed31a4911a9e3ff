"""Parity of the CUDA barycenters (rwig_barycenter_parallel / _log) with the CPU
oracle (Barycenter::compute_parallel / compute_log restated), rwig's
known-answer vectors, and central finite differences of the engine's own
gradients."""
import numpy as np
import pytest

import oracle
import rwig_b200 as rw
from rwig_b200 import synth
from tests.util import GOLDEN_TOL, PARITY_TOL, dual_scale, mean_rel_diff, rel_err

pytestmark = pytest.mark.gpu


def _compare(method, A, C, w, be, reg, with_grad=True, max_iter=1000, zero_tol=1e-6):
    f = oracle.barycenter_log if method == "log" else oracle.barycenter_parallel
    ref = f(A, C, w, be, reg, with_grad=with_grad, max_iter=max_iter, zero_tol=zero_tol)
    got = rw.barycenter(A, C, w, be if with_grad else None,
                        {"reg": reg, "method": method, "with_grad": with_grad, "max_iter": max_iter,
                         "zero_tol": zero_tol})
    assert got["iter"] == ref["iter"] and got["return_status"] == ref["return_status"]
    assert rel_err(got["b"], ref["b"]) <= PARITY_TOL, rel_err(got["b"], ref["b"])
    if method == "log":
        sc = dual_scale(ref["F"], ref["G"])
        for k in ("F", "G"):
            assert rel_err(got[k], ref[k], sc) <= PARITY_TOL, (k, rel_err(got[k], ref[k], sc))
    else:
        for k in ("U", "V"):
            assert rel_err(got[k], ref[k]) <= PARITY_TOL, (k, rel_err(got[k], ref[k]))
    if with_grad:
        for k in ("grad_A", "grad_w"):
            assert rel_err(got[k], ref[k]) <= PARITY_TOL, (k, rel_err(got[k], ref[k]))
        assert abs(got["loss"] - ref["loss"]) <= PARITY_TOL * abs(ref["loss"])
    assert abs(got["err"] - ref["err"]) <= 1e-8 * abs(ref["err"]) + 1e-13
    return got, ref


@pytest.mark.parametrize("method", ["parallel", "log"])
def test_golden_vectors(golden, method):
    g = golden["barycenter"]
    A, C = np.array(g["inputs"]["A"]), np.array(g["inputs"]["C"])
    w, be, reg = np.array(g["inputs"]["w"]), np.array(g["inputs"]["b"]), g["inputs"]["reg"]
    r = rw.barycenter(A, C, w, be, {"reg": reg, "method": method, "with_grad": True})
    keys = ("loss", "grad_A", "grad_w", "b") + (("U", "V") if method == "parallel" else ("F", "G"))
    for k in keys:
        assert mean_rel_diff(g[method][k], r[k]) <= GOLDEN_TOL, k
    _compare(method, A, C, w, be, reg)


@pytest.mark.parametrize("method", ["parallel", "log"])
@pytest.mark.parametrize("n,S,dim,reg,L,tol", [
    (64, 4, 3, 0.1, 1000, 1e-9), (200, 7, 5, 0.1, 30, 0.0), (256, 32, 50, 0.05, 50, 0.0),
    (513, 3, 2, 0.2, 1000, 1e-10), (2, 2, 2, 0.1, 5, 0.0),
])
def test_parity_shapes(method, n, S, dim, reg, L, tol):
    A, C, w, be = synth.barycenter_config(n=n, S=S, dim=dim, salt=n + S)
    _compare(method, A, C, w, be, reg, max_iter=L, zero_tol=tol)


@pytest.mark.parametrize("method", ["parallel", "log"])
def test_rectangular_cost(method):
    """M != N: histograms on M points, barycenter on N."""
    g = synth.rng(31)
    x, y = g.random((150, 3)), g.random((90, 3))
    C = synth.sq_euclid_cost(x, y)
    A = synth.dirichlet(g, 0.5, 150, 5)
    w = synth.dirichlet(g, 1.0, 5)
    be = synth.dirichlet(g, 1.0, 90)
    _compare(method, A, C, w, be, 0.1, max_iter=40, zero_tol=0.0)


@pytest.mark.parametrize("method", ["parallel", "log"])
def test_without_gradient(method):
    A, C, w, be = synth.barycenter_config(n=300, S=6, dim=4, salt=9)
    _compare(method, A, C, w, be, 0.1, with_grad=False, max_iter=1000, zero_tol=1e-8)


def _fd(fun, x, idx, h=1e-6):
    out = []
    for k in idx:
        xp, xm = x.copy(), x.copy()
        xp.flat[k] += h
        xm.flat[k] -= h
        out.append((fun(xp) - fun(xm)) / (2 * h))
    return np.array(out)


@pytest.mark.parametrize("method", ["parallel", "log"])
def test_gradient_finite_differences(method):
    """Central differences (h = 1e-6) of the engine's objective: ||b - b_ext||^2
    with the un-normalised b (parallel), or with the normaliser held at its
    value (log), which is what the reference's backward differentiates."""
    A, C, w, be = synth.barycenter_config(n=256, S=8, dim=10, salt=3)
    L, reg = 30, 0.05
    ctrl = {"reg": reg, "method": method, "with_grad": True, "max_iter": L, "zero_tol": 0.0}
    r = rw.barycenter(A, C, w, be, ctrl)
    Z0 = rw.last_report()["bary_norm"]

    def obj(A_, w_):
        q = rw.barycenter(A_, C, w_, be, ctrl)
        z = rw.last_report()["bary_norm"]
        braw = q["b"] * z
        return float((((braw / Z0) if method == "log" else braw) - be) @ (((braw / Z0) if method == "log" else braw) - be))

    gw = _fd(lambda x: obj(A, x), w, range(w.size))
    assert np.abs(gw - r["grad_w"]).max() <= 1e-6 * max(1.0, np.abs(gw).max())
    g = np.random.default_rng(0)
    idx = [k for k in g.choice(A.size, 40, replace=False) if A.flat[k] > 1e-3]
    gA = _fd(lambda X: obj(X, w), A, idx)
    assert np.abs(gA - r["grad_A"].flat[idx]).max() <= 1e-6 * max(1.0, np.abs(gA).max())


@pytest.mark.parametrize("method", ["parallel", "log"])
def test_graph_replay_is_bitwise_identical(method):
    """A fixed-iteration call that repeats is captured into a CUDA graph on the
    second call and replayed after that: eager, captured and replayed solves
    give the same bits, and a changed argument goes back to an eager run."""
    A, C, w, be = synth.barycenter_config(n=300, S=9, dim=4, salt=77)
    ctrl = {"reg": 0.1, "method": method, "with_grad": True, "max_iter": 12, "zero_tol": 0.0}
    runs = [rw.barycenter(A, C, w, be, ctrl) for _ in range(4)]
    for r in runs[1:]:
        for k in ("b", "grad_A", "grad_w"):
            assert np.array_equal(r[k], runs[0][k]), k
        assert r["loss"] == runs[0]["loss"] and r["err"] == runs[0]["err"] and r["iter"] == 12
    # new inputs at the same buffers: the replayed graph reads them afresh
    A2 = A[:, ::-1].copy()
    got = rw.barycenter(A2, C, w, be, ctrl)
    ref = rw.barycenter(A2, C, w, be, dict(ctrl, max_iter=13))  # a different sequence, eager
    assert got["iter"] == 12 and ref["iter"] == 13
    _compare(method, A2, C, w, be, 0.1, max_iter=12, zero_tol=0.0)


@pytest.mark.parametrize("method", ["parallel", "log"])
def test_zero_iterations(method):
    """max_iter = 0 with gradient: b is the initial b normalised (0/0 = NaN for
    parallel, 1/N for log) and the loss is taken against b_ext all the same
    (barycenter_impl_parallel.cpp:39-42, barycenter_impl_log.cpp:268-271);
    nothing is unrolled, so the gradients are zero."""
    A, C, w, be = synth.barycenter_config(n=50, S=3, dim=3, salt=4)
    f = oracle.barycenter_log if method == "log" else oracle.barycenter_parallel
    ref = f(A, C, w, be, 0.1, with_grad=True, max_iter=0, zero_tol=1e-6)
    got = rw.barycenter(A, C, w, be, {"reg": 0.1, "method": method, "with_grad": True, "max_iter": 0,
                                      "zero_tol": 1e-6})
    assert got["iter"] == ref["iter"] == 0 and got["return_status"] == ref["return_status"]
    assert rel_err(got["b"], ref["b"]) <= PARITY_TOL
    if method == "parallel":
        assert np.isnan(ref["loss"]) and np.isnan(got["loss"])
    else:
        assert abs(got["loss"] - ref["loss"]) <= PARITY_TOL * abs(ref["loss"])
    assert not got["grad_A"].any() and not got["grad_w"].any()


class _LogPath:
    """Sets the engine option barycenter.log_path for a block (NaN restores the default)."""

    def __init__(self, value):
        self.value = value

    def __enter__(self):
        rw.load().rwig_set_option(b"barycenter.log_path", float(self.value))

    def __exit__(self, *exc):
        rw.load().rwig_set_option(b"barycenter.log_path", float("nan"))


@pytest.mark.parametrize("n,S,dim,reg,L,tol,scale", [
    (200, 5, 3, 1e-3, 20, 0.0, 1.0),     # max C / eps = 1000 on a max-normalised cost
    (256, 8, 10, 1e-3, 15, 0.0, 1.0),
    (180, 6, 3, 0.05, 20, 0.0, 100.0),   # un-normalised cost, max C = 100: max C / eps = 2000
    (300, 4, 2, 0.05, 25, 0.0, 100.0),
    (150, 3, 2, 1e-3, 200, 1.0, 1.0),    # with a stopping test (stops at iteration 78)
])
def test_log_barycenter_where_the_gibbs_kernel_underflows(n, S, dim, reg, L, tol, scale):
    """exp(-C/eps) has entries that underflow to zero: the scaling form's range
    check fails and the solve runs in the log domain, as the reference's
    compute_log does (barycenter_impl_log.cpp:189-382), with its gradients."""
    A, C, w, be = synth.barycenter_config(n=n, S=S, dim=dim, salt=n + S)
    C = C * scale
    assert (np.exp(-C / reg) == 0).any()
    got, ref = _compare("log", A, C, w, be, reg, max_iter=L, zero_tol=tol)
    assert rw.last_report()["fallback_events"] == 1
    assert np.isfinite(got["grad_A"]).all() and np.isfinite(got["F"]).all()


def test_log_barycenter_scaling_form_kept_in_range():
    """Within range (max C / eps = 20) the scaling form's result stands."""
    A, C, w, be = synth.barycenter_config(n=256, S=8, dim=10, salt=5)
    _compare("log", A, C, w, be, 0.05, max_iter=30, zero_tol=0.0)
    assert rw.last_report()["fallback_events"] == 0


@pytest.mark.parametrize("n,m,S,reg,L,tol", [
    (64, 64, 4, 0.1, 1000, 1e-9), (200, 150, 7, 0.1, 30, 0.0), (256, 256, 32, 0.05, 50, 0.0),
    (513, 300, 3, 0.2, 40, 0.0), (2, 2, 2, 0.1, 5, 0.0), (90, 700, 17, 0.02, 12, 0.0), (1000, 64, 64, 0.1, 6, 0.0),
])
def test_log_domain_kernels_against_oracle(n, m, S, reg, L, tol):
    """The log-domain kernels forced on (barycenter.log_path = 1) at ordinary
    regularisation, rectangular costs and S up to 64."""
    g = synth.rng(41, n + m + S)
    x, y = g.random((n, 3)), g.random((m, 3))
    C = synth.sq_euclid_cost(x, y)
    A = synth.dirichlet(g, 0.5, n, S)
    w = synth.dirichlet(g, 1.0, S)
    be = synth.dirichlet(g, 1.0, m)
    with _LogPath(1):
        got, ref = _compare("log", A, C, w, be, reg, max_iter=L, zero_tol=tol)
        assert rw.last_report()["fallback_events"] == 1
        again = rw.barycenter(A, C, w, be, {"reg": reg, "method": "log", "with_grad": True, "max_iter": L,
                                            "zero_tol": tol})
    for k in ("b", "F", "G", "grad_A", "grad_w"):  # fixed-order reductions: repeatable bit for bit
        assert np.array_equal(again[k], got[k]), k


def test_log_domain_gradient_finite_differences():
    """Central differences (h = 1e-6) of ||b - b_ext||^2 with the normaliser held
    at its value, through the log-domain kernels (forced on)."""
    A, C, w, be = synth.barycenter_config(n=120, S=4, dim=3, salt=8)
    L, reg = 15, 0.05
    ctrl = {"reg": reg, "method": "log", "with_grad": True, "max_iter": L, "zero_tol": 0.0}
    with _LogPath(1):
        _fd_check(A, C, w, be, ctrl)


def _fd_check(A, C, w, be, ctrl):
    r = rw.barycenter(A, C, w, be, ctrl)
    assert rw.last_report()["fallback_events"] == 1
    Z0 = rw.last_report()["bary_norm"]

    def obj(A_, w_):
        q = rw.barycenter(A_, C, w_, be, ctrl)
        braw = q["b"] * rw.last_report()["bary_norm"] / Z0
        return float((braw - be) @ (braw - be))

    gw = _fd(lambda x: obj(A, x), w, range(w.size))
    assert np.abs(gw - r["grad_w"]).max() <= 1e-5 * max(1.0, np.abs(gw).max())
    g = np.random.default_rng(1)
    idx = [k for k in g.choice(A.size, 30, replace=False) if A.flat[k] > 1e-3]
    gA = _fd(lambda X: obj(X, w), A, idx)
    assert np.abs(gA - r["grad_A"].flat[idx]).max() <= 1e-5 * max(1.0, np.abs(gA).max())


def test_batched_log_barycenter_falls_back_per_problem():
    """In a batch, only the problems whose scaling form leaves its range are
    re-run in the log domain; every result equals the single call's."""
    probs = []
    for i, (n, S, reg, scale) in enumerate([(150, 4, 1e-3, 1.0), (160, 5, 0.1, 1.0), (170, 3, 0.05, 100.0)]):
        A, C, w, be = synth.barycenter_config(n=n, S=S, dim=3, salt=60 + i)
        probs.append({"A": A, "C": C * scale, "w": w, "b_ext": be, "reg": reg, "method": "log",
                      "with_grad": True, "max_iter": 10, "zero_tol": 0.0})
    got = rw.batch_barycenter(probs)
    for i, q in enumerate(probs):
        ref = rw.barycenter(q["A"], q["C"], q["w"], q["b_ext"],
                            {k: q[k] for k in ("reg", "method", "with_grad", "max_iter", "zero_tol")})
        for k in ("b", "F", "G", "grad_A", "grad_w"):
            assert np.array_equal(got[i][k], ref[k]), (i, k)
        o = oracle.barycenter_log(q["A"], q["C"], q["w"], q["b_ext"], q["reg"], with_grad=True, max_iter=10,
                                  zero_tol=0.0)
        assert rel_err(got[i]["grad_A"], o["grad_A"]) <= PARITY_TOL


def _bary2048():
    import os
    ref = np.load(os.path.join(os.path.dirname(__file__), "golden", "bary2048_oracle.npz"))
    A, C, w, be = synth.barycenter_config(n=2048, S=32, dim=50)
    return ref, A, C, w, be


def test_full_size_against_oracle_fixture():
    """The log-barycenter benchmark workload at full size (N = 2048, S = 32,
    eps = 0.05, L = 50, with gradient) against the CPU oracle's solve
    (tests/golden/bary2048_oracle.npz, made by tests/golden/make_fullsize.py)."""
    ref, A, C, w, be = _bary2048()
    got = rw.barycenter(A, C, w, be, {"reg": 0.05, "method": "log", "with_grad": True, "max_iter": 50,
                                      "zero_tol": 0.0})
    assert got["iter"] == int(ref["iter"]) == 50 and got["return_status"] == int(ref["return_status"])
    for k in ("b", "grad_A", "grad_w"):
        assert rel_err(got[k], ref[k]) <= PARITY_TOL, (k, rel_err(got[k], ref[k]))
    sc = dual_scale(ref["F4"], ref["G4"])
    assert rel_err(got["F"][::4], ref["F4"], sc) <= PARITY_TOL
    assert rel_err(got["G"][::4], ref["G4"], sc) <= PARITY_TOL
    assert abs(got["loss"] - float(ref["loss"])) <= PARITY_TOL * abs(float(ref["loss"]))
    assert abs(got["err"] - float(ref["err"])) <= 1e-8 * abs(float(ref["err"]))


def test_full_size_gradient_finite_differences():
    """Central differences (h = 1e-6) of the full-size workload's objective
    ||b - b_ext||^2 (normaliser held at its value, as the reference's backward
    differentiates it) on 20 entries of A and every entry of w."""
    _, A, C, w, be = _bary2048()
    ctrl = {"reg": 0.05, "method": "log", "with_grad": True, "max_iter": 50, "zero_tol": 0.0}
    r = rw.barycenter(A, C, w, be, ctrl)
    Z0 = rw.last_report()["bary_norm"]
    fctrl = dict(ctrl, with_grad=False)

    def obj(A_, w_):
        q = rw.barycenter(A_, C, w_, None, fctrl)
        braw = q["b"] * rw.last_report()["bary_norm"] / Z0
        return float((braw - be) @ (braw - be))

    gw = _fd(lambda x: obj(A, x), w, range(w.size))
    assert np.abs(gw - r["grad_w"]).max() <= 1e-6 * max(1.0, np.abs(gw).max()), np.abs(gw - r["grad_w"]).max()
    g = np.random.default_rng(2)
    idx = [k for k in g.choice(A.size, 200, replace=False) if A.flat[k] > 1e-3][:20]
    gA = _fd(lambda X: obj(X, w), A, idx)
    assert np.abs(gA - r["grad_A"].flat[idx]).max() <= 1e-6 * max(1.0, np.abs(gA).max())
