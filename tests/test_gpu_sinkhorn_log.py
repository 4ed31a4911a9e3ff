"""Parity of the CUDA log-Sinkhorn (rwig_sinkhorn_log*) with the CPU oracle.

Bar: relative error <= 1e-10 (tests.util.PARITY_TOL) on the plan, the dual
potentials and the loss, on identical inputs and an identical iteration count;
and rwig's own known-answer vectors at rwig's own tolerance."""
import ctypes

import numpy as np
import pytest

import oracle
import rwig_b200 as rw
from rwig_b200 import synth
from tests.util import GOLDEN_TOL, PARITY_TOL, dual_scale, mean_rel_diff, rel_err

pytestmark = pytest.mark.gpu


def _compare(a, b, C, reg, max_iter=1000, zero_tol=1e-9, n_threads=8):
    ref = oracle.sinkhorn_log(a, b, C, reg, max_iter=max_iter, zero_tol=zero_tol, n_threads=n_threads)
    got = rw.sinkhorn(a, b, C, {"reg": reg, "method": "log", "max_iter": max_iter, "zero_tol": zero_tol})
    assert got["iter"] == ref["iter"]
    assert got["return_status"] == ref["return_status"]
    assert rel_err(got["P"], ref["P"]) <= PARITY_TOL, rel_err(got["P"], ref["P"])
    sc = dual_scale(ref["f"], ref["g"])
    for k in ("f", "g"):
        assert rel_err(got[k], ref[k], sc) <= PARITY_TOL, (k, rel_err(got[k], ref[k], sc))
    assert abs(got["loss"] - ref["loss"]) <= PARITY_TOL * abs(ref["loss"])
    # the stopping error is a difference of nearly equal quantities; both sides
    # carry rounding of ~1e-13 absolute in it
    assert abs(got["err"] - ref["err"]) <= 1e-6 * abs(ref["err"]) + 1e-12
    return got, ref


def test_golden_vectors(golden):
    g = golden["sinkhorn"]
    a, b, C = np.array(g["inputs"]["a"]), np.array(g["inputs"]["b"]), np.array(g["inputs"]["C"])
    reg = g["inputs"]["reg"]
    r = rw.sinkhorn(a, b, C, {"reg": reg, "method": "log"})
    exp = g["log"]
    for k in ("loss", "P", "f", "g"):
        assert mean_rel_diff(exp[k], r[k]) <= GOLDEN_TOL, k
    _compare(a, b, C, reg, zero_tol=1e-6)


@pytest.mark.parametrize("m,n,reg", [
    (64, 64, 0.05), (100, 37, 0.1), (37, 100, 0.1), (513, 300, 0.05), (1024, 1024, 0.05),
    (2048, 700, 0.02), (4096, 256, 0.05), (8192, 64, 0.1), (1, 5, 0.1), (5, 1, 0.1), (2, 2, 0.5),
])
def test_parity_shapes(m, n, reg):
    a, b, C = synth.sinkhorn_problem(m, n, 0.5, salt=m * 7919 + n)
    _compare(a, b, C, reg)


@pytest.mark.parametrize("iters", [0, 1, 2, 37])
def test_pinned_iterations(iters):
    a, b, C = synth.sinkhorn_problem(300, 200, 1.0, salt=5)
    got, ref = _compare(a, b, C, 0.05, max_iter=iters, zero_tol=0.0)
    assert got["iter"] == iters
    assert got["return_status"] == 1


def test_support_reduction_zero_masses():
    """Zero entries of a and b are dropped (sinkhorn_impl_log.cpp:238-249):
    f, g are -inf there and the plan rows/columns are zero."""
    a, b, C = synth.sinkhorn_problem(120, 90, 1.0, salt=11)
    a[[0, 5, 17, 119]] = 0.0
    b[[3, 4, 89]] = 0.0
    a /= a.sum()
    b /= b.sum()
    got, ref = _compare(a, b, C, 0.05)
    assert np.all(np.isneginf(got["f"][[0, 5, 17, 119]]))
    assert np.all(np.isneginf(got["g"][[3, 4, 89]]))
    assert np.all(got["P"][[0, 5, 17, 119], :] == 0.0)
    rep = rw.last_report()
    assert rep["support_m"] == 116 and rep["support_n"] == 87


def test_odd_leading_dimension():
    a, b, C = synth.sinkhorn_problem(333, 129, 0.5, salt=3)
    _compare(a, b, C, 0.05)


def test_small_eps_uses_safe_row_softmin():
    """eps small enough that some merged row sums of the one-exponential plan
    leave the safe range: the kernel re-runs those sweeps with per-row minima."""
    g = synth.rng(99)
    m, n = 200, 150
    x = g.random((m, 2))
    y = g.random((n, 2)) * 0.3
    C = synth.sq_euclid_cost(x, y)
    a = synth.dirichlet(g, 1.0, m)
    b = synth.dirichlet(g, 1.0, n)
    got, ref = _compare(a, b, C, 2e-3, max_iter=60, zero_tol=0.0)


def test_report_marginals():
    a, b, C = synth.sinkhorn_problem(700, 500, 0.5, salt=1)
    got, ref = _compare(a, b, C, 0.05)
    rep = rw.last_report()
    P = ref["P"]
    assert abs(rep["marg_l1_row"] - np.abs(P.sum(1) - a).sum()) <= 1e-9 * max(1e-12, np.abs(P.sum(1) - a).sum()) + 1e-15
    assert abs(rep["marg_l1_col"] - np.abs(P.sum(0) - b).sum()) <= 1e-12
    assert rep["iter"] == got["iter"] and rep["device_ms"] > 0 and rep["kernel_launches"] >= 2


def test_device_entry_matches_host_entry():
    import torch
    a, b, C = synth.sinkhorn_problem(640, 512, 0.5, salt=2)
    host = rw.sinkhorn(a, b, C, {"reg": 0.05, "method": "log", "zero_tol": 1e-9})
    dev = torch.device("cuda:0")
    ta = torch.from_numpy(a).to(dev)
    tb = torch.from_numpy(b).to(dev)
    tC = torch.from_numpy(np.ascontiguousarray(C.T)).to(dev)  # column-major M x N
    P = torch.empty((512, 640), dtype=torch.float64, device=dev)
    f = torch.empty(640, dtype=torch.float64, device=dev)
    gg = torch.empty(512, dtype=torch.float64, device=dev)
    st = torch.cuda.Stream()
    r = rw.sinkhorn_log_device(ta, tb, tC, 0.05, 1000, 1e-9, P=P, f=f, g=gg, stream=st)
    torch.cuda.synchronize()
    assert r["iter"] == host["iter"]
    assert np.array_equal(P.cpu().numpy().T, host["P"])
    assert np.array_equal(f.cpu().numpy(), host["f"])
    assert np.array_equal(gg.cpu().numpy(), host["g"])


def test_invalid_arguments_raise():
    with pytest.raises(rw.RwigError):
        rw.sinkhorn(np.zeros(3), np.ones(2) / 2, np.ones((3, 2)), {"method": "log"})
    with pytest.raises(rw.RwigError):
        rw.sinkhorn(np.ones(3) / 3, np.ones(2) / 2, np.ones((3, 2)), {"method": "log", "reg": -1.0})


def test_repeatable_bitwise():
    a, b, C = synth.sinkhorn_problem(1500, 1100, 0.5, salt=8)
    r1 = rw.sinkhorn(a, b, C, {"reg": 0.03, "method": "log", "zero_tol": 1e-9})
    r2 = rw.sinkhorn(a, b, C, {"reg": 0.03, "method": "log", "zero_tol": 1e-9})
    for k in ("P", "f", "g"):
        assert np.array_equal(r1[k], r2[k])
    assert r1["loss"] == r2["loss"] and r1["iter"] == r2["iter"]


@pytest.fixture
def engine_option():
    """Sets engine options for one test and restores the defaults."""
    L = rw.load()
    set_opts = []

    def _set(name, value):
        assert L.rwig_set_option(name.encode(), float(value)) == 0
        set_opts.append(name)

    yield _set
    L.rwig_set_option(b"log_sinkhorn.scaled", 1.0)
    L.rwig_set_option(b"log_sinkhorn.tau", 100.0)


@pytest.mark.parametrize("m,n,reg", [(700, 500, 0.02), (4096, 300, 0.01), (129, 1000, 0.05)])
def test_log_domain_only_mode(engine_option, m, n, reg):
    """Every iteration in the log domain (no scaled form): same parity bar."""
    engine_option("log_sinkhorn.scaled", 0)
    a, b, C = synth.sinkhorn_problem(m, n, 0.5, salt=m + 3 * n)
    _compare(a, b, C, reg)


@pytest.mark.parametrize("tau", [0.5, 5.0])
def test_frequent_absorption(engine_option, tau):
    """A small absorption bound rebuilds the scaled kernel many times; the
    results must not move."""
    engine_option("log_sinkhorn.tau", tau)
    a, b, C = synth.sinkhorn_problem(900, 700, 0.5, salt=17)
    got, ref = _compare(a, b, C, 0.01)
    if tau < 1.0:
        assert rw.last_report()["kernel_launches"] > 6  # more than one absorption


def test_unknown_option_rejected():
    assert rw.load().rwig_set_option(b"no.such.option", 1.0) == -1


def test_benchmark_workload_iterations():
    """The 4096 x 4096 log workload converges in the iteration count the CPU
    reference arm of bench.py extrapolates to (the CPU port's own full solve of
    it takes ~30 s, so the count is recorded there)."""
    import bench
    wl = bench.WORKLOADS["log4096"]
    a, b, C = wl.inputs()
    r = rw.sinkhorn(a, b, C, {"reg": wl.reg, "method": "log", "max_iter": wl.max_iter, "zero_tol": wl.tol})
    assert r["iter"] == wl.reference_iters()


def test_full_size_against_oracle_fixture():
    """The 4096 x 4096 benchmark solve against the CPU oracle's full solve
    (tests/golden/log4096_oracle.npz, made by tests/golden/make_log4096.py)."""
    import os
    ref = np.load(os.path.join(os.path.dirname(__file__), "golden", "log4096_oracle.npz"))
    a, b, C = synth.log_config(4096, 4096)
    got = rw.sinkhorn(a, b, C, {"reg": 0.01, "method": "log", "max_iter": 2000, "zero_tol": 1e-9})
    assert got["iter"] == int(ref["iter"]) and got["return_status"] == int(ref["return_status"])
    sc = dual_scale(ref["f"], ref["g"])
    assert rel_err(got["f"], ref["f"], sc) <= PARITY_TOL
    assert rel_err(got["g"], ref["g"], sc) <= PARITY_TOL
    assert abs(got["loss"] - float(ref["loss"])) <= PARITY_TOL * abs(float(ref["loss"]))
