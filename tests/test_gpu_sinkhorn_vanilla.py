"""Parity of the CUDA vanilla Sinkhorn (rwig_sinkhorn_vanilla*) with the CPU
oracle (Sinkhorn::compute_vanilla restated) and rwig's known-answer vectors."""
import numpy as np
import pytest

import oracle
import rwig_b200 as rw
from rwig_b200 import synth
from tests.util import GOLDEN_TOL, PARITY_TOL, mean_rel_diff, rel_err

pytestmark = pytest.mark.gpu


def _compare(a, b, C, reg, max_iter=1000, zero_tol=1e-9):
    ref = oracle.sinkhorn_vanilla(a, b, C, reg, max_iter=max_iter, zero_tol=zero_tol)
    got = rw.sinkhorn(a, b, C, {"reg": reg, "method": "vanilla", "max_iter": max_iter, "zero_tol": zero_tol})
    assert got["iter"] == ref["iter"]
    assert got["return_status"] == ref["return_status"]
    for k in ("P", "u", "v"):
        assert rel_err(got[k], ref[k]) <= PARITY_TOL, (k, rel_err(got[k], ref[k]))
    assert abs(got["loss"] - ref["loss"]) <= PARITY_TOL * abs(ref["loss"])
    assert abs(got["err"] - ref["err"]) <= 1e-6 * abs(ref["err"]) + 1e-13
    return got, ref


def test_golden_vectors(golden):
    g = golden["sinkhorn"]
    a, b, C = np.array(g["inputs"]["a"]), np.array(g["inputs"]["b"]), np.array(g["inputs"]["C"])
    r = rw.sinkhorn(a, b, C, {"reg": g["inputs"]["reg"], "method": "vanilla"})
    for k in ("loss", "P", "u", "v"):
        assert mean_rel_diff(g["vanilla"][k], r[k]) <= GOLDEN_TOL, k
    _compare(a, b, C, g["inputs"]["reg"], zero_tol=1e-6)


@pytest.mark.parametrize("m,n,reg", [
    (256, 256, 0.1), (100, 37, 0.2), (37, 100, 0.2), (513, 300, 0.1), (2048, 700, 0.1),
    (4096, 256, 0.1), (1, 5, 0.1), (5, 1, 0.1), (2, 2, 0.5),
])
def test_parity_shapes(m, n, reg):
    a, b, C = synth.sinkhorn_problem(m, n, 1.0, salt=m * 31 + n)
    _compare(a, b, C, reg)


def test_benchmark_workload():
    a, b, C = synth.vanilla_config()
    got, ref = _compare(a, b, C, 0.1)
    assert got["return_status"] == 0


@pytest.mark.parametrize("iters", [0, 1, 2, 15])
def test_pinned_iterations(iters):
    a, b, C = synth.sinkhorn_problem(300, 200, 1.0, salt=5)
    got, ref = _compare(a, b, C, 0.1, max_iter=iters, zero_tol=0.0)
    assert got["iter"] == iters


def test_support_reduction_zero_masses():
    a, b, C = synth.sinkhorn_problem(120, 90, 1.0, salt=11)
    a[[0, 5, 119]] = 0.0
    b[[3, 89]] = 0.0
    a /= a.sum()
    b /= b.sum()
    got, ref = _compare(a, b, C, 0.1)
    assert np.all(got["u"][[0, 5, 119]] == 0.0) and np.all(got["v"][[3, 89]] == 0.0)
    assert np.all(got["P"][[0, 5, 119], :] == 0.0) and np.all(got["P"][:, [3, 89]] == 0.0)


def test_device_entry_matches_host_entry():
    import torch
    a, b, C = synth.vanilla_config()
    host = rw.sinkhorn(a, b, C, {"reg": 0.1, "method": "vanilla", "zero_tol": 1e-9})
    d = torch.device("cuda:0")
    P = torch.empty((256, 256), dtype=torch.float64, device=d)
    u = torch.empty(256, dtype=torch.float64, device=d)
    v = torch.empty(256, dtype=torch.float64, device=d)
    r = rw.sinkhorn_vanilla_device(torch.from_numpy(a).to(d), torch.from_numpy(b).to(d),
                                   torch.from_numpy(np.ascontiguousarray(C.T)).to(d), 0.1, 1000, 1e-9,
                                   P=P, u=u, v=v)
    assert r["iter"] == host["iter"]
    assert np.array_equal(P.cpu().numpy().T, host["P"])
    assert np.array_equal(u.cpu().numpy(), host["u"]) and np.array_equal(v.cpu().numpy(), host["v"])


def _outlier_problem(m, n, seed, far):
    """Sources and targets in [0, 0.1]^2 except `far` targets near (1, 1):
    with the cost normalised by its maximum, K^T u at those targets is about
    exp(-1/eps) times the other column sums."""
    g = np.random.default_rng(seed)
    x = g.random((m, 2)) * 0.1
    y = g.random((n, 2)) * 0.1
    y[:far] = 1.0 - 0.01 * g.random((far, 2))
    C = synth.sq_euclid_cost(x, y)
    a = g.gamma(1.0, size=m)
    b = g.gamma(1.0, size=n)
    return a / a.sum(), b / b.sum(), C


@pytest.mark.parametrize("m,n,reg,seed,far", [(256, 256, 0.01, 1, 1), (300, 200, 0.01, 4, 4),
                                              (256, 256, 0.012, 3, 2)])
def test_column_sums_below_float_range(m, n, reg, seed, far):
    """Column sums K^T u far below FLT_MIN (1e-40 at eps = 0.01): v = b / K^T u
    must be the IEEE quotient, as sinkhorn_impl_vanilla.cpp:133 computes it."""
    a, b, C = _outlier_problem(m, n, seed, far)
    got, ref = _compare(a, b, C, reg, max_iter=2000)
    ktu = b / ref["v"]
    if reg == 0.01:
        assert ktu.min() < 1e-38
    assert np.isfinite(got["P"]).all() and np.isfinite(got["v"]).all()
