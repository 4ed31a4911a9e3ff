"""Batched log-Sinkhorn (rwig_batch_sinkhorn_log): every problem of a mixed-size
batch against the CPU oracle (Sinkhorn::compute_log restated) at the parity
tolerance, each result the same alone and in the mix, and the routing of
problems the one-CTA kernel does not take."""
import numpy as np
import pytest

import oracle
import rwig_b200 as rw
from rwig_b200 import synth
from tests.util import PARITY_TOL, dual_scale, rel_err

pytestmark = pytest.mark.gpu


def _problem(m, n, reg, dim=2, salt=0, max_iter=2000, tol=1e-9):
    a, b, C = synth.sinkhorn_problem(m, n, 1.0, dim=dim, salt=salt)
    return {"a": a, "b": b, "C": C, "reg": reg, "max_iter": max_iter, "zero_tol": tol}


def _check(q, got):
    ref = oracle.sinkhorn_log(q["a"], q["b"], q["C"], q["reg"], max_iter=q["max_iter"], zero_tol=q["zero_tol"],
                              n_threads=8)
    assert got["iter"] == ref["iter"], (got["iter"], ref["iter"])
    assert got["return_status"] == ref["return_status"]
    sc = dual_scale(ref["f"], ref["g"])
    for k in ("f", "g"):
        assert rel_err(got[k], ref[k], sc) <= PARITY_TOL, (k, rel_err(got[k], ref[k], sc))
    if "P" in got:
        assert rel_err(got["P"], ref["P"]) <= PARITY_TOL, rel_err(got["P"], ref["P"])
    assert abs(got["loss"] - ref["loss"]) <= PARITY_TOL * abs(ref["loss"])
    assert abs(got["err"] - ref["err"]) <= 1e-6 * abs(ref["err"]) + 1e-12


MIX = [(64, 64, 0.05, 2), (100, 37, 0.1, 3), (37, 100, 0.1, 64), (513, 300, 0.05, 2), (700, 1500, 0.01, 3),
       (1024, 1024, 0.05, 2), (2048, 700, 0.1, 64), (3000, 257, 0.05, 2), (5000, 90, 0.1, 3), (8192, 64, 0.1, 2),
       (1, 5, 0.1, 2), (5, 1, 0.1, 2), (2, 2, 0.5, 2)]


def test_mixed_batch_matches_oracle():
    probs = [_problem(m, n, reg, dim, salt=i + 1) for i, (m, n, reg, dim) in enumerate(MIX)]
    out = rw.batch_sinkhorn_log(probs, with_plan=True)
    assert all(o["path"] == 0 for o in out), [o["path"] for o in out]
    for q, o in zip(probs, out):
        _check(q, o)


def test_alone_equals_in_mix():
    """A problem's result is bitwise the same alone and inside a batch."""
    probs = [_problem(m, n, reg, dim, salt=i + 1) for i, (m, n, reg, dim) in enumerate(MIX)]
    mix = rw.batch_sinkhorn_log(probs)
    for i in (0, 4, 7, 9):
        alone = rw.batch_sinkhorn_log([probs[i]])[0]
        for k in ("f", "g"):
            assert np.array_equal(alone[k], mix[i][k]), (i, k)
        assert alone["loss"] == mix[i]["loss"] and alone["iter"] == mix[i]["iter"] and alone["err"] == mix[i]["err"]


def test_routing_and_rejection():
    """Zero masses and max_iter = 0 go through the per-call path; an invalid
    problem is rejected alone; all results still match the oracle."""
    z = _problem(300, 200, 0.05, salt=11)
    z["a"] = z["a"].copy()
    z["a"][[3, 17]] = 0.0
    z["a"] /= z["a"].sum()
    none = _problem(50, 60, 0.1, salt=12, max_iter=0)
    ok = _problem(400, 500, 0.05, salt=13)
    bad = {"a": np.ones(3) / 3, "b": np.ones(4) / 4, "C": np.ones((3, 4)), "reg": -1.0}
    out = rw.batch_sinkhorn_log([z, none, bad, ok])
    assert [o["path"] for o in (out[0], out[1], out[3])] == [1, 1, 0]
    assert out[2]["return_status"] < 0
    for q, o in ((z, out[0]), (none, out[1]), (ok, out[3])):
        _check(q, o)


def test_marginals_reported():
    q = _problem(600, 450, 0.05, salt=21)
    o = rw.batch_sinkhorn_log([q], with_plan=True)[0]
    P = o["P"]
    assert abs(o["marg_l1_row"] - np.abs(P.sum(1) - q["a"]).sum()) <= 1e-12
    assert abs(o["marg_l1_col"] - np.abs(P.sum(0) - q["b"]).sum()) <= 1e-12


def test_batch_equals_per_call_path():
    """The batched result agrees with the per-call rwig_sinkhorn_log to the
    parity tolerance (the two sum in different orders)."""
    q = _problem(1500, 1200, 0.05, salt=31)
    o = rw.batch_sinkhorn_log([q])[0]
    r = rw.sinkhorn(q["a"], q["b"], q["C"], {"reg": 0.05, "method": "log", "max_iter": 2000, "zero_tol": 1e-9})
    assert o["iter"] == r["iter"]
    sc = dual_scale(r["f"], r["g"])
    assert rel_err(o["f"], r["f"], sc) <= PARITY_TOL and rel_err(o["g"], r["g"], sc) <= PARITY_TOL


def test_streamed_8192_against_oracle_fixture():
    """One 8192 x 8192 request of the serving stream's kind through the batched
    kernel, where its K (512 MB) is streamed from memory in strips every
    iteration (it cannot stay in the shared memory of a team), alone and
    beside small problems, against the CPU oracle's full solve
    (tests/golden/sink8192_oracle.npz, made by tests/golden/make_fullsize.py)."""
    import os
    ref = np.load(os.path.join(os.path.dirname(__file__), "golden", "sink8192_oracle.npz"))
    a, b, x, y = synth.stream_request_data(8192, 8192, 3, 777)
    C = synth.sq_euclid_cost(x, y)
    big = {"a": a, "b": b, "C": C, "reg": 0.05, "max_iter": 2000, "zero_tol": 1e-9}
    alone = rw.batch_sinkhorn_log([big])[0]
    mixed = rw.batch_sinkhorn_log([_problem(300, 200, 0.05, salt=1), big, _problem(64, 900, 0.1, salt=2)])[1]
    for got in (alone, mixed):
        assert got["path"] == 0
        assert got["iter"] == int(ref["iter"]) and got["return_status"] == int(ref["return_status"])
        sc = dual_scale(ref["f"], ref["g"])
        assert rel_err(got["f"], ref["f"], sc) <= PARITY_TOL, rel_err(got["f"], ref["f"], sc)
        assert rel_err(got["g"], ref["g"], sc) <= PARITY_TOL, rel_err(got["g"], ref["g"], sc)
        assert abs(got["loss"] - float(ref["loss"])) <= PARITY_TOL * abs(float(ref["loss"]))
    assert np.array_equal(alone["f"], mixed["f"]) and np.array_equal(alone["g"], mixed["g"])
