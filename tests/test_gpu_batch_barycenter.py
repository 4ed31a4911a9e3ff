"""Many barycenter problems in one call (rwig_batch_barycenter_dev): uneven
M, N, S, both methods, with and without gradients, fixed iteration counts run
side by side and stopping tests one after another; every result bitwise
equal to the single call's on the same problem (rwig_barycenter_*), an
invalid problem rejected alone, and results against the CPU oracle
(Barycenter::compute_parallel / compute_log restated)."""
import numpy as np
import pytest

import oracle
import rwig_b200 as rw
from rwig_b200 import synth
from tests.util import PARITY_TOL, rel_err

pytestmark = pytest.mark.gpu

CASES = [  # M, N, S, method, with_grad, max_iter, zero_tol
    (2048, 2048, 32, "log", True, 20, 0.0),
    (500, 300, 8, "parallel", True, 15, 0.0),
    (300, 500, 5, "log", False, 25, 0.0),
    (1000, 1000, 64, "parallel", False, 10, 0.0),
    (128, 64, 3, "log", True, 30, 1e-6),
    (64, 64, 1, "parallel", True, 0, 0.0),
    (700, 900, 16, "log", True, 12, 0.0),
    (257, 129, 40, "parallel", True, 8, 0.0),
]


def _problem(i, M, N, S, method, wg, L, tol):
    g = synth.rng(synth.SEED_X, 700 + i)
    x, y = g.random((M, 3)), g.random((N, 3))
    C = synth.sq_euclid_cost(x, y)
    A = synth.dirichlet(g, 1.0, M, S)
    w = synth.dirichlet(g, 1.0, S)
    be = synth.dirichlet(g, 1.0, N)
    return {"A": A, "C": C, "w": w, "b_ext": be if wg else None, "reg": 0.1, "method": method, "with_grad": wg,
            "max_iter": L, "zero_tol": tol}


def _single(q):
    ctrl = {k: q[k] for k in ("reg", "method", "with_grad", "max_iter", "zero_tol")}
    return rw.barycenter(q["A"], q["C"], q["w"], q["b_ext"], ctrl)


def test_batch_equals_single_calls():
    probs = [_problem(i, *c) for i, c in enumerate(CASES)]
    got = rw.batch_barycenter(probs)
    for i, q in enumerate(probs):
        ref = _single(q)
        keys = ["b", "F", "G"] if q["method"] == "log" else ["b", "U", "V"]
        if q["with_grad"]:
            keys += ["grad_A", "grad_w"]
        for k in keys:
            assert np.array_equal(got[i][k], ref[k], equal_nan=True), (i, k)
        assert got[i]["iter"] == ref["iter"] and got[i]["return_status"] == ref["return_status"], i
        assert got[i]["err"] == ref["err"] or (np.isnan(got[i]["err"]) and np.isnan(ref["err"])), i
        if q["with_grad"]:
            assert got[i]["loss"] == ref["loss"] or (np.isnan(got[i]["loss"]) and np.isnan(ref["loss"])), i
        if q["with_grad"] and q["max_iter"] == 0:  # nothing unrolled: zero gradient
            assert not got[i]["grad_A"].any() and not got[i]["grad_w"].any()


def test_batch_against_oracle():
    probs = [_problem(i, *c) for i, c in enumerate(CASES) if c[0] <= 1000 and c[5] > 0]
    got = rw.batch_barycenter(probs)
    for q, r in zip(probs, got):
        fn = oracle.barycenter_log if q["method"] == "log" else oracle.barycenter_parallel
        ref = fn(q["A"], q["C"], q["w"], q["b_ext"], q["reg"], with_grad=q["with_grad"], max_iter=q["max_iter"],
                 zero_tol=q["zero_tol"])
        assert r["iter"] == ref["iter"]
        assert rel_err(r["b"], ref["b"]) <= PARITY_TOL, rel_err(r["b"], ref["b"])
        if q["with_grad"]:
            assert rel_err(r["grad_A"], ref["grad_A"]) <= PARITY_TOL
            assert rel_err(r["grad_w"], ref["grad_w"]) <= PARITY_TOL


def test_invalid_problem_rejected_alone():
    probs = [_problem(0, 300, 200, 4, "log", True, 10, 0.0), _problem(1, 100, 80, 65, "parallel", False, 5, 0.0),
             _problem(2, 200, 300, 6, "parallel", True, 10, 0.0)]
    got = rw.batch_barycenter(probs)
    assert got[1]["return_status"] < 0
    for i in (0, 2):
        ref = _single(probs[i])
        assert np.array_equal(got[i]["b"], ref["b"]) and np.array_equal(got[i]["grad_A"], ref["grad_A"])


def test_more_problems_than_side_streams_growing():
    """Twelve problems on eight side streams, the later ones larger: the
    problems sharing a stream share its slot set, grown to the largest of
    them before anything is enqueued; every result equals the single call's."""
    cases = [(100 + 40 * i, 80 + 30 * i, 2 + i % 5, "log" if i % 2 else "parallel", i % 3 != 0, 6 + i, 0.0)
             for i in range(12)]
    probs = [_problem(20 + i, *c) for i, c in enumerate(cases)]
    got = rw.batch_barycenter(probs)
    for i, q in enumerate(probs):
        ref = _single(q)
        keys = ["b"] + (["grad_A", "grad_w"] if q["with_grad"] else [])
        for k in keys:
            assert np.array_equal(got[i][k], ref[k]), (i, k)
        assert got[i]["iter"] == ref["iter"], i
