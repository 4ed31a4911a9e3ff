"""Continuous-batching server (rwig_server_*): requests admitted while others
run give the same bits as the same requests solved alone, agree with the
batched call and with the CPU oracle, and the server applies its memory
budget and restarts after going idle."""
import time

import numpy as np
import pytest

import oracle
import rwig_b200 as rw
from rwig_b200 import synth
from tests.util import PARITY_TOL, dual_scale, rel_err

pytestmark = pytest.mark.gpu

SIZES = [(64, 64, 0.05, 2), (300, 200, 0.1, 3), (700, 1500, 0.01, 3), (1024, 1024, 0.05, 2), (2048, 700, 0.1, 64),
         (5000, 90, 0.1, 3), (37, 100, 0.1, 64), (1500, 1200, 0.05, 2)]


def _prob(i, m, n, reg, dim):
    a, b, C = synth.sinkhorn_problem(m, n, 1.0, dim=dim, salt=500 + i)
    return {"a": a, "b": b, "C": C, "reg": reg, "max_iter": 2000, "zero_tol": 1e-9}


def _wait(server, tickets, timeout=60.0):
    out, t0 = {}, time.time()
    while len(out) < len(tickets):
        for t in tickets:
            if t not in out:
                r = server.poll(t)
                if r is not None:
                    out[t] = r
        assert time.time() - t0 < timeout, "server did not finish"
    return [out[t] for t in tickets]


class _SameTeams:
    """Sets batch.max_team for the block: a server's and a batched call's
    default team limits differ, and their results are bitwise equal under the
    same limit."""

    def __enter__(self):
        import torch
        from rwig_b200 import _lib
        sm = torch.cuda.get_device_properties(0).multi_processor_count
        assert _lib.load().rwig_set_option(b"batch.max_team", float(int(0.4 * sm))) == 0

    def __exit__(self, *exc):
        from rwig_b200 import _lib
        _lib.load().rwig_set_option(b"batch.max_team", float("nan"))


def _submit(server, q):
    while True:
        t = server.submit(q["a"], q["b"], q["C"], q["reg"], q["max_iter"], q["zero_tol"])
        if t is not None:
            return t
        time.sleep(0.001)


def test_in_mix_equals_alone_and_oracle():
    probs = [_prob(i, *s) for i, s in enumerate(SIZES)]
    with _SameTeams(), rw.Server(idle_ms=5.0) as srv:
        alone = []
        for q in probs:  # one at a time
            alone.append(_wait(srv, [_submit(srv, q)])[0])
        # staggered: half now, the rest while the first half runs
        first = [_submit(srv, q) for q in probs[::2]]
        time.sleep(0.002)
        second = [_submit(srv, q) for q in probs[1::2]]
        mix = _wait(srv, first + second)
    order = list(range(0, len(probs), 2)) + list(range(1, len(probs), 2))
    for k, i in enumerate(order):
        for key in ("f", "g"):
            assert np.array_equal(mix[k][key], alone[i][key]), (i, key)
        assert mix[k]["loss"] == alone[i]["loss"] and mix[k]["iter"] == alone[i]["iter"]
    with _SameTeams():
        batch = rw.batch_sinkhorn_log(probs)
    for i, q in enumerate(probs):
        assert np.array_equal(batch[i]["f"], alone[i]["f"]) and batch[i]["iter"] == alone[i]["iter"]
    for i in (0, 2, 5):
        q = probs[i]
        ref = oracle.sinkhorn_log(q["a"], q["b"], q["C"], q["reg"], max_iter=q["max_iter"], zero_tol=q["zero_tol"],
                                  n_threads=8, want_P=False)
        assert alone[i]["iter"] == ref["iter"]
        sc = dual_scale(ref["f"], ref["g"])
        assert rel_err(alone[i]["f"], ref["f"], sc) <= PARITY_TOL and rel_err(alone[i]["g"], ref["g"], sc) <= PARITY_TOL
        assert abs(alone[i]["loss"] - ref["loss"]) <= PARITY_TOL * abs(ref["loss"])


def test_memory_budget_and_idle_restart():
    q = _prob(0, 400, 300, 0.05, 2)
    big = _prob(1, 1500, 1500, 0.05, 2)
    with rw.Server(mem_budget_bytes=12e6, idle_ms=1.0) as srv:  # holds the small one (~1 MB), not the big one (~19 MB)
        t1 = srv.submit(q["a"], q["b"], q["C"], q["reg"], 2000, 1e-9)
        assert t1 is not None
        assert srv.submit(big["a"], big["b"], big["C"], big["reg"], 2000, 1e-9) is None  # over the budget
        r1 = _wait(srv, [t1])[0]
        time.sleep(0.05)  # the kernel goes idle and ends
        t2 = _submit(srv, q)
        r2 = _wait(srv, [t2])[0]
    assert np.array_equal(r1["f"], r2["f"]) and r1["iter"] == r2["iter"]


def test_cost_from_points_matches_host_cost():
    """Requests given as point clouds (cost built on the device) give the same
    bits as the same requests given the host-built cost matrix."""
    cases = [(300, 200, 0.05, 2), (1000, 700, 0.01, 64), (64, 3000, 0.1, 3)]
    with_c, with_pts = [], []
    for i, (m, n, reg, dim) in enumerate(cases):
        x = synth.rng(synth.SEED_X, 900 + i).random((m, dim))
        y = synth.rng(synth.SEED_Y, 900 + i).random((n, dim))
        a = synth.dirichlet(synth.rng(synth.SEED_A, 900 + i), 1.0, m)
        b = synth.dirichlet(synth.rng(synth.SEED_B, 900 + i), 1.0, n)
        with_c.append({"a": a, "b": b, "C": synth.sq_euclid_cost(x, y), "reg": reg, "max_iter": 2000,
                       "zero_tol": 1e-9})
        with_pts.append({"a": a, "b": b, "x": x, "y": y, "reg": reg, "max_iter": 2000, "zero_tol": 1e-9})
    with _SameTeams():
        rc = rw.batch_sinkhorn_log(with_c, with_plan=True)
        rp = rw.batch_sinkhorn_log(with_pts, with_plan=True)
    for u, v in zip(rc, rp):
        for k in ("f", "g", "P"):
            assert np.array_equal(u[k], v[k]), k
        assert u["loss"] == v["loss"] and u["iter"] == v["iter"]
    with _SameTeams(), rw.Server(idle_ms=2.0) as srv:
        tickets = [srv.submit(q["a"], q["b"], None, q["reg"], 2000, 1e-9, x=q["x"], y=q["y"]) for q in with_pts]
        got = _wait(srv, tickets)
    for u, v in zip(rc, got):
        assert np.array_equal(u["f"], v["f"]) and u["iter"] == v["iter"]


def test_slot_reuse_over_many_requests():
    """More requests than descriptor slots (512): request h lives in slot
    h % 512, reused once its previous request has been collected, without the
    launch draining.  1300 requests cycling over 8 problems, submitted as the
    window of outstanding tickets allows, with a pause longer than idle_ms in
    the middle (the launch ends and the next one starts its scan at the first
    unfinished request); every result bitwise equals the batched call's."""
    small = [(64, 64, 0.1, 2), (100, 37, 0.1, 3), (37, 100, 0.1, 64), (200, 150, 0.05, 2), (128, 300, 0.1, 3),
             (90, 90, 0.05, 2), (300, 64, 0.1, 2), (150, 200, 0.1, 3)]
    probs = [_prob(100 + i, *s) for i, s in enumerate(small)]
    with _SameTeams():
        ref = rw.batch_sinkhorn_log(probs)
    n_req, window = 1300, 700
    got = {}
    with _SameTeams(), rw.Server(idle_ms=2.0) as srv:
        pending = {}
        nxt, t0 = 0, time.time()
        while len(got) < n_req:
            while nxt < n_req and len(pending) < window:
                q = probs[nxt % len(probs)]
                t = srv.submit(q["a"], q["b"], q["C"], q["reg"], q["max_iter"], q["zero_tol"])
                if t is None:
                    break
                assert t == nxt  # tickets are request numbers
                pending[t] = nxt
                nxt += 1
                if nxt == 650:
                    time.sleep(0.05)  # > idle_ms: the launch may end while requests are out
            for t in list(pending):
                r = srv.poll(t)
                if r is not None:
                    got[pending.pop(t)] = r
            assert time.time() - t0 < 120.0, "server did not finish"
    for h in range(n_req):
        e = ref[h % len(probs)]
        assert np.array_equal(got[h]["f"], e["f"]) and np.array_equal(got[h]["g"], e["g"]), h
        assert got[h]["iter"] == e["iter"] and got[h]["loss"] == e["loss"], h
