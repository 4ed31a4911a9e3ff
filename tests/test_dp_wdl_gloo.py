"""Data-parallel WDL gradient (rwig_b200.wdl_batch_grad_dp) on two CPU ranks
over gloo: each rank's shard gradient comes from the CPU oracle (the test
injects it as grad_fn), and the all-reduced result must equal the oracle's
gradient of the whole batch -- the sharding and the weighting of the shard
means are what is checked.  Uneven shards (D odd) and a rank with an empty
shard are covered."""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

import oracle
from rwig_b200 import synth


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _oracle_grad(A, WB, YB, C, reg, L, mode):
    K = np.exp(-np.asarray(C) / reg)  # mode 1: the cost is given; the Gibbs kernel exp(-C / reg)
    return oracle.wdl_batch_grad(A, WB, YB, K, L)


def _inputs(D):
    Y, C, A0, L0 = synth.wdl_config(V=40, M=D, S=3, dim=4, salt=5)
    A = np.exp(A0) / np.exp(A0).sum(0)
    W = np.exp(L0) / np.exp(L0).sum(0)
    return A, W, Y, C


def _worker(rank, world, port, D, q):
    import torch.distributed as dist
    import rwig_b200 as rw
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        A, W, Y, C = _inputs(D)
        gA, gl = rw.wdl_batch_grad_dp(A, W, Y, C, reg=0.1, L=6, mode=1, grad_fn=_oracle_grad)
        q.put((rank, gA, gl))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,D", [(2, 7), (2, 8), (3, 2)])
def test_dp_gradient_equals_whole_batch(world, D):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, D, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    A, W, Y, C = _inputs(D)
    rA, rl = _oracle_grad(A, W, Y, C, 0.1, 6, 1)
    for rank, gA, gl in got:
        assert np.abs(gA - rA).max() <= 1e-13 * np.abs(rA).max(), rank
        assert np.abs(gl - rl).max() <= 1e-13 * max(np.abs(rl).max(), 1e-300), rank
    # every rank holds the same bits (one all-reduce)
    assert all(np.array_equal(got[0][1], g[1]) and np.array_equal(got[0][2], g[2]) for g in got)
