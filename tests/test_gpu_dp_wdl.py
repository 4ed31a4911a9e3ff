"""Data-parallel WDL gradient through the engine.

* One rank: the all-reduced gradient (host and device entries) equals the
  engine's direct wdl_batch_grad of the batch, up to the rounding of the
  shard weighting.
* Two ranks: two gloo processes on the one GPU, each computing its shard with
  the engine's device entry (rwig_wdl_batch_grad_dev) and all-reducing the
  device buffer; both ranks hold the whole batch's gradient.  The engine's
  kernels never wait on another process, so sharing the GPU is safe."""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

import rwig_b200 as rw
from rwig_b200 import synth

pytestmark = pytest.mark.gpu


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _inputs(D=24):
    Y, C, A0, L0 = synth.wdl_config(V=300, M=D, S=4, dim=8, salt=9)
    A = np.exp(A0) / np.exp(A0).sum(0)
    W = np.exp(L0) / np.exp(L0).sum(0)
    return A, W, Y, C


def _dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(np.asarray(x).T)).to("cuda:0")


def test_one_rank_equals_direct_gradient():
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_port()))
    A, W, Y, C = _inputs()
    dist.init_process_group("gloo", rank=0, world_size=1)
    try:
        gA, gl = rw.wdl_batch_grad_dp(A, W, Y, C, reg=0.05, L=10, mode=1)
        dA, dl = rw.wdl_batch_grad_dp_dev(_dev(A), _dev(W), _dev(Y), _dev(C), reg=0.05, L=10, mode=1)
        dA, dl = dA.cpu().numpy().T, dl.cpu().numpy()
    finally:
        dist.destroy_process_group()
    rA, rl = rw.wdl_batch_grad(A, W, Y, C, reg=0.05, L=10, mode=1)
    for x, y in ((gA, rA), (dA, rA), (gl, rl), (dl, rl)):
        assert np.abs(x - y).max() <= 1e-14 * np.abs(y).max()


def _worker(rank, world, port, D, q):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        A, W, Y, C = _inputs(D)
        K = np.exp(-C / 0.05)
        gA, gl = rw.wdl_batch_grad_dp_dev(_dev(A), _dev(W), _dev(Y), _dev(K), reg=0.05, L=10, mode=0)
        q.put((rank, gA.cpu().numpy().T.copy(), gl.cpu().numpy().copy()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("D", [24, 7])
def test_two_ranks_on_device_buffers(D):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, D, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=300) for _ in range(2)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    A, W, Y, C = _inputs(D)
    rA, rl = rw.wdl_batch_grad(A, W, Y, np.exp(-C / 0.05), reg=0.05, L=10, mode=0)
    for rank, gA, gl in got:
        assert np.abs(gA - rA).max() <= 1e-13 * np.abs(rA).max(), rank
        assert np.abs(gl - rl).max() <= 1e-13 * np.abs(rl).max(), rank
    assert np.array_equal(got[0][1], got[1][1]) and np.array_equal(got[0][2], got[1][2])


def _train_inputs():
    Y, C, A0, L0 = synth.wdl_config(V=250, M=20, S=4, dim=6, salt=31)
    return Y, C, A0, L0


_TRAIN = dict(reg=0.05, L=8, B=8, E=2, eta=5e-3)


def _train_worker(rank, world, port, opt, q):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        Y, C, A0, L0 = _train_inputs()
        out = rw.wdl_train_dp_dev(Y, C, 4, optimizer=opt, Alpha0=A0, Lambda0=L0, **_TRAIN)
        q.put((rank, out["A"], out["W"], out["steps"]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("opt", [0, 1, 2])
def test_data_parallel_training_matches_one_gpu(opt):
    """Two ranks train with each batch's documents split between them (the
    gradient all-reduced on the device, the optimizer step and softmaxes on
    the device by rwig_wdl_update_dev on both): both end with the same
    parameters, equal to rwig_wdl's one-GPU training from the same logits up
    to the rounding of the shard weighting (SGD, Adam, AdamW; a last batch of
    4 documents, so a rank's shard is 2 or 4)."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    procs = [ctx.Process(target=_train_worker, args=(r, 2, port, opt, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=300) for _ in range(2)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    Y, C, A0, L0 = _train_inputs()
    ref = rw.wdl_cpp(Y, C, _TRAIN["reg"], 4, _TRAIN["B"], _TRAIN["E"], max_iter=_TRAIN["L"], zero_tol=1e-6,
                     optimizer=opt, eta=_TRAIN["eta"], Alpha0=A0, Lambda0=L0)
    assert np.array_equal(got[0][1], got[1][1]) and np.array_equal(got[0][2], got[1][2])
    assert got[0][3] == 2 * 3
    for _, A, W, _ in got:
        assert np.abs(A - ref["A"]).max() <= 1e-11 * np.abs(ref["A"]).max()
        assert np.abs(W - ref["W"]).max() <= 1e-11 * np.abs(ref["W"]).max()
