"""Data-parallel WDL gradient through the engine: in a one-rank group the
all-reduced gradient equals the engine's direct wdl_batch_grad of the batch
(up to the rounding of the shard weighting)."""
import os
import socket

import numpy as np
import pytest

import rwig_b200 as rw
from rwig_b200 import synth

pytestmark = pytest.mark.gpu


def test_one_rank_equals_direct_gradient():
    import torch.distributed as dist
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    Y, C, A0, L0 = synth.wdl_config(V=300, M=24, S=4, dim=8, salt=9)
    A = np.exp(A0) / np.exp(A0).sum(0)
    W = np.exp(L0) / np.exp(L0).sum(0)
    dist.init_process_group("gloo", rank=0, world_size=1)
    try:
        gA, gl = rw.wdl_batch_grad_dp(A, W, Y, C, reg=0.05, L=10, mode=1)
    finally:
        dist.destroy_process_group()
    rA, rl = rw.wdl_batch_grad(A, W, Y, C, reg=0.05, L=10, mode=1)
    assert np.abs(gA - rA).max() <= 1e-14 * np.abs(rA).max()
    assert np.abs(gl - rl).max() <= 1e-14 * np.abs(rl).max()
