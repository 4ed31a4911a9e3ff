"""The engine against rwig's own GPU code (src/cuda_sinkhorn.cu,
src/cuda_barycenter.cu), compiled from the reference's sources into
oracle/_ref by `make -C oracle ref`: the same problems give the same
iteration counts and results to the parity tolerance.  Skipped where that
library was not built."""
import numpy as np
import pytest

import oracle
import rwig_b200 as rw
from rwig_b200 import synth
from tests.util import PARITY_TOL, rel_err

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.ref_gpu_available(), reason="oracle/_ref not built")]


@pytest.mark.parametrize("m,n,reg", [(256, 256, 0.1), (300, 200, 0.05), (64, 512, 0.2)])
def test_vanilla_sinkhorn_matches_reference_gpu(m, n, reg):
    a, b, C = synth.sinkhorn_problem(m, n, 1.0, salt=m + 3 * n)
    ref = oracle.ref_gpu_sinkhorn_vanilla(a, b, C, reg, max_iter=1000, zero_tol=1e-9)
    got = rw.sinkhorn(a, b, C, {"reg": reg, "method": "vanilla", "max_iter": 1000, "zero_tol": 1e-9})
    assert got["iter"] == ref["iter"], (got["iter"], ref["iter"])
    for k in ("P", "u", "v"):
        assert rel_err(got[k], ref[k]) <= PARITY_TOL, (k, rel_err(got[k], ref[k]))
    assert abs(got["loss"] - ref["loss"]) <= PARITY_TOL * abs(ref["loss"])


@pytest.mark.parametrize("N,S,L", [(128, 4, 20), (512, 8, 30)])
def test_parallel_barycenter_matches_reference_gpu(N, S, L):
    A, C, w, be = synth.barycenter_config(n=N, S=S, dim=10)
    ref = oracle.ref_gpu_barycenter_parallel(A, C, w, be, reg=0.1, with_grad=True, max_iter=L, zero_tol=0.0)
    got = rw.barycenter(A, C, w, be, {"reg": 0.1, "method": "parallel", "with_grad": True, "max_iter": L,
                                      "zero_tol": 0.0})
    assert got["iter"] == ref["iter"] == L
    for k in ("b", "U", "V", "grad_A", "grad_w"):
        assert rel_err(got[k], ref[k]) <= PARITY_TOL, (k, rel_err(got[k], ref[k]))
    assert abs(got["loss"] - ref["loss"]) <= PARITY_TOL * abs(ref["loss"])


def _wdl_batch_inputs(N, D, S, reg, salt, dim=8):
    Y, C, A0, L0 = synth.wdl_config(V=N, M=D, S=S, dim=dim, salt=salt)
    A = oracle.col_softmax(A0)
    W = oracle.col_softmax(L0)
    K = np.asfortranarray(np.exp(-C / reg))
    return Y, C, K, A, W


@pytest.mark.parametrize("N,D,S,L", [(200, 8, 4, 5), (333, 5, 16, 3), (150, 9, 7, 4), (64, 1, 3, 6),
                                     (257, 3, 64, 2)])
def test_wdl_batch_grad_matches_reference_gpu(N, D, S, L):
    """The engine's batched WDL gradient, the oracle's and the reference's own
    unrolled wdl_batch (src/cuda_wdl.cu:385-537) on the same batch."""
    reg = 0.1
    Y, C, K, A, W = _wdl_batch_inputs(N, D, S, reg, salt=N + 2 * D + S)
    rgA, rgl, _ = oracle.ref_gpu_wdl_batch_grad(A, W, Y, K, reg, L, mode=0)
    ogA, ogl = oracle.wdl_batch_grad(A, W, Y, K, L)
    gA, gl = rw.wdl_batch_grad(A, W, Y, K, reg, L, mode=0)
    # the oracle (CPU restatement) against the reference's GPU code
    assert rel_err(ogA, rgA) <= PARITY_TOL and rel_err(ogl, rgl) <= PARITY_TOL, (rel_err(ogA, rgA), rel_err(ogl, rgl))
    assert rel_err(gA, rgA) <= PARITY_TOL, rel_err(gA, rgA)
    assert rel_err(gl, rgl) <= PARITY_TOL, rel_err(gl, rgl)
    # the cost given instead of the kernel: both sides form exp(-C/reg)
    rgA1, rgl1, _ = oracle.ref_gpu_wdl_batch_grad(A, W, Y, C, reg, L, mode=1)
    gA1, gl1 = rw.wdl_batch_grad(A, W, Y, C, reg, L, mode=1)
    assert rel_err(gA1, rgA1) <= PARITY_TOL and rel_err(gl1, rgl1) <= PARITY_TOL


def test_wdl_batch_grad_full_size_matches_reference_gpu():
    """One batch of the WDL training workload at full size: V = 5000
    embeddings in R^64, K = 16 topics, B = 64 documents, eps = 0.05, L = 20."""
    Y, C, A0, L0 = synth.wdl_config(V=5000, M=64, S=16, dim=64, salt=0)
    A, W = oracle.col_softmax(A0), oracle.col_softmax(L0)
    rgA, rgl, _ = oracle.ref_gpu_wdl_batch_grad(A, W, Y, C, 0.05, 20, mode=1)
    gA, gl = rw.wdl_batch_grad(A, W, Y, C, 0.05, 20, mode=1)
    assert np.isfinite(rgA).all() and np.abs(rgA).max() > 0
    assert rel_err(gA, rgA) <= PARITY_TOL, rel_err(gA, rgA)
    assert rel_err(gl, rgl) <= PARITY_TOL, rel_err(gl, rgl)


@pytest.mark.parametrize("opt", [0, 1, 2])
def test_wdl_training_matches_reference_gpu(opt):
    """Seeded training over two epochs with a ragged last batch: the engine's
    rwig_wdl draws the initial logits as cuda_wdl does (mt19937(seed), N(0,1),
    Alpha then Lambda, src/cuda_wdl.cu:592-689), so the learned topics A and
    weights W agree.  Yhat is not compared: the reference's inference reads
    history slots its forward-only barycenter never wrote (cuda_wdl.cu:765-769)."""
    N, M, S, B, E, L, reg, seed = 120, 21, 4, 8, 2, 5, 0.1, 11
    Y, C, _, _ = synth.wdl_config(V=N, M=M, S=S, dim=6, salt=opt + 50)
    ref = oracle.ref_gpu_wdl(Y, C, S, reg, L, 1e-6, B, E, opt=opt, eta=1e-2, seed=seed)
    got = rw.wdl_cpp(Y, C, reg, S, B, E, max_iter=L, zero_tol=1e-6, optimizer=opt, eta=1e-2, seed=seed)
    assert rel_err(got["A"], ref["A"]) <= PARITY_TOL, rel_err(got["A"], ref["A"])
    assert rel_err(got["W"], ref["W"]) <= PARITY_TOL, rel_err(got["W"], ref["W"])
