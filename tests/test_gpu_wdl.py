"""Parity of the CUDA Wasserstein dictionary learning (rwig_wdl_batch_grad,
rwig_wdl) with the CPU oracle (WassersteinDictionaryLearning::
_train_batch_batched and _compute_serial restated).  WDL has no known-answer
vectors in the reference's own tests, so the oracle is the pin here; its
batched adjoint is the parallel-barycenter adjoint, which the barycenter tests
check against finite differences."""
import numpy as np
import pytest

import oracle
import rwig_b200 as rw
from rwig_b200 import RwigError, synth
from tests.util import PARITY_TOL, rel_err

pytestmark = pytest.mark.gpu


def _batch(N, M, S, dim, reg, salt):
    Y, C, A0, L0 = synth.wdl_config(V=N, M=M, S=S, dim=dim, salt=salt)
    A = oracle.col_softmax(A0)
    W = oracle.col_softmax(L0)
    K = np.asfortranarray(np.exp(-C / reg))
    return Y, C, K, A, W


@pytest.mark.parametrize("N,D,S,L", [(200, 8, 4, 5), (333, 5, 16, 3), (150, 9, 7, 4), (64, 1, 3, 6),
                                     (257, 3, 64, 2), (100, 4, 5, 1)])
def test_batch_grad_matches_oracle(N, D, S, L):
    reg = 0.1
    Y, C, K, A, W = _batch(N, D, S, 8, reg, salt=N + D + S)
    ref_gA, ref_gl = oracle.wdl_batch_grad(A, W, Y, K, L)
    gA, gl = rw.wdl_batch_grad(A, W, Y, K, reg, L, mode=0)
    assert rel_err(gA, ref_gA) <= PARITY_TOL, rel_err(gA, ref_gA)
    assert rel_err(gl, ref_gl) <= PARITY_TOL, rel_err(gl, ref_gl)
    # mode 1: the engine forms K = exp(-C/reg) itself
    gA1, gl1 = rw.wdl_batch_grad(A, W, Y, C, reg, L, mode=1)
    assert rel_err(gA1, ref_gA) <= PARITY_TOL and rel_err(gl1, ref_gl) <= PARITY_TOL


def test_batch_grad_zero_iterations_is_zero():
    Y, C, K, A, W = _batch(50, 3, 4, 4, 0.1, salt=3)
    gA, gl = rw.wdl_batch_grad(A, W, Y, K, 0.1, 0, mode=0)
    assert not gA.any() and not gl.any()


def test_batch_grad_repeatable():
    Y, C, K, A, W = _batch(300, 16, 16, 8, 0.1, salt=9)
    first = rw.wdl_batch_grad(A, W, Y, K, 0.1, 4, mode=0)
    for _ in range(2):
        again = rw.wdl_batch_grad(A, W, Y, K, 0.1, 4, mode=0)
        assert np.array_equal(again[0], first[0]) and np.array_equal(again[1], first[1])


@pytest.mark.parametrize("opt", [0, 1, 2])
def test_training_matches_oracle(opt):
    """Training with a ragged last batch (M % B != 0) over two epochs."""
    N, M, S, B, E, L, reg = 120, 21, 4, 8, 2, 5, 0.1
    Y, C, A0, L0 = synth.wdl_config(V=N, M=M, S=S, dim=6, salt=opt + 40)
    ref = oracle.wdl_train(Y, C, S, reg, L, B, E, A0, L0, opt=opt, eta=1e-2)
    got = rw.wdl_cpp(Y, C, reg, S, B, E, max_iter=L, zero_tol=1e-6, optimizer=opt, eta=1e-2, Alpha0=A0,
                     Lambda0=L0)
    assert rel_err(got["A"], ref["A"]) <= PARITY_TOL, rel_err(got["A"], ref["A"])
    assert rel_err(got["W"], ref["W"]) <= PARITY_TOL, rel_err(got["W"], ref["W"])
    assert rw.last_report()["iter"] == ref["steps"] == E * 3


def test_max_steps_and_inference():
    """max_steps stops training early; Yhat is the parallel barycenter of every
    document under the learned topics (wdl_impl.cpp:349-377)."""
    N, M, S, B, L, reg = 90, 10, 3, 4, 6, 0.1
    Y, C, A0, L0 = synth.wdl_config(V=N, M=M, S=S, dim=5, salt=7)
    ref = oracle.wdl_train(Y, C, S, reg, L, B, 3, A0, L0, opt=2, eta=5e-3, max_steps=4)
    got = rw.wdl_cpp(Y, C, reg, S, B, 3, max_iter=L, zero_tol=1e-6, optimizer=2, eta=5e-3, Alpha0=A0,
                     Lambda0=L0, max_steps=4)
    assert rel_err(got["A"], ref["A"]) <= PARITY_TOL and rel_err(got["W"], ref["W"]) <= PARITY_TOL
    for m in range(M):
        b = oracle.barycenter_parallel(ref["A"], C, ref["W"][:, m], None, reg, with_grad=False, max_iter=L,
                                       zero_tol=1e-6)["b"]
        assert rel_err(got["Yhat"][:, m], b) <= 1e-9, m


def test_seeded_initialisation_is_deterministic():
    N, M, S = 60, 6, 3
    Y, C, _, _ = synth.wdl_config(V=N, M=M, S=S, dim=4, salt=1)
    r1 = rw.wdl_cpp(Y, C, 0.1, S, 3, 1, max_iter=3, seed=5)
    r2 = rw.wdl_cpp(Y, C, 0.1, S, 3, 1, max_iter=3, seed=5)
    r3 = rw.wdl_cpp(Y, C, 0.1, S, 3, 1, max_iter=3, seed=6)
    assert np.array_equal(r1["A"], r2["A"]) and not np.array_equal(r1["A"], r3["A"])
    np.testing.assert_allclose(r1["A"].sum(axis=0), 1.0, rtol=1e-12)
    np.testing.assert_allclose(r1["W"].sum(axis=0), 1.0, rtol=1e-12)


def test_invalid_arguments():
    Y, C, K, A, W = _batch(40, 2, 3, 3, 0.1, salt=2)
    with pytest.raises(RwigError):
        rw.wdl_batch_grad(A, W, Y, K, 0.1, 3, mode=2)
    with pytest.raises(RwigError):
        rw.wdl_batch_grad(A, W, Y, C, -1.0, 3, mode=1)
    Abig = np.full((40, 65), 1 / 40)
    with pytest.raises(RwigError):
        rw.wdl_batch_grad(Abig, np.full((65, 2), 1 / 65), Y, K, 0.1, 3)
    with pytest.raises(ValueError):
        rw.wdl_cpp(Y, C[:, :-1], 0.1, 3, 2, 1)


def test_batched_inference_chunks_and_per_document_stops():
    """Inference solves every document's barycenter in stacked columns and
    freezes each document at its own stop (iter < max_iter && err >= tol);
    chunks of 1024, 4 or 1 documents give the oracle's per-document results."""
    N, M, S, B, L, reg, tol = 80, 9, 3, 3, 25, 0.1, 1e-6
    Y, C, A0, L0 = synth.wdl_config(V=N, M=M, S=S, dim=5, salt=13)
    lib = rw.load()
    outs = []
    try:
        for docs in (1024, 4, 1):
            lib.rwig_set_option(b"wdl.infer_docs", float(docs))
            outs.append(rw.wdl_cpp(Y, C, reg, S, B, 1, max_iter=L, zero_tol=tol, optimizer=1, eta=1e-3,
                                   Alpha0=A0, Lambda0=L0, max_steps=2))
    finally:
        lib.rwig_set_option(b"wdl.infer_docs", 1024.0)
    ref = oracle.wdl_train(Y, C, S, reg, L, B, 1, A0, L0, opt=1, eta=1e-3, max_steps=2)
    iters = set()
    for m in range(M):
        r = oracle.barycenter_parallel(ref["A"], C, ref["W"][:, m], None, reg, with_grad=False, max_iter=L,
                                       zero_tol=tol)
        iters.add(r["iter"])
        for o in outs:
            assert rel_err(o["Yhat"][:, m], r["b"]) <= 1e-9, (m, rel_err(o["Yhat"][:, m], r["b"]))
    assert len(iters) > 1, iters  # the documents stopped at different iterations


class _Option:
    def __init__(self, name, value):
        self.name, self.value = name.encode(), value

    def __enter__(self):
        rw.load().rwig_set_option(self.name, float(self.value))

    def __exit__(self, *exc):
        rw.load().rwig_set_option(self.name, float("nan"))


@pytest.mark.parametrize("k", [1, 2, 3, 6, 7])
def test_checkpointed_adjoint_is_bitwise_full_history(k):
    """wdl.checkpoint = k keeps the forward state every k-th iteration and
    recomputes the segments in the backward: the same gradient bits as the
    full history (L = 7, so k = 2, 3 leave a short last segment)."""
    reg, L = 0.1, 7
    Y, C, K, A, W = _batch(230, 6, 5, 8, reg, salt=17)
    full = rw.wdl_batch_grad(A, W, Y, K, reg, L, mode=0)
    with _Option("wdl.checkpoint", k):
        got = rw.wdl_batch_grad(A, W, Y, K, reg, L, mode=0)
        launches = rw.last_report()["kernel_launches"]
    assert np.array_equal(got[0], full[0]) and np.array_equal(got[1], full[1])
    ref_gA, ref_gl = oracle.wdl_batch_grad(A, W, Y, K, L)
    assert rel_err(got[0], ref_gA) <= PARITY_TOL
    assert launches > 0


def test_checkpointed_training_matches_full_history():
    N, M, S, B, E, L, reg = 120, 21, 4, 8, 2, 5, 0.1
    Y, C, A0, L0 = synth.wdl_config(V=N, M=M, S=S, dim=6, salt=41)
    full = rw.wdl_cpp(Y, C, reg, S, B, E, max_iter=L, zero_tol=1e-6, optimizer=1, eta=1e-2, Alpha0=A0, Lambda0=L0)
    with _Option("wdl.checkpoint", 2):
        got = rw.wdl_cpp(Y, C, reg, S, B, E, max_iter=L, zero_tol=1e-6, optimizer=1, eta=1e-2, Alpha0=A0,
                         Lambda0=L0)
    for k in ("A", "W", "Yhat"):
        assert np.array_equal(got[k], full[k]), k


@pytest.mark.parametrize("N,D,S,L", [(200, 8, 4, 5), (333, 5, 16, 3), (257, 3, 64, 2), (100, 4, 5, 1),
                                     (1100, 6, 8, 4)])
def test_batch_grad_on_int8_tensor_cores_matches_oracle(N, D, S, L):
    """wdl.int8 = 2: every product of the step emulated on the INT8 tensor
    cores (24 modular planes, CRT); the gradient still within 1e-10 of the
    oracle's, and bitwise repeatable."""
    reg = 0.1
    Y, C, K, A, W = _batch(N, D, S, 8, reg, salt=N + 2 * D)
    ref_gA, ref_gl = oracle.wdl_batch_grad(A, W, Y, K, L)
    with _Option("wdl.int8", 2):
        gA, gl = rw.wdl_batch_grad(A, W, Y, K, reg, L, mode=0)
        again = rw.wdl_batch_grad(A, W, Y, K, reg, L, mode=0)
    assert rel_err(gA, ref_gA) <= PARITY_TOL, rel_err(gA, ref_gA)
    assert rel_err(gl, ref_gl) <= PARITY_TOL, rel_err(gl, ref_gl)
    assert np.array_equal(again[0], gA) and np.array_equal(again[1], gl)


def test_int8_residues_reused_only_for_the_same_K():
    """The K residue planes of the last INT8-path call are reused only when
    the new K equals it bit for bit: the same K skips the preparation (fewer
    launches, the same bits); a K with one row changed, or a K differing in a
    single last bit, is prepared anew (its gradient is its own)."""
    N, D, S, L, reg = 300, 4, 6, 3, 0.1
    Y, C, K, A, W = _batch(N, D, S, 8, reg, salt=17)
    K2 = K.copy()
    K2[5, :] *= 0.9
    K3 = K.copy()
    K3[N - 1, N - 1] = np.nextafter(K3[N - 1, N - 1], 2.0)
    with _Option("wdl.int8", 2):
        g1 = rw.wdl_batch_grad(A, W, Y, K, reg, L, mode=0)
        n1 = rw.last_report()["kernel_launches"]
        g1b = rw.wdl_batch_grad(A, W, Y, K, reg, L, mode=0)
        n1b = rw.last_report()["kernel_launches"]
        g2 = rw.wdl_batch_grad(A, W, Y, K2, reg, L, mode=0)
        n2 = rw.last_report()["kernel_launches"]
        g3 = rw.wdl_batch_grad(A, W, Y, K3, reg, L, mode=0)
        n3 = rw.last_report()["kernel_launches"]
        g1c = rw.wdl_batch_grad(A, W, Y, K, reg, L, mode=0)
        n1c = rw.last_report()["kernel_launches"]
    assert np.array_equal(g1[0], g1b[0]) and np.array_equal(g1[1], g1b[1])
    assert np.array_equal(g1[0], g1c[0]) and np.array_equal(g1[1], g1c[1])
    assert n1b < n1 and n2 > n1b and n3 > n1b and n1c > n1b
    ref2 = oracle.wdl_batch_grad(A, W, Y, K2, L)
    assert rel_err(g2[0], ref2[0]) <= PARITY_TOL and rel_err(g2[1], ref2[1]) <= PARITY_TOL
    ref3 = oracle.wdl_batch_grad(A, W, Y, K3, L)
    assert rel_err(g3[0], ref3[0]) <= PARITY_TOL
    assert not np.array_equal(g2[0], g1[0])


def test_int8_options_keep_the_gradient_bits():
    """wdl.halves = 2 (the batch's two document halves on two streams) and
    oz.tile_m = 128 (the double-buffered GEMM) change scheduling only: the
    same gradient bits.  profile.gemm = 1 times every INT8 GEMM launch of the
    call and reports them."""
    N, D, S, L, reg = 400, 6, 8, 3, 0.1
    Y, C, K, A, W = _batch(N, D, S, 8, reg, salt=23)
    with _Option("wdl.int8", 2):
        base = rw.wdl_batch_grad(A, W, Y, K, reg, L, mode=0)
        with _Option("wdl.halves", 2):
            halves = rw.wdl_batch_grad(A, W, Y, K, reg, L, mode=0)
        with _Option("oz.tile_m", 128):
            tiles = rw.wdl_batch_grad(A, W, Y, K, reg, L, mode=0)
        with _Option("profile.gemm", 1):
            timed = rw.wdl_batch_grad(A, W, Y, K, reg, L, mode=0)
            rep = rw.last_report()
    for got in (halves, tiles, timed):
        assert np.array_equal(got[0], base[0]) and np.array_equal(got[1], base[1])
    assert rep["gemm_launches"] == 4 * L - 1 and rep["gemm_ms"] > 0.0
    assert rep["gemm_ms"] < rep["device_ms"]


def test_training_and_inference_on_int8_tensor_cores():
    N, M, S, B, L, reg = 150, 10, 3, 4, 6, 0.1
    Y, C, A0, L0 = synth.wdl_config(V=N, M=M, S=S, dim=5, salt=71)
    ref = oracle.wdl_train(Y, C, S, reg, L, B, 3, A0, L0, opt=1, eta=5e-3, max_steps=4)
    with _Option("wdl.int8", 2):
        got = rw.wdl_cpp(Y, C, reg, S, B, 3, max_iter=L, zero_tol=1e-6, optimizer=1, eta=5e-3, Alpha0=A0,
                         Lambda0=L0, max_steps=4)
    assert rel_err(got["A"], ref["A"]) <= PARITY_TOL and rel_err(got["W"], ref["W"]) <= PARITY_TOL
    for m in range(M):
        b = oracle.barycenter_parallel(ref["A"], C, ref["W"][:, m], None, reg, with_grad=False, max_iter=L,
                                       zero_tol=1e-6)["b"]
        assert rel_err(got["Yhat"][:, m], b) <= 1e-9, m
