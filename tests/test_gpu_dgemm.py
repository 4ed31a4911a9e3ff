"""The engine's FP64 tensor-core GEMM (mma.sync m16n8k4 .f64, cluster split-K) against
numpy on the host, for both orientations and ragged shapes."""
import ctypes

import numpy as np
import pytest

from rwig_b200 import _lib

pytestmark = pytest.mark.gpu


def _run(K, X, trans, splits=0, ldy_extra=0):
    import torch
    d = torch.device("cuda:0")
    Mk, Nk = K.shape
    Mo, Kd = (Nk, Mk) if trans else (Mk, Nk)
    S = X.shape[1]
    ldk = Mk + (Mk % 2)  # even leading dimension
    Kp = np.zeros((ldk, Nk), order="F")
    Kp[:Mk, :] = K
    tK = torch.from_numpy(np.ascontiguousarray(Kp.T)).to(d)  # column-major ldk x Nk
    tX = torch.from_numpy(np.ascontiguousarray(X.T)).to(d)
    ldy = Mo + ldy_extra
    tY = torch.full((S, ldy), np.nan, dtype=torch.float64, device=d)
    vp = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    rc = _lib.check(_lib.load().rwig_selftest_dgemm(vp(tK), ldk, int(trans), Mo, Kd, S, vp(tX), Kd, vp(tY), ldy,
                                                    splits, None))
    assert rc >= 1
    _run.splits = rc
    return tY.cpu().numpy().T[:Mo, :]


@pytest.mark.parametrize("trans", [0, 1])
@pytest.mark.parametrize("Mk,Nk,S", [(64, 64, 32), (2048, 2048, 32), (130, 70, 5), (1, 3, 1), (333, 517, 47),
                                     (5000, 257, 64)])
def test_against_numpy(trans, Mk, Nk, S):
    g = np.random.default_rng(Mk * 7 + Nk + S)
    K = g.standard_normal((Mk, Nk))
    X = g.standard_normal((Mk if trans else Nk, S))
    ref = (K.T if trans else K) @ X
    got = _run(K, X, trans)
    assert np.abs(got - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max()) * np.sqrt(X.shape[0])


@pytest.mark.parametrize("splits,used", [(1, 1), (2, 2), (3, 2), (4, 4), (8, 8), (17, 8)])
def test_split_counts_agree(splits, used):
    """Cluster split-K: requested counts round down to 1, 2, 4 or 8."""
    g = np.random.default_rng(5)
    K = g.random((512, 384))
    X = g.random((384, 32))
    ref = K @ X
    got = _run(K, X, 0, splits=splits)
    assert _run.splits == used
    assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()


@pytest.mark.parametrize("trans", [0, 1])
def test_bitwise_repeatable(trans):
    """Fixed-order split reduction: identical bits on every run."""
    g = np.random.default_rng(11)
    K = g.standard_normal((2048, 2048))
    X = g.standard_normal((2048, 32))
    first = _run(K, X, trans)
    for _ in range(3):
        assert np.array_equal(_run(K, X, trans), first)


@pytest.mark.parametrize("W", [65, 130, 1024])
def test_wide_outputs(W):
    """Outputs wider than one 64-column tile."""
    g = np.random.default_rng(W)
    K = g.standard_normal((300, 257))
    X = g.standard_normal((257, W))
    ref = K @ X
    got = _run(K, X, 0)
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max() * 16
