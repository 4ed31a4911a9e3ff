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


class _Tile:
    """Forces the GEMM's tile height (option dgemm.tile) and DMMA shape
    (dgemm.kshape) for the duration of a block."""

    def __init__(self, tile, kshape=None):
        self.tile, self.kshape = tile, kshape

    def __enter__(self):
        lib = _lib.load()
        assert lib.rwig_set_option(b"dgemm.tile", float(self.tile)) == 0
        if self.kshape:
            assert lib.rwig_set_option(b"dgemm.kshape", float(self.kshape)) == 0

    def __exit__(self, *exc):
        lib = _lib.load()
        lib.rwig_set_option(b"dgemm.tile", 0.0)
        lib.rwig_set_option(b"dgemm.kshape", 4.0)


@pytest.mark.parametrize("trans", [0, 1])
@pytest.mark.parametrize("kshape", [4, 8, 16])
@pytest.mark.parametrize("Mk,Nk,S", [(333, 517, 47), (130, 70, 64), (1000, 129, 200), (127, 1, 33)])
def test_wide_tiles(trans, kshape, Mk, Nk, S):
    """128-row tiles (32 x 32 warp blocks) and every DMMA shape
    (m16n8k4 / k8 / k16) on ragged shapes."""
    g = np.random.default_rng(Mk + Nk * 3 + S)
    K = g.standard_normal((Mk, Nk))
    X = g.standard_normal((Mk if trans else Nk, S))
    ref = (K.T if trans else K) @ X
    with _Tile(128, kshape):
        got = _run(K, X, trans)
    assert np.abs(got - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max()) * np.sqrt(X.shape[0])


@pytest.mark.parametrize("splits", [1, 2, 3, 4, 5, 6, 7, 8])
def test_wide_tile_split_counts(splits):
    """Wide tiles under every split count: CTA z of the cluster owns rows
    [z r, z r + r) of the tile with r = 8 ceil(128 / (8 splits)), so counts
    that do not divide 128 leave the last CTAs fewer (or no) rows."""
    g = np.random.default_rng(splits)
    K = g.random((300, 1100))
    X = g.random((1100, 64))
    ref = K @ X
    with _Tile(128):
        got = _run(K, X, 0, splits=splits)
        assert _run.splits == splits
        again = _run(K, X, 0, splits=splits)
    assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()
    assert np.array_equal(got, again)


@pytest.mark.parametrize("Kd", [300, 1000])
def test_wide_tile_tail_wave(Kd):
    """Automatic tiles at the WDL product's width (1024 columns, 5000 rows):
    whole waves of unsplit 128-row tiles, then the last partial wave's tiles
    as a split-K launch (2 or 3 slices here)."""
    g = np.random.default_rng(Kd)
    K = g.standard_normal((5000, Kd))
    X = g.standard_normal((Kd, 1024))
    ref = K @ X
    got = _run(K, X, 0)
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max() * np.sqrt(Kd)
    with _Tile(64):
        narrow = _run(K, X, 0)
    assert np.abs(narrow - ref).max() <= 1e-12 * np.abs(ref).max() * np.sqrt(Kd)
