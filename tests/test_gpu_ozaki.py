"""FP64 products emulated on the INT8 tensor cores (ozaki.cu / ozaki.cuh).

* The tcgen05 kind::i8 GEMM itself (rwig_selftest_i8gemm) is exact: its
  int32 products equal numpy's int64 products bit for bit, on tile-aligned
  and ragged shapes.
* The emulated FP64 product (rwig_selftest_ozaki: scaling, 24 residue planes,
  CRT reconstruction) agrees with an exactly rounded reference computed in
  extended precision (numpy longdouble sums of the FP64 products) to a few
  ulp, for K and K^T, positive and mixed-sign operands, wide dynamic range."""
import ctypes

import numpy as np
import pytest

from rwig_b200 import _lib, synth

pytestmark = pytest.mark.gpu


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


@pytest.mark.parametrize("tile_m", [0, 128, 256])
@pytest.mark.parametrize("M,N,Kd", [(128, 16, 128), (256, 256, 512), (200, 40, 300), (1000, 300, 5000),
                                    (5000, 1024, 256), (130, 257, 129)])
def test_int8_gemm_is_exact(M, N, Kd, tile_m):
    """Both tile shapes (256 rows with one accumulator, 128 rows with two)
    and the default choice; persistent CTAs walk several tiles each."""
    import torch
    g = np.random.default_rng(M + N + Kd)
    A = g.integers(-128, 128, size=(M, Kd), dtype=np.int8)
    B = g.integers(-128, 128, size=(N, Kd), dtype=np.int8)
    d = torch.device("cuda:0")
    tA, tB = torch.from_numpy(A).to(d), torch.from_numpy(B).to(d)
    tD = torch.zeros((N, M), dtype=torch.int32, device=d)
    lib = _lib.load()
    lib.rwig_set_option(b"oz.tile_m", float(tile_m) if tile_m else float("nan"))
    try:
        _lib.check(lib.rwig_selftest_i8gemm(_vp(tA), _vp(tB), M, N, Kd, _vp(tD), None))
    finally:
        lib.rwig_set_option(b"oz.tile_m", float("nan"))
    ref = A.astype(np.int64) @ B.astype(np.int64).T
    assert np.array_equal(tD.cpu().numpy().T.astype(np.int64), ref)


def _exact(K, X):
    """K X with every product and sum in extended precision, then rounded."""
    return (K.astype(np.longdouble) @ X.astype(np.longdouble)).astype(np.float64)


@pytest.mark.parametrize("n,W,trans,signed", [(500, 64, 0, False), (500, 64, 1, False), (777, 40, 0, True),
                                              (2048, 300, 1, True), (5000, 1024, 0, False)])
def test_emulated_fp64_product(n, W, trans, signed):
    import torch
    g = np.random.default_rng(n + W)
    x = g.standard_normal((n, 16))
    C = synth.sq_euclid_cost(x, x)
    K = np.asfortranarray(np.exp(-C / 0.05))  # entries from 1 down to e^-20
    X = np.asfortranarray(np.exp(g.uniform(-8, 8, size=(n, W))))  # column dynamic range e^16
    if signed:
        X *= np.where(g.random((n, W)) < 0.5, -1.0, 1.0)
    d = torch.device("cuda:0")
    tK = torch.from_numpy(np.ascontiguousarray(K.T)).to(d)
    tX = torch.from_numpy(np.ascontiguousarray(X.T)).to(d)
    tY = torch.zeros((W, n), dtype=torch.float64, device=d)
    _lib.check(_lib.load().rwig_selftest_ozaki(_vp(tK), n, trans, n, _vp(tX), n, W, _vp(tY), n, None))
    Y = tY.cpu().numpy().T
    op = K.T if trans else K
    ref = _exact(op, X) if n <= 800 else op @ X
    err = np.abs(Y - ref) / (np.abs(op) @ np.abs(X))  # relative to the FP64 GEMM error scale sum |K||X|
    assert err.max() <= 1e-14, err.max()
    if not signed:  # positive operands: no cancellation, relative to each entry
        assert (np.abs(Y - ref) / np.abs(ref)).max() <= 1e-13


@pytest.mark.parametrize("trans", [0, 1])
def test_emulated_product_with_cancellation(trans):
    """Two identical support points make two identical columns of K; X's
    columns e_0 (1 + 2^-52) - e_1 and e_0 - e_1 give products 2^-52 K[:, 0]
    and exactly 0, far below the scale of the operands, where the
    reconstruction needs all 256 bits of its fraction."""
    import torch
    g = np.random.default_rng(5)
    n = 300
    x = g.standard_normal((n, 8))
    x[1] = x[0]
    C = synth.sq_euclid_cost(x, x)
    K = np.asfortranarray(np.exp(-C / 0.05))
    X = np.zeros((n, 4), order="F")
    X[0, 0], X[1, 0] = 1.0 + 2.0 ** -52, -1.0
    X[0, 2], X[1, 2] = 1.0, -1.0
    X[:, 1] = np.exp(g.uniform(-8, 8, n))
    X[:, 3] = g.standard_normal(n)
    d = torch.device("cuda:0")
    tK = torch.from_numpy(np.ascontiguousarray(K.T)).to(d)
    tX = torch.from_numpy(np.ascontiguousarray(X.T)).to(d)
    tY = torch.zeros((4, n), dtype=torch.float64, device=d)
    _lib.check(_lib.load().rwig_selftest_ozaki(_vp(tK), n, trans, n, _vp(tX), n, 4, _vp(tY), n, None))
    Y = tY.cpu().numpy().T
    op = K.T if trans else K
    exact0 = op[:, 0] * 2.0 ** -52  # op[:, 0] == op[:, 1] exactly
    assert np.array_equal(op[:, 0], op[:, 1])
    assert np.abs(Y[:, 0] - exact0).max() <= 2.0 ** -52 * np.abs(exact0).max()
    assert np.all(np.abs(Y[:, 0] - exact0) <= 2.0 ** -51 * np.abs(exact0))
    assert not Y[:, 2].any()
    ref = _exact(op, X)
    for j in (1, 3):
        err = np.abs(Y[:, j] - ref[:, j]) / (np.abs(op) @ np.abs(X[:, j]))
        assert err.max() <= 1e-14, (j, err.max())
