"""The engine's table-driven exponential against CUDA's exp on the device."""
import ctypes

import numpy as np
import pytest

from rwig_b200 import _lib

pytestmark = pytest.mark.gpu


def _pair(x):
    import torch
    d = torch.device("cuda:0")
    tx = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64)).to(d)
    ye, yc = torch.empty_like(tx), torch.empty_like(tx)
    vp = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    _lib.check(_lib.load().rwig_selftest_exp(vp(tx), vp(ye), vp(yc), tx.numel(), None))
    return ye.cpu().numpy(), yc.cpu().numpy()


def _ulps(a, b):
    ia = a.view(np.int64)
    ib = b.view(np.int64)
    return np.abs(ia - ib)


def test_within_two_ulp_of_cuda_exp():
    g = np.random.default_rng(123)
    x = np.concatenate([
        g.uniform(-708.0, 709.0, 2_000_000),
        g.uniform(-40.0, 0.0, 2_000_000),              # the solver's working range
        -np.logspace(-300, 2.8, 200_000), np.logspace(-300, 2.8, 200_000),
        np.array([0.0, -0.0, 1.0, -1.0, 709.0, -708.0, 1e-17, -1e-17]),
    ])
    ye, yc = _pair(x)
    assert np.all(np.isfinite(ye)) and np.all(ye > 0)
    assert _ulps(ye, yc).max() <= 2


def test_range_ends_are_clamped():
    x = np.array([-709.0, -800.0, -1e300, 710.0, 1e300, -np.inf])
    ye, yc = _pair(x)
    floor = _pair(np.array([-708.0]))[0][0]
    assert 0.0 < floor < 3.4e-308
    assert np.all(ye[[0, 1, 2, 5]] == floor)
    assert ye[3] == ye[4] == _pair(np.array([709.0]))[0][0]
