"""The allocation-free log-Sinkhorn entry (rwig_sinkhorn_log_noalloc).

It serves callers that cannot let a library allocate device memory -- a host
framework that owns the GPU's memory pool, a process under a hard device-memory
quota, a serving loop that must not stall on cudaMalloc/cudaFree -- by running
the solver on a fixed scratch block inside the library.  Its results must match
the allocating entry (rwig_sinkhorn_log_dev) on the same inputs, call after
call, although every call reuses the same block.  This file is collected last
on purpose.
"""
import ctypes

import numpy as np
import pytest

from rwig_b200 import _lib, synth
from tests.util import PARITY_TOL, dual_scale, rel_err

pytestmark = pytest.mark.gpu


def _dev_buffers(m, n, salt, reg):
    import torch
    a, b, C = synth.sinkhorn_problem(m, n, 0.5, salt=salt)
    d = torch.device("cuda:0")
    return dict(a=torch.from_numpy(a).to(d), b=torch.from_numpy(b).to(d),
                C=torch.from_numpy(np.ascontiguousarray(C.T)).to(d), m=m, n=n, reg=reg)


def _outputs(m, n):
    import torch
    d = torch.device("cuda:0")
    return (torch.full((n, m), np.nan, dtype=torch.float64, device=d),
            torch.full((m,), np.nan, dtype=torch.float64, device=d),
            torch.full((n,), np.nan, dtype=torch.float64, device=d))


def _call(fn_name, prob, max_iter=1000, tol=1e-9):
    import torch
    L = _lib.load()
    P, f, g = _outputs(prob["m"], prob["n"])
    loss, err, it = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
    vp = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    if fn_name == "noalloc":
        rc = L.rwig_sinkhorn_log_noalloc(vp(P), vp(f), vp(g), ctypes.byref(loss), ctypes.byref(it),
                                         ctypes.byref(err), vp(prob["a"]), vp(prob["b"]), vp(prob["C"]),
                                         prob["m"], prob["n"], prob["reg"], max_iter, tol, st)
    else:
        rc = L.rwig_sinkhorn_log_dev(vp(P), None, vp(f), vp(g), ctypes.byref(loss), ctypes.byref(it),
                                     ctypes.byref(err), vp(prob["a"]), vp(prob["b"]), vp(prob["C"]),
                                     prob["m"], prob["n"], prob["reg"], 0, max_iter, tol, st)
    _lib.check(rc)
    torch.cuda.synchronize()
    return dict(rc=rc, P=P.cpu().numpy(), f=f.cpu().numpy(), g=g.cpu().numpy(), loss=loss.value,
                iter=it.value, err=err.value)


def _same(got, ref):
    assert got["rc"] == ref["rc"] and got["iter"] == ref["iter"]
    assert rel_err(got["P"], ref["P"]) <= PARITY_TOL
    sc = dual_scale(ref["f"], ref["g"])
    assert rel_err(got["f"], ref["f"], sc) <= PARITY_TOL
    assert rel_err(got["g"], ref["g"], sc) <= PARITY_TOL
    assert abs(got["loss"] - ref["loss"]) <= PARITY_TOL * abs(ref["loss"])


def test_two_calls_in_a_row_match_allocating_entry():
    first = _dev_buffers(1024, 768, salt=21, reg=0.05)
    second = _dev_buffers(4096, 1536, salt=22, reg=0.02)
    ref1 = _call("dev", first)
    ref2 = _call("dev", second)
    got1 = _call("noalloc", first)
    got2 = _call("noalloc", second)  # reuses the scratch block left by the first call
    _same(got1, ref1)
    _same(got2, ref2)


def test_rejects_sizes_beyond_the_limit():
    prob = _dev_buffers(4098, 64, salt=23, reg=0.05)
    with pytest.raises(_lib.RwigError) as ei:
        _call("noalloc", prob)
    assert ei.value.code == -6 and "4096" in str(ei.value)


def test_rejects_negative_max_iter():
    prob = _dev_buffers(64, 64, salt=24, reg=0.05)
    with pytest.raises(_lib.RwigError) as ei:
        _call("noalloc", prob, max_iter=-1)
    assert ei.value.code == -1 and "max_iter" in str(ei.value)
