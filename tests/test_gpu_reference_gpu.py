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
