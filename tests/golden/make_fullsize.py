"""Writes the full-size oracle fixtures the GPU parity tests compare against
(each CPU solve takes minutes, the GPU tests seconds):

  bary2048_oracle.npz   the log-barycenter benchmark workload: N = 2048 points
                        ~ N(0, I_50), S = 32 Dirichlet(0.3) histograms,
                        eps = 0.05, L = 50 fixed iterations, with gradient:
                        b, grad_A, grad_w, loss, err and F, G on every 4th row;
  sink8192_oracle.npz   one 8192 x 8192 log-Sinkhorn request of the serving
                        stream's kind (Dirichlet(1), points uniform in [0,1]^3,
                        eps = 0.05, tol 1e-9, max_iter 2000): iter, err, loss, f, g.

Inputs come from rwig_b200.synth (seeded), so only outputs are stored.
Usage: python tests/golden/make_fullsize.py [bary|sink ...]"""
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from rwig_b200 import synth  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
THREADS = os.cpu_count() or 1


def sink8192_inputs():
    a, b, x, y = synth.stream_request_data(8192, 8192, 3, 777)
    return a, b, synth.sq_euclid_cost(x, y)


def make_bary():
    A, C, w, be = synth.barycenter_config(n=2048, S=32, dim=50)
    t0 = time.time()
    r = oracle.barycenter_log(A, C, w, be, 0.05, with_grad=True, n_threads=THREADS, max_iter=50, zero_tol=0.0)
    dst = os.path.join(HERE, "bary2048_oracle.npz")
    np.savez_compressed(dst, b=r["b"], grad_A=r["grad_A"], grad_w=r["grad_w"], loss=r["loss"], err=r["err"],
                        iter=r["iter"], return_status=r["return_status"], F4=r["F"][::4], G4=r["G"][::4])
    print("wrote", dst, r["iter"], r["loss"], f"{time.time() - t0:.0f} s")


def make_sink():
    a, b, C = sink8192_inputs()
    t0 = time.time()
    r = oracle.sinkhorn_log(a, b, C, 0.05, max_iter=2000, zero_tol=1e-9, n_threads=THREADS, want_P=False)
    dst = os.path.join(HERE, "sink8192_oracle.npz")
    np.savez_compressed(dst, iter=r["iter"], err=r["err"], loss=r["loss"], f=r["f"], g=r["g"],
                        return_status=r["return_status"])
    print("wrote", dst, r["iter"], r["loss"], f"{time.time() - t0:.0f} s")


if __name__ == "__main__":
    which = sys.argv[1:] or ["bary", "sink"]
    for k in which:
        {"bary": make_bary, "sink": make_sink}[k]()
