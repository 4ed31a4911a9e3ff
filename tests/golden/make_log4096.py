"""Writes tests/golden/log4096_oracle.npz: the CPU oracle's full solve of the
4096 x 4096 log-Sinkhorn benchmark workload (iterations, error, loss, f, g), so
the GPU parity test can check the engine at full size without the ~1 minute
CPU solve.  Usage: python tests/golden/make_log4096.py"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from rwig_b200 import synth  # noqa: E402


def main():
    a, b, C = synth.log_config(4096, 4096)
    r = oracle.sinkhorn_log(a, b, C, 0.01, max_iter=2000, zero_tol=1e-9, n_threads=os.cpu_count() or 1,
                            want_P=False)
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "log4096_oracle.npz")
    np.savez_compressed(dst, iter=r["iter"], err=r["err"], loss=r["loss"], f=r["f"], g=r["g"],
                        return_status=r["return_status"])
    print("wrote", dst, r["iter"], r["loss"])


if __name__ == "__main__":
    main()
