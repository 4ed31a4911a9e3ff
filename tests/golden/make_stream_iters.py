"""Writes tests/golden/stream_iters.json: the iteration count of every request
of the 200-request benchmark stream (bench.py --workload stream), which the
CPU reference arm needs to scale its timed sample to the whole stream without
solving the largest requests on the CPU (each would take minutes).  The counts
come from the engine's batched call on a GPU; the engine's iteration counts
equal the oracle's (tests/test_gpu_batch.py, and bench.py checks the batched
and per-call counts agree).  Usage (needs a GPU):
    python tests/golden/make_stream_iters.py [output path]"""
import ctypes
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def main():
    import torch

    from rwig_b200 import _lib
    dev = torch.device("cuda", 0)
    wl = bench.StreamWorkload()
    data = wl.build(dev)
    res = (_lib.Result * len(data))()
    _lib.check(_lib.load().rwig_batch_sinkhorn_log_dev(wl.problems(data), len(data), res,
                                                        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    iters = [res[i].iter for i in range(len(data))]
    dst = sys.argv[1] if len(sys.argv) > 1 else os.path.join(os.path.dirname(os.path.abspath(__file__)),
                                                              "stream_iters.json")
    with open(dst, "w") as fh:
        json.dump({"requests": len(data), "max_iter": wl.max_iter, "tol": wl.tol, "iters": iters}, fh)
    print("wrote", dst, sum(iters))


if __name__ == "__main__":
    main()
