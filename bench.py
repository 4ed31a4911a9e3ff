"""Benchmark: log-stabilised Sinkhorn, one 4096 x 4096 FP64 problem per solve.

Workload: a, b ~ Dirichlet(0.5) (n = m = 4096), support points uniform in
[0,1]^2, squared-Euclidean cost normalised by its max, eps = 0.01,
max_iter = 2000, zero_tol = 1e-9; outputs plan P, potentials f, g, loss.
Synthetic, seeded inputs (rwig_b200.synth); no dataset.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

One step = one full solve.  `value` = solves/s over all ranks with inputs
already resident in HBM (CUDA events on the launching stream, L2 flushed
between steps); `e2e` = the same through the host-pointer C ABI
(rwig_sinkhorn_log) with pinned host buffers, copies included.  With N > 1
each rank solves its own replica (the path has no exchange step).
--impl reference times the reference algorithm's CPU implementation (the C++
restatement in oracle/) on this host's cores.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import re
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

M = N = 4096
REG = 0.01
MAX_ITER = 2000
TOL = 1e-9
WORKLOAD = (f"log-Sinkhorn {M}x{N} FP64, Dirichlet(0.5) marginals, uniform points in [0,1]^2, "
            f"squared-Euclidean cost / max, eps={REG}, max_iter={MAX_ITER}, tol={TOL:g}, outputs P,f,g,loss")
METRIC = "log-Sinkhorn solves/s (4096x4096, FP64)"
UNIT = "solves/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    # profiling entry point: one warm-up and one measured solve of a chosen size
    ap.add_argument("--single", action="store_true")
    ap.add_argument("--m", type=int, default=M)
    ap.add_argument("--n", type=int, default=N)
    ap.add_argument("--iters", type=int, default=20)
    ap.add_argument("--l2-hot", type=float, default=None, help="engine option log_sinkhorn.l2_hot")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic(iters):
    """DRAM bytes of the scaled sweep kernel over `iters` iterations, from the
    committed ncu summary of a smaller launch of the same kernel (traffic grows
    in proportion to the iterations), or None."""
    p = os.path.join(ROOT, "profiles", "scaled_kernel_4096.md")
    if not os.path.exists(p):
        return None
    m = re.search(r"dram_bytes_per_iteration:\s*([0-9.eE+]+)", open(p).read())
    return float(m.group(1)) * iters if m else None


class ClockSampler:
    """Samples nvidia-smi SM clocks and throttle reasons while running."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        import tempfile
        self.fh = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
            time.sleep(0.5)  # let the sampler start before the timed region
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.3)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        self.fh.close()
        with open(self.fh.name) as fh:
            self.lines = [ln.strip() for ln in fh if ln.strip()]
        os.unlink(self.fh.name)

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_solve_estimate(a, b, C, threads, iters_full, lo=2, hi=8):
    """Time the oracle at two iteration counts and extrapolate one full solve.
    Returns (seconds per solve, description of the sample)."""
    import oracle
    t = {}
    for it in (lo, hi):
        t0 = time.perf_counter()
        oracle.sinkhorn_log(a, b, C, REG, max_iter=it, zero_tol=0.0, n_threads=threads)
        t[it] = time.perf_counter() - t0
    per_iter = max((t[hi] - t[lo]) / (hi - lo), 1e-9)
    fixed = max(t[lo] - lo * per_iter, 0.0)
    secs = fixed + iters_full * per_iter
    sample = (f"{lo}- and {hi}-iteration runs of the same {M}x{N} problem ({threads} threads), "
              f"extrapolated to a {iters_full}-iteration solve: {per_iter * 1e3:.1f} ms/iteration, "
              f"{fixed * 1e3:.0f} ms fixed")
    return secs, sample


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    import numpy as np  # noqa: F401
    from rwig_b200 import synth
    a, b, C = synth.log_config(M, N)
    threads = os.cpu_count() or 1
    # one step = one estimated full solve, timed as two bounded oracle runs
    for _ in range(args.warmup):
        cpu_solve_estimate(a, b, C, threads, MAX_ITER, lo=1, hi=2)
    secs = []
    sample = ""
    for _ in range(args.steps):
        s, sample = cpu_solve_estimate(a, b, C, threads, MAX_ITER)
        secs.append(s)
    tot = sum(secs)
    value = args.steps / tot
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": WORKLOAD, "parallelism": "cpu"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_engine(args):
    import numpy as np
    import torch

    import rwig_b200 as rw
    from rwig_b200 import _lib, synth

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    a, b, C = synth.log_config(M, N)
    ta = torch.from_numpy(a).to(dev)
    tb = torch.from_numpy(b).to(dev)
    tC = torch.from_numpy(C.T).to(dev)  # column-major M x N as a contiguous (N, M) block
    P = torch.empty((N, M), dtype=torch.float64, device=dev)
    f = torch.empty(M, dtype=torch.float64, device=dev)
    g = torch.empty(N, dtype=torch.float64, device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > L2
    stream = torch.cuda.current_stream()

    def solve():
        return rw.sinkhorn_log_device(ta, tb, tC, REG, MAX_ITER, TOL, P=P, f=f, g=g, stream=stream)

    for _ in range(args.warmup):
        flush.zero_()
        solve()
    torch.cuda.synchronize()

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()

    times, kern, iters, launches, sweep_ms, sweep_it = [], [], [], 0, [], []
    with ClockSampler(local) as clocks:
        barrier()
        for _ in range(args.steps):
            flush.zero_()  # L2 flush between timed steps (outside the timed region)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            r = solve()
            e1.record(stream)
            e1.synchronize()
            rep = rw.last_report()
            times.append(e0.elapsed_time(e1))
            kern.append(rep["kernel_ms"])
            sweep_ms.append(rep["sweep_ms"])
            sweep_it.append(rep["sweep_iters"])
            iters.append(r["iter"])
            launches += rep["kernel_launches"]
        barrier()
    tot_ms = sum(times)
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([tot_ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        tot_ms = float(t.item())
    value = args.steps * world / (tot_ms / 1e3)

    # end to end through the host-pointer C ABI, pinned host buffers
    hC = torch.from_numpy(C.T.copy()).pin_memory()
    ha = torch.from_numpy(a).pin_memory()
    hb = torch.from_numpy(b).pin_memory()
    hP = torch.empty((N, M), dtype=torch.float64).pin_memory()
    hf = torch.empty(M, dtype=torch.float64).pin_memory()
    hg = torch.empty(N, dtype=torch.float64).pin_memory()
    L = _lib.load()
    dp = ctypes.POINTER(ctypes.c_double)

    def cp(t):
        return ctypes.cast(ctypes.c_void_p(t.data_ptr()), dp)

    def host_solve():
        loss, err, it = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        rc = L.rwig_sinkhorn_log(cp(hP), None, cp(hf), cp(hg), ctypes.byref(loss), ctypes.byref(it),
                                 ctypes.byref(err), cp(ha), cp(hb), cp(hC), M, N, REG, 0, MAX_ITER, TOL)
        _lib.check(rc)
        return loss.value

    host_solve()
    barrier()
    e2e_s = 0.0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        host_solve()
        e2e_s += time.perf_counter() - t0
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_value = args.steps * world / e2e_s
    assert np.array_equal(hP.numpy(), P.cpu().numpy()), "host and device entry points disagree"

    line = None
    if rank == 0:
        peak, peak_kind = measured_peaks()
        it_mean = sum(iters) / len(iters)
        kms = sum(kern) / len(kern)
        # dominant kernel: the scaled-form sweep kernel; algorithmic bytes = one
        # read of the M x N kernel matrix per iteration it runs
        s_ms = sum(sweep_ms) / len(sweep_ms)
        s_it = sum(sweep_it) / len(sweep_it)
        alg_bytes = s_it * M * N * 8
        achieved = alg_bytes / (s_ms / 1e3) / 1e9 if s_ms > 0 else None
        tr = profiled_traffic(s_it)
        roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None,
                "traffic": tr, "peak_source": peak_kind,
                "kernel": "scaled_kernel (scaled-form log-Sinkhorn sweep)", "kernel_ms_per_solve": s_ms,
                "kernel_iters_per_solve": s_it, "alg_bytes_per_solve": alg_bytes,
                "all_kernels_ms_per_solve": kms,
                "all_kernels_alg_GBps": (it_mean + 2) * M * N * 8 / (kms / 1e3) / 1e9}
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            threads = os.cpu_count() or 1
            secs, sample = cpu_solve_estimate(a, b, C, threads, int(round(it_mean)))
            cpu = {"value": 1.0 / secs, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample}
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": tot_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": WORKLOAD, "parallelism": f"replicas x{world}",
                           "iterations_per_solve": it_mean, "l2": "flushed between steps (256 MB write)"},
                "e2e": {"value": e2e_value, "unit": UNIT,
                        "h2d_bytes_per_step": (M * N + M + N) * 8,
                        "d2h_bytes_per_step": (M * N + M + N) * 8 + 8},
                "gpu_launches": launches, "roofline": roof, "cpu_baseline": cpu,
                "clocks": clocks.summary()}
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_single(args):
    """One warm-up plus one solve of an m x n problem with a fixed iteration
    count (tol 0): the small case the kernel profiles are captured on."""
    import torch

    import rwig_b200 as rw
    from rwig_b200 import synth
    a, b, C = synth.log_config(args.m, args.n)
    if args.l2_hot is not None:
        rw.load().rwig_set_option(b"log_sinkhorn.l2_hot", float(args.l2_hot))
    dev = torch.device("cuda", 0)
    ta, tb = torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)
    tC = torch.from_numpy(C.T).to(dev)
    P = torch.empty((args.n, args.m), dtype=torch.float64, device=dev)
    for _ in range(2):
        r = rw.sinkhorn_log_device(ta, tb, tC, REG, args.iters, 0.0, P=P)
    torch.cuda.synchronize()
    rep = rw.last_report()
    print(json.dumps({"m": args.m, "n": args.n, "iter": r["iter"], "kernel_ms": rep["kernel_ms"],
                      "us_per_iter": rep["kernel_ms"] * 1e3 / max(1, r["iter"]),
                      "sweep_ms": rep["sweep_ms"], "sweep_iters": rep["sweep_iters"],
                      "sweep_us_per_iter": rep["sweep_ms"] * 1e3 / max(1, rep["sweep_iters"]),
                      "launches": rep["kernel_launches"]}))
    return 0


def main():
    args = parse()
    if args.single:
        return run_single(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_engine(args)


if __name__ == "__main__":
    sys.exit(main())
