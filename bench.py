"""Benchmark of the rwig_b200 engine.

Default workload (the headline, --workload stream): the serving stream of 200
mixed-size log-Sinkhorn requests (n, m log-uniform in [64, 8192], eps from
{0.01, 0.05, 0.1}, Dirichlet(1) histograms, points uniform in [0,1]^d with d
from {2, 3, 64}, squared-Euclidean cost / max, tol 1e-9, max_iter 2000).  One
step = one batched call over the whole stream with device-resident inputs;
`value` = requests solved per second.  The same line carries the plain
per-call path on the same stream ("plain"), the end-to-end batched call on
pinned host buffers ("e2e"), the continuous-batching server's p50/p99
latency under Poisson arrivals at 50/80/100 % of its capacity ("latency"),
the autotuned batched call, and the WDL training workload ("wdl": V = 5000,
K = 16 topics, batch 64, L = 20, Adam; engine steps/s, FP64-tensor fraction,
and one batched adjoint step against the reference's own unrolled GPU step).
Other workloads, one JSON line each:
--workload log4096 (log-Sinkhorn 4096 x 4096, eps = 0.01, Dirichlet(0.5)),
--workload vanilla256 (vanilla Sinkhorn 256 x 256, eps = 0.1, Dirichlet(1)),
--workload barycenter2048 (log barycenter + gradient, N = 2048, S = 32, L = 50),
--workload wdl5000 (WDL training steps, V = 5000, K = 16, batch 64, L = 20, Adam),
--workload sinkgrad2048 (log-Sinkhorn 2048 x 2048 with its gradient w.r.t. a, L = 100).
Synthetic, seeded inputs (rwig_b200.synth); no dataset.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference] [--workload W]

Timing: CUDA events on the launching stream, max over ranks; `e2e` through
the host-pointer C ABI with pinned host buffers, copies included.  With N > 1
each rank runs its own replica (the path has no exchange step).
--impl reference times the reference algorithm's CPU implementation (the C++
restatement in oracle/) on this host's cores, whole solves.
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

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

DEFAULT_WORKLOAD = "stream"
def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--serve-requests", type=int, default=20000,
                    help="stream workload: requests per arrival rate of the serving run")
    ap.add_argument("--no-wdl", action="store_true", help="stream: leave out the WDL block")
    ap.add_argument("--no-autotune", action="store_true",
                    help="stream workload: skip tuning the batch.* options on the stream")
    # profiling entry point: one warm-up and one measured solve of a chosen size
    ap.add_argument("--single", action="store_true")
    ap.add_argument("--gemm", action="store_true",
                    help="with --single: time the engine's FP64 product K X (--n x --n, --m columns) against "
                         "cuBLAS (torch.matmul) on the same operands")
    ap.add_argument("--m", type=int, default=4096)
    ap.add_argument("--n", type=int, default=4096)
    ap.add_argument("--iters", type=int, default=20)
    ap.add_argument("--s", type=int, default=32, help="histograms / topics (barycenter, wdl --single)")
    ap.add_argument("--l2-hot", type=float, default=None, help="engine option log_sinkhorn.l2_hot")
    ap.add_argument("--stream-profile", action="store_true",
                    help="with --single --workload stream: one batched call over the whole 200-request stream "
                         "with engine option batch.profile (per-class phase times on stderr)")
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


class SinkhornWorkload:
    """One full solve of a single Sinkhorn problem per step."""

    higher_is_better = True

    def __init__(self, method, m, n, reg, alpha, max_iter, tol):
        self.method, self.m, self.n, self.reg = method, m, n, reg
        self.alpha, self.max_iter, self.tol = alpha, max_iter, tol
        self.unit = "solves/s"
        kind = "log-Sinkhorn" if method == "log" else "vanilla Sinkhorn"
        self.metric = f"{kind} solves/s ({m}x{n}, FP64)"
        self.desc = (f"{kind} {m}x{n} FP64, Dirichlet({alpha:g}) marginals, uniform points in [0,1]^2, "
                     f"squared-Euclidean cost / max, eps={reg:g}, max_iter={max_iter}, tol={tol:g}, "
                     f"outputs P, {'f, g' if method == 'log' else 'u, v'}, loss")

    def inputs(self):
        from rwig_b200 import synth
        return synth.sinkhorn_problem(self.m, self.n, self.alpha, 2)

    def cpu_seconds(self, threads, iters_full=None):
        """CPU port time of one whole solve of the problem, timed (vanilla:
        repeated whole solves for at least 2 s, 1 thread)."""
        import oracle
        a, b, C = self.inputs()
        if self.method == "vanilla":
            threads = 1  # the reference's vanilla path runs on one BLAS thread
            t0 = time.perf_counter()
            k = 0
            while True:
                oracle.sinkhorn_vanilla(a, b, C, self.reg, max_iter=self.max_iter, zero_tol=self.tol)
                k += 1
                if time.perf_counter() - t0 > 2.0:
                    break
            secs = (time.perf_counter() - t0) / k
            return secs, threads, f"{k} full solves of the same problem, 1 thread"
        t0 = time.perf_counter()
        r = oracle.sinkhorn_log(a, b, C, self.reg, max_iter=self.max_iter, zero_tol=self.tol, n_threads=threads,
                                want_P=True)
        secs = time.perf_counter() - t0
        sample = (f"one whole {r['iter']}-iteration solve of the same {self.m}x{self.n} problem with the plan "
                  f"({threads} threads): {secs:.1f} s")
        return secs, threads, sample

    def reference_iters(self):
        """Iteration count of the full solve (run by the CPU port once, cached)."""
        import oracle
        if self.method == "vanilla":
            a, b, C = self.inputs()
            return oracle.sinkhorn_vanilla(a, b, C, self.reg, max_iter=self.max_iter, zero_tol=self.tol)["iter"]
        # the 4096^2 log solve takes ~30 s on the CPU port: its count is recorded
        # here and re-checked by tests/test_gpu_sinkhorn_log.py::test_benchmark_workload_iterations
        return {("log", 4096, 4096, 0.01): 221}.get((self.method, self.m, self.n, self.reg), self.max_iter)

    def run(self, args, dev, world, rank, clocks_cls):
        import numpy as np
        import torch

        import rwig_b200 as rw
        from rwig_b200 import _lib
        m, n = self.m, self.n
        a, b, C = self.inputs()
        ta, tb = torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)
        tC = torch.from_numpy(C.T).to(dev)  # column-major m x n as a contiguous (n, m) block
        P = torch.empty((n, m), dtype=torch.float64, device=dev)
        x = torch.empty(m, dtype=torch.float64, device=dev)
        y = torch.empty(n, dtype=torch.float64, device=dev)
        flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > L2
        stream = torch.cuda.current_stream()
        dev_fn = rw.sinkhorn_log_device if self.method == "log" else rw.sinkhorn_vanilla_device

        def solve():
            if self.method == "log":
                return dev_fn(ta, tb, tC, self.reg, self.max_iter, self.tol, P=P, f=x, g=y, stream=stream)
            return dev_fn(ta, tb, tC, self.reg, self.max_iter, self.tol, P=P, u=x, v=y, stream=stream)

        for _ in range(args.warmup):
            flush.zero_()
            solve()
        torch.cuda.synchronize()

        def barrier():
            if world > 1:
                import torch.distributed as dist
                dist.barrier()
            torch.cuda.synchronize()

        times, reps, iters = [], [], []
        with clocks_cls(dev.index) as clocks:
            barrier()
            for _ in range(args.steps):
                flush.zero_()  # L2 flush between timed steps (outside the timed region)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                r = solve()
                e1.record(stream)
                e1.synchronize()
                times.append(e0.elapsed_time(e1))
                reps.append(rw.last_report())
                iters.append(r["iter"])
            barrier()
        tot_ms = max_over_ranks(sum(times), world, dev)
        value = args.steps * world / (tot_ms / 1e3)

        # end to end through the host-pointer C ABI, pinned host buffers
        hC = torch.from_numpy(C.T.copy()).pin_memory()
        ha, hb = torch.from_numpy(a).pin_memory(), torch.from_numpy(b).pin_memory()
        hP = torch.empty((n, m), dtype=torch.float64).pin_memory()
        hx = torch.empty(m, dtype=torch.float64).pin_memory()
        hy = torch.empty(n, dtype=torch.float64).pin_memory()
        L = _lib.load()
        fn = L.rwig_sinkhorn_log if self.method == "log" else L.rwig_sinkhorn_vanilla
        dp = ctypes.POINTER(ctypes.c_double)

        def cp(t):
            return ctypes.cast(ctypes.c_void_p(t.data_ptr()), dp)

        def host_solve():
            loss, err, it = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
            rc = fn(cp(hP), None, cp(hx), cp(hy), ctypes.byref(loss), ctypes.byref(it), ctypes.byref(err),
                    cp(ha), cp(hb), cp(hC), m, n, self.reg, 0, self.max_iter, self.tol)
            _lib.check(rc)

        host_solve()
        barrier()
        e2e_s = 0.0
        for _ in range(args.steps):
            t0 = time.perf_counter()
            host_solve()
            e2e_s += time.perf_counter() - t0
        e2e_s = max_over_ranks(e2e_s, world, dev)
        assert np.array_equal(hP.numpy(), P.cpu().numpy()), "host and device entry points disagree"
        if rank != 0:
            return None

        peak, peak_kind = measured_peaks()
        it_mean = sum(iters) / len(iters)
        kms = sum(r["kernel_ms"] for r in reps) / len(reps)
        s_ms = sum(r["sweep_ms"] for r in reps) / len(reps)
        s_it = sum(r["sweep_iters"] for r in reps) / len(reps)
        # dominant kernel: the scaled sweep kernel; algorithmic bytes = one read
        # of the m x n kernel matrix per iteration it runs
        alg_bytes = s_it * m * n * 8
        achieved = alg_bytes / (s_ms / 1e3) / 1e9 if s_ms > 0 else None
        tr = profiled_traffic(s_it) if (self.method, m, n) == ("log", 4096, 4096) else None
        roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None, "traffic": tr, "peak_source": peak_kind,
                "kernel": "scaled_kernel (Sinkhorn sweep)", "kernel_ms_per_solve": s_ms,
                "kernel_iters_per_solve": s_it, "alg_bytes_per_solve": alg_bytes,
                "all_kernels_ms_per_solve": kms}
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            secs, cores, sample = self.cpu_seconds(os.cpu_count() or 1)
            cpu = {"value": 1.0 / secs, "unit": self.unit, "cores": cores, "kind": "port", "sample": sample}
        ref_gpu = None
        if self.method == "vanilla" and world == 1:
            import oracle
            ref_gpu = reference_gpu_timing(
                lambda: oracle.ref_gpu_sinkhorn_vanilla(a, b, C, self.reg, self.max_iter, self.tol),
                lambda: rw.sinkhorn(a, b, C, {"reg": self.reg, "method": "vanilla", "max_iter": self.max_iter,
                                              "zero_tol": self.tol}),
                args.steps, "cuda_sinkhorn_vanilla (src/cuda_sinkhorn.cu:181) vs rw.sinkhorn(method='vanilla'), "
                            "host arrays in and out")
        return {"value": value, "ms_per_step": tot_ms / args.steps, "reference_gpu": ref_gpu,
                "config": {"workload": self.desc, "parallelism": f"replicas x{world}",
                           "iterations_per_solve": it_mean, "l2": "flushed between steps (256 MB write)"},
                "e2e": {"value": args.steps * world / e2e_s, "unit": self.unit,
                        "h2d_bytes_per_step": (m * n + m + n) * 8, "d2h_bytes_per_step": (m * n + m + n) * 8 + 8},
                "gpu_launches": sum(r["kernel_launches"] for r in reps), "roofline": roof, "cpu_baseline": cpu,
                "clocks": clocks.summary()}

    def reference(self, args):
        """Each step one whole solve on all host threads (one untimed solve first)."""
        threads = os.cpu_count() or 1
        self.cpu_seconds(threads)
        secs, cores, sample = [], 1, ""
        for _ in range(args.steps):
            s_, cores, sample = self.cpu_seconds(threads)
            secs.append(s_)
        return sum(secs), cores, sample


def measured_dgemm_tflops(dev):
    """cuBLAS FP64 GEMM throughput on this GPU (torch.matmul float64, 8192^3,
    best of 5): the denominator for the FP64 tensor-core kernels, since the
    peak file records bf16 and HBM only."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = None
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        best = ms if best is None else min(best, ms)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (best / 1e3) / 1e12


def measured_i8gemm_tops(dev):
    """cuBLASLt INT8 GEMM throughput on this GPU (torch._int_mm, int8 operands,
    int32 result, 8192^3, best of 5) in TOP/s: the denominator for the INT8
    tensor-core GEMM of the emulated FP64 products; None if torch has no
    INT8 GEMM here."""
    import torch
    n = 8192
    try:
        a = torch.randint(-128, 128, (n, n), dtype=torch.int8, device=dev)
        b = torch.randint(-128, 128, (n, n), dtype=torch.int8, device=dev)
        torch._int_mm(a, b)
        torch.cuda.synchronize()
        best = None
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            torch._int_mm(a, b)
            e1.record()
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            best = ms if best is None else min(best, ms)
    except (RuntimeError, AttributeError):
        return None
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (best / 1e3) / 1e12


class BarycenterWorkload:
    """One log-barycenter solve with its gradient per step (fixed L iterations)."""

    higher_is_better = True

    def __init__(self, n=2048, S=32, dim=50, reg=0.05, L=50):
        self.n, self.S, self.dim, self.reg, self.L = n, S, dim, reg, L
        self.unit = "solves/s"
        self.metric = f"log-barycenter + gradient solves/s (N={n}, S={S}, L={L}, FP64)"
        self.desc = (f"log-domain Wasserstein barycenter of S={S} Dirichlet(0.3) histograms on N={n} points "
                     f"~ N(0, I_{dim}), squared-Euclidean cost / max, w ~ Dirichlet(1), b_ext ~ Dirichlet(0.3), "
                     f"eps={reg:g}, L={L} unrolled iterations (max_iter={L}, zero_tol=0), outputs b, F, G, "
                     f"grad_A, grad_w, loss")

    def inputs(self):
        from rwig_b200 import synth
        return synth.barycenter_config(n=self.n, S=self.S, dim=self.dim)

    def gemm_flops(self):
        # forward: K 1, then K^T U and K V per iteration, plus the residual
        # Gram matrix; backward: K T2 at the seed step, K^T T and K T2 at the others
        n, S, L = self.n, self.S, self.L
        products = 1 + 2 * L + (2 * L - 1)
        return products * 2.0 * n * n * S + 2.0 * n * S * S

    def cpu_seconds(self, threads):
        import oracle
        A, C, w, be = self.inputs()
        t = {}
        for it in (1, 2):
            t0 = time.perf_counter()
            oracle.barycenter_log(A, C, w, be, self.reg, with_grad=True, n_threads=threads, max_iter=it,
                                  zero_tol=0.0)
            t[it] = time.perf_counter() - t0
        per = max(t[2] - t[1], 1e-9)
        fixed = max(t[1] - per, 0.0)
        secs = fixed + self.L * per
        sample = (f"1- and 2-iteration runs (forward + backward, {threads} threads) of the same problem, "
                  f"extrapolated to L={self.L}: {per:.2f} s per iteration, {fixed:.2f} s fixed")
        return secs, threads, sample

    def run(self, args, dev, world, rank, clocks_cls):
        import torch

        import rwig_b200 as rw
        from rwig_b200 import _lib
        n, S = self.n, self.S
        A, C, w, be = self.inputs()
        tA = torch.from_numpy(np.ascontiguousarray(A.T)).to(dev)
        tC = torch.from_numpy(np.ascontiguousarray(C.T)).to(dev)
        tw, tbe = torch.from_numpy(w).to(dev), torch.from_numpy(be).to(dev)
        F = torch.empty((S, n), dtype=torch.float64, device=dev)
        G = torch.empty((S, n), dtype=torch.float64, device=dev)
        b = torch.empty(n, dtype=torch.float64, device=dev)
        gA = torch.empty((S, n), dtype=torch.float64, device=dev)
        gw = torch.empty(S, dtype=torch.float64, device=dev)
        flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
        stream = torch.cuda.current_stream()
        L = _lib.load()
        vp = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731

        def solve():
            loss, err, it = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
            rc = L.rwig_barycenter_log_dev(vp(F), vp(G), vp(b), vp(gA), vp(gw), ctypes.byref(loss), ctypes.byref(it),
                                           ctypes.byref(err), vp(tA), vp(tw), vp(tC), vp(tbe), n, n, S, self.reg, 1,
                                           self.L, 0.0, ctypes.c_void_p(stream.cuda_stream))
            _lib.check(rc)
            return rw.last_report()

        for _ in range(args.warmup):
            flush.zero_()
            solve()
        torch.cuda.synchronize()
        times, reps = [], []
        with clocks_cls(dev.index) as clocks:
            if world > 1:
                import torch.distributed as dist
                dist.barrier()
            torch.cuda.synchronize()
            for _ in range(args.steps):
                flush.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                reps.append(solve())
                e1.record(stream)
                e1.synchronize()
                times.append(e0.elapsed_time(e1))
            torch.cuda.synchronize()
        tot_ms = max_over_ranks(sum(times), world, dev)

        # end to end through the host-pointer entry
        hA = np.asfortranarray(A)
        hC = np.asfortranarray(C)
        hF, hG = np.zeros((n, S), order="F"), np.zeros((n, S), order="F")
        hb, hgA, hgw = np.zeros(n), np.zeros((n, S), order="F"), np.zeros(S)
        dp = lambda x: x.ctypes.data_as(ctypes.POINTER(ctypes.c_double))  # noqa: E731

        def host_solve():
            loss, err, it = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
            _lib.check(L.rwig_barycenter_log(dp(hF), dp(hG), dp(hb), dp(hgA), dp(hgw), ctypes.byref(loss),
                                             ctypes.byref(it), ctypes.byref(err), dp(hA), dp(w), dp(hC), dp(be), n, n,
                                             S, self.reg, 1, self.L, 0.0))

        for _ in range(2):
            host_solve()
        e2e_s = 0.0
        for _ in range(args.steps):
            t0 = time.perf_counter()
            host_solve()
            e2e_s += time.perf_counter() - t0
        e2e_s = max_over_ranks(e2e_s, world, dev)
        assert np.array_equal(hgw, gw.cpu().numpy()), "host and device entry points disagree"
        if rank != 0:
            return None
        tf_peak = measured_dgemm_tflops(dev)
        kms = sum(r["kernel_ms"] for r in reps) / len(reps)
        achieved = self.gemm_flops() / (kms / 1e3) / 1e12
        roof = {"bound": "tensor", "achieved": achieved, "peak": tf_peak, "unit": "TFLOP/s",
                "frac": achieved / tf_peak, "traffic": None,
                "peak_source": "measured cuBLAS FP64 GEMM (torch.matmul float64 8192^3) on this GPU",
                "kernel": "dgemm_kernel with fused epilogues (whole solve, device time)",
                "flops_per_solve": self.gemm_flops(), "ms_per_solve": kms}
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            secs, cores, sample = self.cpu_seconds(os.cpu_count() or 1)
            cpu = {"value": 1.0 / secs, "unit": self.unit, "cores": cores, "kind": "port", "sample": sample}
        MS, NN = n * S * 8, n * n * 8
        ref_gpu = None
        if world == 1:
            import oracle
            ref_gpu = reference_gpu_timing(
                lambda: oracle.ref_gpu_barycenter_parallel(A, C, w, be, reg=self.reg, with_grad=True,
                                                          max_iter=self.L, zero_tol=0.0),
                lambda: rw.barycenter(A, C, w, be, {"reg": self.reg, "method": "parallel", "with_grad": True,
                                                    "max_iter": self.L, "zero_tol": 0.0}),
                args.steps, "parallel barycenter + gradient on this workload's inputs (the reference has no GPU log "
                            "barycenter): cuda_barycenter_parallel (src/cuda_barycenter.cu:268) vs "
                            "rw.barycenter(method='parallel'), host arrays")
        batch = self.batch_timing(dev)
        return {"value": args.steps * world / (tot_ms / 1e3), "ms_per_step": tot_ms / args.steps,
                "reference_gpu": ref_gpu, "batch": batch,
                "config": {"workload": self.desc, "parallelism": f"replicas x{world}",
                           "l2": "flushed between steps (256 MB write)"},
                "e2e": {"value": args.steps * world / e2e_s, "unit": self.unit,
                        "h2d_bytes_per_step": MS + NN + (S + n) * 8, "d2h_bytes_per_step": 3 * MS + (n + S) * 8},
                "gpu_launches": sum(r["kernel_launches"] for r in reps), "roofline": roof, "cpu_baseline": cpu,
                "clocks": clocks.summary()}

    def batch_timing(self, dev):
        """16 log barycenters with gradient of uneven sizes (N in {256, 512,
        1024, 2048} x S in {4, 8, 16, 32}, L = 50, fixed iteration count) on
        device buffers: one rwig_batch_barycenter_dev call against 16
        rwig_barycenter_log_dev calls on the same stream, each the median of
        3 rounds timed with CUDA events; results compared bitwise."""
        import torch

        from rwig_b200 import _lib, synth
        L = _lib.load()
        stream = torch.cuda.current_stream()
        sp = ctypes.c_void_p(stream.cuda_stream)
        vp = lambda t: ctypes.c_void_p(t.data_ptr()) if t is not None else None  # noqa: E731
        shapes = [(nn, ss) for nn in (256, 512, 1024, 2048) for ss in (4, 8, 16, 32)]
        keep = []
        arr = (_lib.BaryProblem * len(shapes))()
        res = (_lib.BaryResult * len(shapes))()
        for i, (nn, ss) in enumerate(shapes):
            A, C, w, be = synth.barycenter_config(n=nn, S=ss, dim=10, salt=50 + i)
            t = [torch.from_numpy(np.ascontiguousarray(x)).to(dev) for x in (A.T, C.T, w, be)]
            outs = [torch.empty(ss * nn, dtype=torch.float64, device=dev) for _ in range(3)] + \
                   [torch.empty(nn, dtype=torch.float64, device=dev), torch.empty(ss, dtype=torch.float64, device=dev)]
            keep.append((t, outs, nn, ss))
            arr[i] = _lib.BaryProblem(vp(t[0]), vp(t[2]), vp(t[1]), vp(t[3]), nn, nn, ss, self.reg, 1, 1, self.L, 0.0,
                                      vp(outs[0]), vp(outs[1]), vp(outs[3]), vp(outs[2]), vp(outs[4]))

        def batched():
            _lib.check(L.rwig_batch_barycenter_dev(arr, len(shapes), res, sp))

        loss, err, it = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()

        def one_by_one():
            for (t, outs, nn, ss) in keep:
                _lib.check(L.rwig_barycenter_log_dev(vp(outs[0]), vp(outs[1]), vp(outs[3]), vp(outs[2]), vp(outs[4]),
                                                     ctypes.byref(loss), ctypes.byref(it), ctypes.byref(err),
                                                     vp(t[0]), vp(t[2]), vp(t[1]), vp(t[3]), nn, nn, ss, self.reg, 1,
                                                     self.L, 0.0, sp))

        def timed(fn):
            fn()
            ts = []
            for _ in range(3):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                e0.record(stream)
                fn()
                e1.record(stream)
                e1.synchronize()
                ts.append(e0.elapsed_time(e1))
            return float(np.median(ts))

        b_ms = timed(batched)
        bref = [[o.clone() for o in outs] for (_, outs, _, _) in keep]
        s_ms = timed(one_by_one)
        same = all(torch.equal(a, b) for (_, outs, _, _), br in zip(keep, bref) for a, b in zip(outs, br))
        n = len(shapes)
        return {"problems": n, "shapes": "N in {256, 512, 1024, 2048} x S in {4, 8, 16, 32}, log, gradient, L = 50",
                "batched_solves_per_s": n / (b_ms / 1e3), "one_by_one_solves_per_s": n / (s_ms / 1e3),
                "speedup": s_ms / b_ms, "bitwise_equal": bool(same)}

    def reference(self, args):
        threads = os.cpu_count() or 1
        secs, sample = [], ""
        for _ in range(args.steps):
            s_, cores, sample = self.cpu_seconds(threads)
            secs.append(s_)
        return sum(secs), threads, sample


class WdlWorkload:
    """WDL training steps (one batch each: batched barycenter forward, adjoint,
    softmax Jacobians, Adam update, softmax)."""

    higher_is_better = True

    def __init__(self, V=5000, M=2048, S=16, dim=64, B=64, reg=0.05, L=20, lr=1e-3):
        self.V, self.M, self.S, self.dim, self.B, self.reg, self.L, self.lr = V, M, S, dim, B, reg, L, lr
        self.unit = "steps/s"
        self.metric = f"WDL training steps/s (V={V}, M={M}, K={S} topics, batch {B}, L={L}, Adam, FP64)"
        self.desc = (f"WDL training: V={V} vocabulary embeddings ~ N(0, I_{dim}), squared-Euclidean cost / max; "
                     f"M={M} documents of U{{20..200}} Zipf(1.1) tokens as normalised counts; K={S} topics with "
                     f"N(0, 0.01) logits; batch {B}, eps={reg:g}, L={L} unrolled parallel-barycenter iterations, "
                     f"quadratic loss, Adam lr={lr:g} (0.9, 0.999, 1e-8)")
        self._data = None

    def data(self):
        if self._data is None:
            from rwig_b200 import synth
            self._data = synth.wdl_config(V=self.V, M=self.M, S=self.S, dim=self.dim)
        return self._data

    def products(self):
        return 2 * self.L + 2 * self.L - 1  # forward K V, K^T U per iteration; backward K T2, K^T T

    def step_flops(self):
        return self.products() * 2.0 * self.V * self.V * self.S * self.B

    def cpu_seconds(self, threads):
        """Oracle batched gradient on a bounded sample (one document, L = 1:
        three products of width S), scaled by FLOPs to one full step."""
        import oracle
        Y, C, A0, L0 = self.data()
        K = np.asfortranarray(np.exp(-C / self.reg))
        A = oracle.col_softmax(A0)
        W = oracle.col_softmax(L0)
        t0 = time.perf_counter()
        oracle.wdl_batch_grad(A, W[:, :1], Y[:, :1], K, 1)
        dt = time.perf_counter() - t0
        scale = self.step_flops() / (3 * 2.0 * self.V * self.V * self.S)
        sample = (f"oracle batched gradient of 1 document at L=1 (3 products of width {self.S}, 1 thread): "
                  f"{dt:.2f} s, scaled by FLOPs x{scale:.0f} to one {self.B}-document L={self.L} step")
        return dt * scale, 1, sample

    def run(self, args, dev, world, rank, clocks_cls):
        import torch

        import rwig_b200 as rw
        from rwig_b200 import _lib
        Y, C, A0, L0 = self.data()
        L = _lib.load()
        N, M, S = self.V, self.M, self.S
        A = np.zeros((N, S), order="F")
        W = np.zeros((S, M), order="F")
        dp = lambda x: x.ctypes.data_as(ctypes.POINTER(ctypes.c_double))  # noqa: E731

        def train(steps):
            rc = L.rwig_wdl(dp(A), dp(W), None, dp(Y), dp(C), N, M, S, self.reg, self.L, 1e-6, self.B, 1000, 1,
                            self.lr, 0.01, 0.9, 0.999, 1e-8, 42, 0, dp(A0), dp(L0), int(steps))
            _lib.check(rc)
            return rw.last_report()

        train(args.warmup)
        torch.cuda.synchronize()
        with clocks_cls(dev.index) as clocks:
            if world > 1:
                import torch.distributed as dist
                dist.barrier()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            rep = train(args.steps)
            wall = time.perf_counter() - t0
            torch.cuda.synchronize()
        dev_ms = max_over_ranks(rep["device_ms"], world, dev)
        wall = max_over_ranks(wall, world, dev)
        # inference: every document's parallel barycenter (max_iter = L,
        # zero_tol 1e-6, per-document stop) under the initial topics, one
        # rwig_wdl call with no training epoch (host buffers, copies and K included)
        Yh = np.zeros((N, M), order="F")
        t0 = time.perf_counter()
        _lib.check(L.rwig_wdl(dp(A), dp(W), dp(Yh), dp(Y), dp(C), N, M, S, self.reg, self.L, 1e-6, self.B, 0, 1,
                              self.lr, 0.01, 0.9, 0.999, 1e-8, 42, 0, dp(A0), dp(L0), 0))
        inf_s = time.perf_counter() - t0
        infer = {"docs": M, "seconds": inf_s, "docs_per_s": M / inf_s, "max_iter": self.L, "zero_tol": 1e-6,
                 "call": "rwig_wdl with no training epoch: all documents in stacked columns, per-document stop"}
        if rank != 0:
            return None
        tf_peak = measured_dgemm_tflops(dev)
        achieved = self.step_flops() * args.steps / (dev_ms / 1e3) / 1e12
        roof = {"bound": "tensor", "achieved": achieved, "peak": tf_peak, "unit": "TFLOP/s",
                "frac": achieved / tf_peak, "traffic": None,
                "peak_source": "measured cuBLAS FP64 GEMM (torch.matmul float64 8192^3) on this GPU",
                "kernel": "the whole step (device time): products emulated on the INT8 tensor cores "
                          "(i8_gemm, res_cols, crt_tiles with fused WDL epilogues)",
                "note": "FP64-equivalent rate: the step's products counted as FP64 GEMM flops over the FP64 "
                        "tensor-core peak; frac > 1 means faster than any FP64 tensor-core step",
                "flops_per_step": self.step_flops(), "products_per_step": self.products()}
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            secs, cores, sample = self.cpu_seconds(1)
            cpu = {"value": 1.0 / secs, "unit": self.unit, "cores": cores, "kind": "port", "sample": sample}
        return {"value": args.steps * world / (dev_ms / 1e3), "ms_per_step": dev_ms / args.steps,
                "config": {"workload": self.desc, "parallelism": f"replicas x{world}",
                           "timing": "device events inside rwig_wdl around the training steps",
                           "l2": "inputs larger than L2 (K = 200 MB)"},
                "e2e": {"value": args.steps * world / wall, "unit": self.unit,
                        "h2d_bytes_per_step": (N * M + N * N + N * S + S * M) * 8 / args.steps,
                        "d2h_bytes_per_step": (N * S + S * M) * 8 / args.steps,
                        "note": "one rwig_wdl call with host buffers (copies, K, training) over all steps"},
                "gpu_launches": rep["kernel_launches"], "roofline": roof, "cpu_baseline": cpu,
                "inference": infer, "clocks": clocks.summary()}

    def reference(self, args):
        secs, sample, cores = [], "", 1
        for _ in range(args.steps):
            s_, cores, sample = self.cpu_seconds(1)
            secs.append(s_)
        return sum(secs), cores, sample


def device_cost(x, y, dev):
    """sq_euclid_cost(x, y) built on the device (same elementwise operations in
    the same order, so the same bits): an (n, m) tensor holding C column-major."""
    import torch
    tx = torch.from_numpy(np.ascontiguousarray(x)).to(dev)
    ty = torch.from_numpy(np.ascontiguousarray(y)).to(dev)
    C = torch.zeros((ty.shape[0], tx.shape[0]), dtype=torch.float64, device=dev)
    for k in range(tx.shape[1]):
        d = tx[None, :, k] - ty[:, k, None]
        C += d * d
    C /= C.max()
    return C


class StreamWorkload:
    """The serving stream of mixed-size log-Sinkhorn requests (the headline).

    One step = one batched call (rwig_batch_sinkhorn_log_dev) over the whole
    200-request stream with device-resident inputs; `value` = requests solved
    per second over the K timed calls.  Beside it on the same line: the plain
    per-call path (one rwig_sinkhorn_log_dev call per request), the end-to-end
    batched call with pinned host buffers, the continuous-batching server's
    p50/p99 latency under Poisson arrivals, the autotuned batched call, and the
    WDL training step (engine vs the reference's own unrolled GPU step)."""

    higher_is_better = True

    def __init__(self, R=200, max_iter=2000, tol=1e-9):
        self.R, self.max_iter, self.tol = R, max_iter, tol
        self.unit = "solves/s"
        self.metric = "batched vs plain solves/s, p50/p99 latency @err<1e-10 FP64; WDL steps/s"
        self.desc = (f"{R} log-Sinkhorn requests: n, m log-uniform in [64, 8192], eps from {{0.01, 0.05, 0.1}}, "
                     f"Dirichlet(1) histograms, points uniform in [0,1]^d with d from {{2, 3, 64}}, "
                     f"squared-Euclidean cost / max, tol {tol:g}, max_iter {max_iter}, outputs f, g, loss")

    def config(self, world):
        """The same dict on the engine and the reference arm."""
        from rwig_b200 import synth
        gb = sum(q["m"] * q["n"] for q in synth.stream_requests(self.R)) * 8 / 1e9
        return {"workload": self.desc, "parallelism": f"replicas x{world}",
                "step": f"one batched call over the whole {self.R}-request stream (value counts requests)",
                "l2": f"no flush: the stream's cost matrices ({gb:.1f} GB) exceed L2"}

    def build(self, dev):
        import torch
        from rwig_b200 import synth
        reqs = synth.stream_requests(self.R)
        data = []
        for q in reqs:
            a, b, x, y = synth.stream_request_data(q["m"], q["n"], q["d"], q["salt"])
            C = device_cost(x, y, dev)
            data.append({"q": q, "a": torch.from_numpy(a).to(dev), "b": torch.from_numpy(b).to(dev), "C": C,
                         "f": torch.empty(q["m"], dtype=torch.float64, device=dev),
                         "g": torch.empty(q["n"], dtype=torch.float64, device=dev),
                         "ha": a, "hb": b})
        return data

    def problems(self, data, rng_idx=None):
        from rwig_b200 import _lib
        idx = list(range(len(data))) if rng_idx is None else rng_idx
        arr = (_lib.Problem * len(idx))()
        vp = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
        for k, i in enumerate(idx):
            d = data[i]
            arr[k] = _lib.Problem(vp(d["a"]), vp(d["b"]), vp(d["C"]), d["q"]["m"], d["q"]["n"], d["q"]["eps"],
                                  self.max_iter, self.tol, None, vp(d["f"]), vp(d["g"]))
        return arr

    def run(self, args, dev, world, rank, clocks_cls):
        import torch

        import rwig_b200 as rw
        from rwig_b200 import _lib
        L = _lib.load()
        data = self.build(dev)
        R = len(data)
        stream = torch.cuda.current_stream()
        sp = ctypes.c_void_p(stream.cuda_stream)
        probs = self.problems(data)
        res = (_lib.Result * R)()
        # warm-up: whole batched calls (the first sizes the engine's scratch arena)
        for _ in range(max(1, args.warmup)):
            _lib.check(L.rwig_batch_sinkhorn_log_dev(probs, R, res, sp))
        torch.cuda.synchronize()
        launches = 0
        with clocks_cls(dev.index) as clocks:
            if world > 1:
                import torch.distributed as dist
                dist.barrier()
            torch.cuda.synchronize()
            evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                   for _ in range(args.steps)]
            for e0, e1 in evs:
                e0.record(stream)
                _lib.check(L.rwig_batch_sinkhorn_log_dev(probs, R, res, sp))
                e1.record(stream)
                launches += rw.last_report()["kernel_launches"]
            torch.cuda.synchronize()
            step_ms = [e0.elapsed_time(e1) for e0, e1 in evs]
        total_ms = max_over_ranks(sum(step_ms), world, dev)
        batch_ms = total_ms / args.steps
        bres = [res[i].as_dict() for i in range(R)]
        bf = [d["f"].cpu().numpy() for d in data]
        # the per-call path on the same inputs; one untimed pass first sizes its
        # scratch arena, as the batched warm-up does for the batched call
        vp = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
        loss, err, it = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()

        def per_call_pass():
            its = []
            for d in data:
                q = d["q"]
                _lib.check(L.rwig_sinkhorn_log_dev(None, None, vp(d["f"]), vp(d["g"]), ctypes.byref(loss),
                                                   ctypes.byref(it), ctypes.byref(err), vp(d["a"]), vp(d["b"]),
                                                   vp(d["C"]), q["m"], q["n"], q["eps"], 0, self.max_iter,
                                                   self.tol, sp))
                its.append(it.value)
            return its

        per_call_pass()
        torch.cuda.synchronize()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        piters = per_call_pass()
        p1.record(stream)
        p1.synchronize()
        plain_ms = p0.elapsed_time(p1)
        # agreement of the two paths (same iteration counts, potentials to 1e-10)
        worst = 0.0
        for i, d in enumerate(data):
            assert bres[i]["iter"] == piters[i], (i, bres[i]["iter"], piters[i])
            pf = d["f"].cpu().numpy()
            worst = max(worst, float(np.abs(bf[i] - pf).max() / max(np.abs(pf).max(), 1e-300)))
        assert worst <= 1e-10, worst
        # end to end: pinned host inputs through rwig_batch_sinkhorn_log (copies in and out every call)
        hC, harr, keep = [], (_lib.Problem * R)(), []
        for i, d in enumerate(data):
            q = d["q"]
            pc = torch.empty(d["C"].shape, dtype=torch.float64, pin_memory=True)
            pc.copy_(d["C"])
            ha = torch.from_numpy(d["ha"]).pin_memory()
            hb = torch.from_numpy(d["hb"]).pin_memory()
            f = torch.zeros(q["m"], dtype=torch.float64, pin_memory=True)
            g = torch.zeros(q["n"], dtype=torch.float64, pin_memory=True)
            keep.append((pc, ha, hb, f, g))
            hC.append(pc.numpy())  # (n, m) row-major = column-major m x n
            hp = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
            harr[i] = _lib.Problem(hp(ha), hp(hb), hp(pc), q["m"], q["n"], q["eps"], self.max_iter, self.tol, None,
                                   hp(f), hp(g))
        n_e2e = max(1, min(args.steps, 3))
        _lib.check(L.rwig_batch_sinkhorn_log(harr, R, res))
        t0 = time.perf_counter()
        for _ in range(n_e2e):
            _lib.check(L.rwig_batch_sinkhorn_log(harr, R, res))
        e2e_s = max_over_ranks((time.perf_counter() - t0) / n_e2e, world, dev)
        serving = self.serve(data, hC, R / (batch_ms / 1e3), args.serve_requests)
        tuned = None if args.no_autotune else self.autotuned(data, hC, probs, res, sp, stream)
        wdl = None if args.no_wdl else self.wdl_block(args, dev)
        if rank != 0:
            return None
        hbm, src = measured_peaks()
        elems = [d["q"]["m"] * d["q"]["n"] for d in data]
        alg = sum((bres[i]["iter"] + 2) * elems[i] * 8.0 for i in range(R))
        achieved = alg / (batch_ms / 1e3) / 1e9
        # DRAM bytes of one service_kernel launch over this stream, from a single-pass
        # ncu capture (dram__bytes_read.sum + dram__bytes_write.sum) of
        # `bench.py --single --workload stream --stream-profile`: 297.99 GB read, 7.51 GB
        # written in 119.94 ms (the stream and its iteration counts are deterministic)
        traffic = 297.99e9 + 7.51e9
        roof = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                "traffic": traffic, "traffic_unit": "bytes per launch (ncu, one capture)",
                "dram_gbs_in_capture": traffic / 119.94e-3 / 1e9, "peak_source": src,
                "kernel": "service_kernel (a team of CTAs per problem), whole batched call",
                "alg_bytes_per_step": alg,
                "note": "K read once per iteration plus the K build and final passes per request; strips of "
                        "small problems stay in shared memory or L2, so this is the stream's effective rate"}
        in_kernel = sum(1 for r in bres if r["path"] == 0)
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            cpu = self.cpu_baseline(budget_s=15.0)
        cfg = self.config(world)
        cfg["requests_in_batched_kernel"] = in_kernel
        return {"value": R * args.steps * world / (total_ms / 1e3), "ms_per_step": batch_ms,
                "config": cfg,
                "plain": {"value": R / (plain_ms / 1e3), "unit": self.unit,
                          "path": "one rwig_sinkhorn_log_dev call per request, device-resident inputs",
                          "speedup_batched_over_plain": plain_ms / batch_ms,
                          "max_rel_diff_f_vs_batched": worst, "iterations_equal": True},
                "e2e": {"value": R / e2e_s, "unit": self.unit,
                        "h2d_bytes_per_step": sum((e + d["q"]["m"] + d["q"]["n"]) * 8 for e, d in zip(elems, data)),
                        "d2h_bytes_per_step": sum((d["q"]["m"] + d["q"]["n"]) * 8 + 16 * 8 for d in data),
                        "call": f"rwig_batch_sinkhorn_log on pinned host buffers, mean of {n_e2e} calls"},
                "latency": serving, "autotuned": tuned, "wdl": wdl,
                "gpu_launches": launches, "roofline": roof, "cpu_baseline": cpu, "clocks": clocks.summary()}

    def autotuned(self, data, hC, probs, res, sp, stream):
        """The batch.* options tuned on this stream by rwig_b200.autotune
        (coordinate search, every trial checked against the starting
        setting's iteration counts and losses), then the whole batched call
        timed again under them; the options are cleared afterwards."""
        import torch

        import rwig_b200 as rw
        from rwig_b200 import _lib
        from rwig_b200.autotune import OPTIONS
        L = _lib.load()
        R = len(data)
        qs = [{"a": d["ha"], "b": d["hb"], "C": hC[i].T, "reg": d["q"]["eps"], "max_iter": self.max_iter,
               "zero_tol": self.tol} for i, d in enumerate(data)]
        t0 = time.perf_counter()
        r = rw.autotune_batch(qs)
        tune_s = time.perf_counter() - t0
        del qs
        try:
            _lib.check(L.rwig_batch_sinkhorn_log_dev(probs, R, res, sp))
            ts = []
            for _ in range(3):  # median of three batched calls
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                e0.record(stream)
                _lib.check(L.rwig_batch_sinkhorn_log_dev(probs, R, res, sp))
                e1.record(stream)
                e1.synchronize()
                ts.append(e0.elapsed_time(e1))
            ms = float(np.median(ts))
        finally:
            for n in OPTIONS:
                L.rwig_set_option(n.encode(), float("nan"))
        return {"value": R / (ms / 1e3), "unit": self.unit, "options": r["options"],
                "search_speedup": r["speedup"], "trials": len(r["trials"]), "rejected": len(r["rejected"]),
                "tuning_seconds": tune_s}

    def serve(self, data, hC, capacity, n_req=20000):
        """The continuous-batching server (rwig_server_*, point-cloud requests,
        cost built on the device) in real time on n_req requests that cycle
        through the stream's distinct requests: first its capacity (2000 of
        them submitted at once), then Poisson arrivals (seeded unit-rate
        exponential gaps) at 50 %, 80 % and 100 % of that capacity; beside it
        the per-call path (rwig_sinkhorn_log, host buffers) as a FIFO queue of
        its measured service times under the same arrivals.  Latency =
        completion - arrival."""
        import rwig_b200 as rw
        from rwig_b200 import synth
        R = len(data)
        reqs = [(d["ha"], d["hb"], hC[i].T, d["q"]["eps"]) for i, d in enumerate(data)]
        pts = []
        for d in data:
            q = d["q"]
            _, _, x, y = synth.stream_request_data(q["m"], q["n"], q["d"], q["salt"])
            pts.append((np.asfortranarray(x), np.asfortranarray(y)))
        n_req = max(R, int(n_req))
        gaps = np.random.default_rng(2024).exponential(1.0, n_req)

        def run_server(arrivals):
            n = len(arrivals)
            lat = np.zeros(n)
            with rw.Server(mem_budget_bytes=64e9, idle_ms=200.0) as srv:
                pending, idx, done = {}, 0, 0
                t0 = time.perf_counter()
                while done < n:
                    now = time.perf_counter() - t0
                    while idx < n and arrivals[idx] <= now:
                        a, b, _, eps = reqs[idx % R]
                        t = srv.submit(a, b, None, eps, self.max_iter, self.tol, x=pts[idx % R][0],
                                       y=pts[idx % R][1])
                        if t is None:
                            break
                        pending[t] = idx
                        idx += 1
                    for t in list(pending):
                        if srv.poll(t) is not None:
                            i = pending.pop(t)
                            lat[i] = time.perf_counter() - t0 - arrivals[i]
                            done += 1
                span = time.perf_counter() - t0 - arrivals[0]
            return lat, span

        run_server(np.zeros(R))  # warm-up
        n_cap = min(n_req, 2000)
        _, span_all = run_server(np.zeros(n_cap))
        cap = n_cap / span_all
        svc = np.zeros(R)
        for i, (a, b, C, eps) in enumerate(reqs):
            t1 = time.perf_counter()
            rw.sinkhorn(a, b, C, {"reg": eps, "method": "log", "max_iter": self.max_iter, "zero_tol": self.tol})
            svc[i] = time.perf_counter() - t1
        ms = lambda x, q: float(np.percentile(x, q) * 1e3)  # noqa: E731
        out = {"server_capacity_per_s": cap, "requests_per_rate": n_req, "distinct_requests": R,
               "capacity": f"{n_cap} requests submitted at once in the stream's order",
               "arrivals": "Poisson (seeded unit-rate exponential gaps / rate)",
               "requests": "server: histograms + point clouds (cost built on the device); per call: histograms + "
                           "host cost matrix",
               "per_call_mean_service_ms": float(svc.mean() * 1e3)}
        for frac in (0.5, 0.8, 1.0):
            rate = frac * cap
            arrivals = np.cumsum(gaps) / rate
            arrivals -= arrivals[0]
            lat, span = run_server(arrivals)
            fin, plat = 0.0, np.zeros(n_req)
            for i in range(n_req):
                fin = max(fin, arrivals[i]) + svc[i % R]
                plat[i] = fin - arrivals[i]
            out[f"at_{int(frac * 100)}pct"] = {
                "arrival_rate_per_s": rate,
                "server": {"solves_per_s": n_req / span, "p50_ms": ms(lat, 50), "p99_ms": ms(lat, 99)},
                "per_call_fifo": {"solves_per_s": n_req / (fin - arrivals[0]), "p50_ms": ms(plat, 50),
                                  "p99_ms": ms(plat, 99)}}
        return out

    def wdl_block(self, args, dev):
        """The WDL training workload (V = 5000, K = 16 topics, batch 64, L = 20,
        Adam) beside the stream: engine training steps through rwig_wdl (device
        time inside the call), and one batched adjoint step -- the engine's
        rwig_wdl_batch_grad_dev against the reference's own unrolled GPU step
        (wdl_batch, src/cuda_wdl.cu:385, compiled from its sources into
        oracle/_ref) on the same device-resident batch, both timed with CUDA
        events, their gradients compared."""
        import torch

        import oracle
        import rwig_b200 as rw
        from rwig_b200 import _lib
        wl = WdlWorkload()
        Y, C, A0, L0 = wl.data()
        L = _lib.load()
        N, M, S, B = wl.V, wl.M, wl.S, wl.B
        A = np.zeros((N, S), order="F")
        W = np.zeros((S, M), order="F")
        dp = lambda x: x.ctypes.data_as(ctypes.POINTER(ctypes.c_double))  # noqa: E731
        steps, warm = 6, 2

        def train(k):
            _lib.check(L.rwig_wdl(dp(A), dp(W), None, dp(Y), dp(C), N, M, S, wl.reg, wl.L, 1e-6, B, 1000, 1,
                                  wl.lr, 0.01, 0.9, 0.999, 1e-8, 42, 0, dp(A0), dp(L0), int(k)))
            return rw.last_report()

        train(warm)
        rep = train(steps)
        tf_peak = measured_dgemm_tflops(dev)
        achieved = wl.step_flops() * steps / (rep["device_ms"] / 1e3) / 1e12
        out = {"workload": wl.desc, "steps_per_s": steps / (rep["device_ms"] / 1e3), "unit": "steps/s",
               "steps_timed": steps, "ms_per_step": rep["device_ms"] / steps,
               "roofline": {"bound": "tensor", "achieved": achieved, "peak": tf_peak, "unit": "TFLOP/s",
                            "frac": achieved / tf_peak, "flops_per_step": wl.step_flops(),
                            "peak_source": "measured cuBLAS FP64 GEMM (torch.matmul float64 8192^3) on this GPU",
                            "note": "FP64-equivalent rate: the step's products counted as FP64 GEMM flops over "
                                    "the FP64 tensor-core peak; the products run emulated on the INT8 tensor "
                                    "cores, so frac > 1 means faster than any FP64 tensor-core step"},
               "gpu_launches_per_step": rep["kernel_launches"] / steps}
        # one batched adjoint step on batch 0, device-resident K: engine vs the reference's wdl_batch
        Ah = oracle.col_softmax(A0)
        Wh = oracle.col_softmax(L0)[:, :B].copy(order="F")
        Yb = np.asfortranarray(Y[:, :B])
        K = np.asfortranarray(np.exp(-C / wl.reg))
        t = lambda x: torch.from_numpy(np.ascontiguousarray(x.T)).to(dev)  # noqa: E731  column-major on device
        dA, dW, dY, dK = t(Ah), t(Wh), t(Yb), t(K)
        gA = torch.empty((S, N), dtype=torch.float64, device=dev)
        gl = torch.empty(S, dtype=torch.float64, device=dev)
        stream = torch.cuda.current_stream()
        vp = lambda x: ctypes.c_void_p(x.data_ptr())  # noqa: E731

        def engine_step():
            _lib.check(L.rwig_wdl_batch_grad_dev(vp(gA), vp(gl), vp(dA), vp(dW), vp(dY), vp(dK), N, S, B, wl.reg,
                                                 wl.L, 0, ctypes.c_void_p(stream.cuda_stream)))

        def timed_step():
            engine_step()
            ts = []
            for _ in range(3):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                engine_step()
                e1.record(stream)
                e1.synchronize()
                ts.append(e0.elapsed_time(e1))
            return float(np.mean(ts))

        L.rwig_set_option(b"wdl.int8", 0.0)  # the same step with every product on the FP64 tensor cores
        try:
            dmma_ms = timed_step()
            dmma_gA = gA.cpu().numpy()
        finally:
            L.rwig_set_option(b"wdl.int8", float("nan"))
        eng_ms = timed_step()
        full_gA = gA.cpu().numpy()
        adj = {"batch": f"batch 0: {B} documents, K given (mode 0)", "engine_ms": eng_ms,
               "engine_call": "rwig_wdl_batch_grad_dev, mean of 3 after 1 untimed; products emulated on the "
                              "INT8 tensor cores (wdl.int8 default)",
               "engine_fp64_tensor_ms": dmma_ms,
               "max_rel_diff_int8_vs_fp64_tensor": float(np.abs(full_gA - dmma_gA).max() / np.abs(dmma_gA).max())}
        # the INT8 GEMM launches of one adjoint step, each bracketed by CUDA events
        # in the engine (option profile.gemm), against cuBLASLt's INT8 GEMM
        L.rwig_set_option(b"profile.gemm", 1.0)
        try:
            engine_step()
            torch.cuda.synchronize()
            grep = rw.last_report()
        finally:
            L.rwig_set_option(b"profile.gemm", float("nan"))
        i8_peak = measured_i8gemm_tops(dev)
        if grep["gemm_launches"] > 0:
            ops = 24.0 * wl.step_flops()  # 24 residue planes per emulated FP64 product, unpadded sizes
            ach = ops / (grep["gemm_ms"] / 1e3) / 1e12
            adj["int8_gemm_roofline"] = {
                "kernel": "i8_gemm (ozaki.cu)", "bound": "tensor", "launches": grep["gemm_launches"],
                "ms_per_launch": grep["gemm_ms"] / grep["gemm_launches"], "share_of_step": grep["gemm_ms"] / eng_ms,
                "achieved": ach, "unit": "TOP/s", "peak": i8_peak,
                "frac": (ach / i8_peak) if i8_peak else None,
                "ops_per_launch": ops / grep["gemm_launches"],
                "peak_source": "measured cuBLASLt INT8 GEMM (torch._int_mm 8192^3) on this GPU; nominal 4500 TOP/s"}
        # checkpointed adjoint (wdl.checkpoint = k): history footprint and step time
        NW, ND = N * S * B * 8, N * B * 8
        ck = {}
        for kk in (wl.L, 5, 4, 1):
            L.rwig_set_option(b"wdl.checkpoint", float(kk))
            try:
                ms_k = timed_step()
                same = bool(np.array_equal(gA.cpu().numpy(), full_gA))
            finally:
                L.rwig_set_option(b"wdl.checkpoint", float("nan"))
            nseg = -(-wl.L // kk)
            hist = (nseg + 4 * kk + 3) * NW + (kk + 1) * ND
            ck[f"k{kk}"] = {"ms": ms_k, "history_bytes": hist, "products": wl.products() + 2 * (wl.L - kk),
                            "gradient_bitwise_equal_to_full_history": same}
        adj["checkpointing"] = ck
        if oracle.ref_gpu_available():
            rgA, rgl, ref_ms = oracle.ref_gpu_wdl_batch_grad(Ah, Wh, Yb, K, wl.reg, wl.L, mode=0, reps=3)
            egA = gA.cpu().numpy().T
            rel = float(np.abs(egA - rgA).max() / np.abs(rgA).max())
            adj.update(reference_ms=ref_ms, speedup_engine_over_reference=ref_ms / eng_ms,
                       reference_call="wdl_batch (src/cuda_wdl.cu:385) built from the reference's sources, cuBLAS "
                                      "DGEMMs, mean of 3 calls (CUDA events on its stream)",
                       max_rel_diff_g_alpha=rel)
        out["adjoint_step"] = adj
        return out

    def _work(self, reqs, iters):
        return [(iters[i] + 2) * reqs[i]["m"] * reqs[i]["n"] for i in range(len(reqs))]

    def cpu_sample(self, budget_s=None, steps=None):
        """Whole log-Sinkhorn solves of the stream's requests by the oracle (all
        host threads), timed one by one: requests taken in the stream's order
        among those of at most 2^24 elements (each seconds, not minutes, on the
        host), until `steps` solves or `budget_s` seconds.  Returns a list of
        (seconds, element-iterations) per solve and the stream's mean
        element-iterations per request, from the per-request iteration counts
        in tests/golden/stream_iters.json (tests/golden/make_stream_iters.py)."""
        import oracle
        from rwig_b200 import synth
        path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tests", "golden", "stream_iters.json")
        with open(path) as fh:
            iters = json.load(fh)["iters"]
        reqs = synth.stream_requests(self.R)
        if len(iters) != len(reqs):
            raise RuntimeError("stream_iters.json does not match the stream")
        work = self._work(reqs, iters)
        mean_work = sum(work) / len(work)
        pick = [i for i, q in enumerate(reqs) if q["m"] * q["n"] <= (1 << 24)]
        threads = os.cpu_count() or 1
        out, k, t_all = [], 0, 0.0
        while (steps is not None and len(out) < steps) or (budget_s is not None and t_all < budget_s):
            q = reqs[pick[k % len(pick)]]
            k += 1
            a, b, x, y = synth.stream_request_data(q["m"], q["n"], q["d"], q["salt"])
            C = synth.sq_euclid_cost(x, y)
            t0 = time.perf_counter()
            r = oracle.sinkhorn_log(a, b, C, q["eps"], max_iter=self.max_iter, zero_tol=self.tol,
                                    n_threads=threads, want_P=False)
            dt = time.perf_counter() - t0
            t_all += dt
            out.append((dt, (r["iter"] + 2) * q["m"] * q["n"]))
        return out, mean_work, threads, len(pick)

    def cpu_baseline(self, budget_s=15.0):
        solves, mean_work, threads, npick = self.cpu_sample(budget_s=budget_s)
        t = sum(s for s, _ in solves)
        w = sum(x for _, x in solves)
        value = (w / mean_work) / t
        return {"value": value, "unit": self.unit, "cores": threads, "kind": "port",
                "sample": f"{len(solves)} whole solves ({t:.1f} s) of the stream's requests of <= 2^24 elements "
                          f"({npick} of {self.R}) by the oracle on {threads} threads; value = stream-mean requests "
                          f"per second, the solves' element-iterations divided by the stream's mean per request "
                          f"({mean_work:.3g})"}

    def reference(self, args):
        """--impl reference: each step one whole solve of a stream request (the
        oracle on all host threads, as cpu_sample); value in stream-mean
        requests per second (element-iteration weighted)."""
        solves, mean_work, threads, npick = self.cpu_sample(steps=max(1, args.warmup) + args.steps)
        timed = solves[max(1, args.warmup):]
        t = sum(s for s, _ in timed)
        w = sum(x for _, x in timed)
        sample = (f"each step one whole log-Sinkhorn solve of a stream request of <= 2^24 elements ({npick} of "
                  f"{self.R}, in stream order) by the oracle on {threads} threads; value = the solves' "
                  f"element-iterations / the stream's mean per request ({mean_work:.3g}) per second")
        return {"seconds": t, "value": (w / mean_work) / t, "cores": threads, "sample": sample,
                "requests_per_step": (w / mean_work) / len(timed)}


class GradWorkload:
    """One log-Sinkhorn solve with a fixed unroll depth plus its gradient with
    respect to a per step: the forward records every iteration's potentials,
    one cooperative launch runs the L backward steps."""

    higher_is_better = True

    def __init__(self, m=2048, n=2048, reg=0.05, L=100):
        self.m, self.n, self.reg, self.L = m, n, reg, L
        self.unit = "solves/s"
        self.metric = f"log-Sinkhorn solve + gradient w.r.t. a per second ({m}x{n}, L={L}, FP64)"
        self.desc = (f"log-Sinkhorn {m}x{n} FP64 with grad_a, Dirichlet(0.5) marginals, uniform points in [0,1]^2, "
                     f"squared-Euclidean cost / max, eps={reg:g}, L={L} unrolled iterations (tol 0), "
                     f"outputs f, g, loss, grad_a")

    def inputs(self):
        from rwig_b200 import synth
        return synth.sinkhorn_problem(self.m, self.n, 0.5, 2)

    def cpu_seconds(self, threads):
        """CPU port time of one step: runs with 2 and 4 unrolled iterations
        (forward + backward), extrapolated to L."""
        import oracle
        a, b, C = self.inputs()
        t = {}
        for it in (2, 4):
            t0 = time.perf_counter()
            oracle.sinkhorn_log(a, b, C, self.reg, with_grad=True, max_iter=it, zero_tol=0.0, n_threads=threads)
            t[it] = time.perf_counter() - t0
        per_iter = max((t[4] - t[2]) / 2, 1e-9)
        fixed = max(t[2] - 2 * per_iter, 0.0)
        sample = (f"2- and 4-iteration runs with gradient of the same {self.m}x{self.n} problem ({threads} threads "
                  f"forward, backward serial as in the reference), extrapolated to L={self.L}: "
                  f"{per_iter * 1e3:.0f} ms per forward+backward iteration")
        return fixed + self.L * per_iter, threads, sample

    def run(self, args, dev, world, rank, clocks_cls):
        import torch

        import rwig_b200 as rw
        from rwig_b200 import _lib
        m, n = self.m, self.n
        a, b, C = self.inputs()
        ta, tb = torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)
        tC = torch.from_numpy(C.T).to(dev)
        f = torch.empty(m, dtype=torch.float64, device=dev)
        g = torch.empty(n, dtype=torch.float64, device=dev)
        ga = torch.empty(m, dtype=torch.float64, device=dev)
        flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > L2
        stream = torch.cuda.current_stream()

        def step():
            return rw.sinkhorn_log_device(ta, tb, tC, self.reg, self.L, 0.0, f=f, g=g, grad_a=ga, stream=stream)

        for _ in range(args.warmup):
            flush.zero_()
            step()
        torch.cuda.synchronize()
        times, reps = [], []
        with clocks_cls(dev.index) as clocks:
            if world > 1:
                import torch.distributed as dist
                dist.barrier()
            torch.cuda.synchronize()
            for _ in range(args.steps):
                flush.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                step()
                e1.record(stream)
                e1.synchronize()
                times.append(e0.elapsed_time(e1))
                reps.append(rw.last_report())
            torch.cuda.synchronize()
        tot_ms = max_over_ranks(sum(times), world, dev)
        # end to end through the host-pointer entry with pinned buffers
        hC = torch.from_numpy(C.T.copy()).pin_memory()
        ha, hb = torch.from_numpy(a).pin_memory(), torch.from_numpy(b).pin_memory()
        hf, hg, hga = (torch.empty(k, dtype=torch.float64).pin_memory() for k in (m, n, m))
        L = _lib.load()
        dp = ctypes.POINTER(ctypes.c_double)

        def cp(t):
            return ctypes.cast(ctypes.c_void_p(t.data_ptr()), dp)

        def host_step():
            loss, err, it = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
            _lib.check(L.rwig_sinkhorn_log(None, cp(hga), cp(hf), cp(hg), ctypes.byref(loss), ctypes.byref(it),
                                           ctypes.byref(err), cp(ha), cp(hb), cp(hC), m, n, self.reg, 1, self.L, 0.0))

        host_step()
        e2e_s = 0.0
        for _ in range(args.steps):
            t0 = time.perf_counter()
            host_step()
            e2e_s += time.perf_counter() - t0
        e2e_s = max_over_ranks(e2e_s, world, dev)
        assert np.array_equal(hga.numpy(), ga.cpu().numpy()), "host and device gradients disagree"
        if rank != 0:
            return None
        peak, peak_kind = measured_peaks()
        gms = sum(r["grad_ms"] for r in reps) / len(reps)
        # backward kernel: one read of the m x n cost per unrolled step
        alg = self.L * m * n * 8.0
        achieved = alg / (gms / 1e3) / 1e9 if gms > 0 else None
        roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak if achieved else None, "traffic": None, "peak_source": peak_kind,
                "kernel": "grad_kernel (unrolled backward, 2 exp per element per step)",
                "kernel_ms_per_step": gms, "alg_bytes_per_step": alg,
                "forward_ms_per_step": tot_ms / args.steps - gms}
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            secs, cores, sample = self.cpu_seconds(os.cpu_count() or 1)
            cpu = {"value": 1.0 / secs, "unit": self.unit, "cores": cores, "kind": "port", "sample": sample}
        return {"value": args.steps * world / (tot_ms / 1e3), "ms_per_step": tot_ms / args.steps,
                "config": {"workload": self.desc, "parallelism": f"replicas x{world}",
                           "l2": "flushed between steps (256 MB write)"},
                "e2e": {"value": args.steps * world / e2e_s, "unit": self.unit,
                        "h2d_bytes_per_step": (m * n + m + n) * 8, "d2h_bytes_per_step": (2 * m + n) * 8},
                "gpu_launches": sum(r["kernel_launches"] for r in reps), "roofline": roof, "cpu_baseline": cpu,
                "clocks": clocks.summary()}

    def reference(self, args):
        threads = os.cpu_count() or 1
        for _ in range(args.warmup):
            self.cpu_seconds(threads)
        secs, cores, sample = [], 1, ""
        for _ in range(args.steps):
            s_, cores, sample = self.cpu_seconds(threads)
            secs.append(s_)
        return sum(secs), cores, sample


WORKLOADS = {
    "log4096": SinkhornWorkload("log", 4096, 4096, 0.01, 0.5, 2000, 1e-9),
    "vanilla256": SinkhornWorkload("vanilla", 256, 256, 0.1, 1.0, 1000, 1e-9),
    "barycenter2048": BarycenterWorkload(),
    "wdl5000": WdlWorkload(),
    "stream": StreamWorkload(),
    "sinkgrad2048": GradWorkload(),
}


def reference_gpu_timing(ref_call, engine_call, steps, what):
    """rwig's own GPU code (oracle/_ref, compiled from the reference's sources:
    cuBLAS products, per-call device allocation) against the engine's
    host-pointer entry on the same problem: wall-clock calls per second of
    each, two untimed calls first.  None when oracle/_ref was not built."""
    import oracle
    if not oracle.ref_gpu_available():
        return None
    out = {}
    for name, fn in (("value", ref_call), ("engine_same_call", engine_call)):
        fn()
        fn()
        t0 = time.perf_counter()
        for _ in range(steps):
            fn()
        out[name] = steps / (time.perf_counter() - t0)
    out.update(unit="solves/s", call=what, speedup_engine_over_reference=out["engine_same_call"] / out["value"])
    return out


def max_over_ranks(x, world, dev):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def base_line(wl, args, world):
    return {"metric": wl.metric, "unit": wl.unit, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": wl.higher_is_better, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic"}


def run_reference(args):
    """The reference's CPU path (the oracle port, all host threads) on the same
    workload; rank 0 alone runs and prints, the other ranks exit."""
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    wl = WORKLOADS[args.workload]
    r = wl.reference(args)
    extra = {}
    if isinstance(r, dict):
        tot, cores, sample, value = r["seconds"], r["cores"], r["sample"], r["value"]
        extra["requests_per_step"] = r["requests_per_step"]
    else:
        tot, cores, sample = r
        value = args.steps / tot
    cfg = wl.config(args.gpus) if hasattr(wl, "config") else {"workload": wl.desc, "parallelism": "cpu"}
    line = {"impl": "reference", **base_line(wl, args, args.gpus), "value": value,
            "ms_per_step": tot / args.steps * 1e3, "config": cfg, **extra,
            "cpu_baseline": {"value": value, "unit": wl.unit, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": wl.unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_engine(args):
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    wl = WORKLOADS[args.workload]
    out = wl.run(args, dev, world, rank, ClockSampler)
    if rank == 0:
        print(json.dumps({**base_line(wl, args, world), **out}), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_gemm(args):
    """Y = K X and Y = K^T X for an --n x --n K and --m columns through the
    engine's GEMM self-check entry (the product kernels of the barycenter and
    WDL paths, EpiStore epilogue) and through torch.matmul (cuBLAS), each the
    median of 9 launches timed with CUDA events; relative max error vs
    cuBLAS."""
    import torch

    from rwig_b200 import _lib
    L = _lib.load()
    dev = torch.device("cuda", 0)
    n, w = args.n, args.m
    g = torch.Generator(device="cpu").manual_seed(1)
    K = torch.rand(n, n, dtype=torch.float64, generator=g).to(dev)  # column-major n x n (row-major K^T)
    X = torch.rand(w, n, dtype=torch.float64, generator=g).to(dev)  # column-major n x w
    Y = torch.empty(w, n, dtype=torch.float64, device=dev)
    vp = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731

    def timed(fn):
        ts = []
        for _ in range(9):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            s.record()
            fn()
            e.record()
            torch.cuda.synchronize()
            ts.append(s.elapsed_time(e))
        return sorted(ts)[len(ts) // 2]

    flops = 2.0 * n * n * w
    for trans in (0, 1):
        st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)  # the events' stream
        ms = timed(lambda: _lib.check(L.rwig_selftest_dgemm(vp(K), n, trans, n, n, w, vp(X), n, vp(Y), n, 0, st)))
        Kop = K.t() if trans == 0 else K
        ref = Kop @ X.t()
        cub = timed(lambda: torch.matmul(Kop, X.t()))
        err = ((Y.t() - ref).abs().max() / ref.abs().max()).item()
        print(json.dumps({"n": n, "columns": w, "trans": trans, "engine_ms": ms, "engine_tflops": flops / ms / 1e9,
                          "cublas_ms": cub, "cublas_tflops": flops / cub / 1e9, "rel_err": err}))
    return 0


def run_single(args):
    """One warm-up plus one solve of an m x n log problem with a fixed iteration
    count (tol 0): the small case the kernel profiles are captured on.  With
    --workload barycenter2048: two log-barycenter solves with gradient on n
    points, --s histograms, --iters iterations (the second one is captured
    into a CUDA graph)."""
    import torch

    import rwig_b200 as rw
    from rwig_b200 import synth
    if args.gemm:
        return run_gemm(args)
    if args.workload.startswith("sinkgrad"):
        # two log-Sinkhorn solves with gradient, --m x --n, --iters unrolled iterations
        dev = torch.device("cuda", 0)
        a, b, C = synth.sinkhorn_problem(args.m, args.n, 0.5, 2)
        ta, tb = torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)
        tC = torch.from_numpy(C.T.copy()).to(dev)
        ga = torch.empty(args.m, dtype=torch.float64, device=dev)
        for _ in range(2):
            r = rw.sinkhorn_log_device(ta, tb, tC, 0.05, args.iters, 0.0, grad_a=ga)
        torch.cuda.synchronize()
        rep = rw.last_report()
        print(json.dumps({"m": args.m, "n": args.n, "iter": r["iter"], "device_ms": rep["device_ms"],
                          "grad_ms": rep["grad_ms"], "launches": rep["kernel_launches"]}))
        return 0
    if args.workload == "stream" and args.stream_profile:
        from rwig_b200 import _lib
        dev = torch.device("cuda", 0)
        L = _lib.load()
        wl = WORKLOADS["stream"]
        data = wl.build(dev)
        probs, res = wl.problems(data), (_lib.Result * len(data))()
        sp = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        _lib.check(L.rwig_batch_sinkhorn_log_dev(probs, len(data), res, sp))  # sizes the scratch
        torch.cuda.synchronize()
        L.rwig_set_option(b"batch.profile", 1.0)
        try:
            _lib.check(L.rwig_batch_sinkhorn_log_dev(probs, len(data), res, sp))
            torch.cuda.synchronize()
        finally:
            L.rwig_set_option(b"batch.profile", float("nan"))
        print(json.dumps({"problems": len(data), "device_ms": rw.last_report()["sweep_ms"]}))
        return 0
    if args.workload == "stream":
        # two batched calls of --iters fixed iterations: one streamed 2048 x 2048
        # problem, then 64 resident 300 x 1500 problems
        from rwig_b200 import _lib
        dev = torch.device("cuda", 0)
        L = _lib.load()
        vp = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
        for cases in ([(2048, 2048)], [(300, 1500)] * 64):
            keep, arr = [], (_lib.Problem * len(cases))()
            for k, (m, n) in enumerate(cases):
                a, b, C = synth.sinkhorn_problem(m, n, 1.0, salt=k + 1)
                t = [torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev),
                     torch.from_numpy(np.ascontiguousarray(C.T)).to(dev),
                     torch.empty(m, dtype=torch.float64, device=dev), torch.empty(n, dtype=torch.float64, device=dev)]
                keep.append(t)
                arr[k] = _lib.Problem(vp(t[0]), vp(t[1]), vp(t[2]), m, n, 0.05, args.iters, 0.0, None, vp(t[3]),
                                      vp(t[4]))
            res = (_lib.Result * len(cases))()
            _lib.check(L.rwig_batch_sinkhorn_log_dev(arr, len(cases), res, None))
            rep = rw.last_report()
            print(json.dumps({"problems": len(cases), "m": cases[0][0], "n": cases[0][1], "iter": res[0].iter,
                              "device_ms": rep["device_ms"], "launches": rep["kernel_launches"]}))
        return 0
    if args.workload.startswith("wdl"):
        # one batched WDL gradient step on device buffers: V = --n words,
        # --s topics, --m documents, --iters iterations
        from rwig_b200 import _lib
        Y, C, A0, L0 = synth.wdl_config(V=args.n, M=args.m, S=args.s, dim=64)
        dev = torch.device("cuda", 0)
        A = torch.from_numpy(np.ascontiguousarray(np.exp(A0) / np.exp(A0).sum(0)).T.copy()).to(dev)
        W = torch.from_numpy(np.ascontiguousarray((np.exp(L0) / np.exp(L0).sum(0)).T)).to(dev)
        tY = torch.from_numpy(np.ascontiguousarray(Y.T)).to(dev)
        tC = torch.from_numpy(np.ascontiguousarray(C.T)).to(dev)
        gA = torch.empty((args.s, args.n), dtype=torch.float64, device=dev)
        gl = torch.empty(args.s, dtype=torch.float64, device=dev)
        vp = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
        L = _lib.load()
        for _ in range(2):
            _lib.check(L.rwig_wdl_batch_grad_dev(vp(gA), vp(gl), vp(A), vp(W), vp(tY), vp(tC), args.n, args.s,
                                                 args.m, 0.05, args.iters, 1, None))
        rep = rw.last_report()
        print(json.dumps({"V": args.n, "S": args.s, "D": args.m, "L": args.iters, "device_ms": rep["device_ms"],
                          "launches": rep["kernel_launches"]}))
        return 0
    if args.workload.startswith("barycenter"):
        A, C, w, be = synth.barycenter_config(n=args.n, S=args.s, dim=50)
        for _ in range(2):
            r = rw.barycenter(A, C, w, be, {"reg": 0.05, "with_grad": True, "method": "log",
                                            "max_iter": args.iters, "zero_tol": 0.0})
        rep = rw.last_report()
        print(json.dumps({"n": args.n, "S": args.s, "iter": r["iter"], "device_ms": rep["device_ms"],
                          "launches": rep["kernel_launches"]}))
        return 0
    a, b, C = synth.log_config(args.m, args.n)
    if args.l2_hot is not None:
        rw.load().rwig_set_option(b"log_sinkhorn.l2_hot", float(args.l2_hot))
    dev = torch.device("cuda", 0)
    ta, tb = torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)
    tC = torch.from_numpy(C.T).to(dev)
    P = torch.empty((args.n, args.m), dtype=torch.float64, device=dev)
    for _ in range(2):
        r = rw.sinkhorn_log_device(ta, tb, tC, 0.01, args.iters, 0.0, P=P)
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
