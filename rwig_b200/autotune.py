"""Autotuner of the batched log-Sinkhorn's team shapes and schedule.

The batched kernel behind rwig_batch_sinkhorn_log*, and the server built on it,
gives every problem a team of CTAs whose shape and schedule follow the
engine's batch.* options:

  batch.max_team           largest team of CTAs per problem;
  batch.resident_team      largest team that keeps its K strips in shared
                           memory (larger problems stream their strips);
  batch.stream_strip_kb    strip per member of a streamed team;
  batch.strip_kb           strip per member of a resident team;
  batch.redundant_rows     teams up to this many partial row sums merge them
                           redundantly (one team barrier per iteration);
  batch.backfill_us        how long a waiting problem may be passed over by
                           smaller ones that fit the free CTAs.

Which values are fastest depends on the mix of sizes and the GPU.
autotune_batch() times the batched call on a sample of the caller's problems
(already on the device) under a coordinate search over those options, keeps
the fastest setting and sets it process-wide.  Results under any setting are
the same problems solved in another summation order: every trial's iteration
counts and losses are checked against those of the starting setting, and a
trial that differs beyond rounding is rejected.  No counterpart in the
reference (rwig solves problems one call at a time).
"""
import ctypes
import math

import numpy as np

from . import _lib

OPTIONS = ("batch.max_team", "batch.resident_team", "batch.stream_strip_kb", "batch.strip_kb",
           "batch.redundant_rows", "batch.backfill_us")


def defaults(sm_count: int) -> dict:
    """Built-in values of the tuned options for a batched call
    (rwig_b200/csrc/batch.cu; a server's largest team is 0.4 x the SMs)."""
    return {"batch.max_team": float(math.floor(0.25 * sm_count)), "batch.resident_team": 32.0,
            "batch.stream_strip_kb": 1024.0, "batch.strip_kb": 184.0, "batch.redundant_rows": 16384.0,
            "batch.backfill_us": 5000.0}


def default_space(sm_count: int) -> dict:
    """Candidate values per option, searched in this order."""
    return {
        "batch.max_team": [float(max(1, int(f * sm_count))) for f in (0.15, 0.25, 0.4, 0.6)],
        "batch.resident_team": [16.0, 32.0, 64.0],
        "batch.stream_strip_kb": [512.0, 1024.0, 2048.0],
        "batch.strip_kb": [96.0, 144.0, 184.0],
        "batch.redundant_rows": [8192.0, 16384.0, 32768.0],
        "batch.backfill_us": [1000.0, 5000.0, 20000.0],
    }


def coordinate_search(measure, space: dict, start: dict, min_gain: float = 0.02):
    """Greedy coordinate search: starting from `start`, for each option of
    `space` in order try its candidate values with the others at the best
    setting so far, and keep a value when it is faster than the best by more
    than the fraction `min_gain` (so timing noise does not move the setting).
    measure(options) -> milliseconds, or None for a rejected trial.  Returns
    (best options, best ms, trials as [(options, ms)])."""
    cur = dict(start)
    best = measure(cur)
    if best is None:
        raise RuntimeError("the starting setting was rejected")
    trials = [(dict(cur), best)]
    for name, values in space.items():
        for v in values:
            if cur.get(name) == v:
                continue
            cand = dict(cur)
            cand[name] = v
            t = measure(cand)
            trials.append((dict(cand), t))
            if t is not None and t < best * (1.0 - min_gain):
                best, cur = t, cand
    return cur, best, trials


def _current(L, names):
    """Options as set now: name -> value, or None where the default applies."""
    out = {}
    for n in names:
        v = ctypes.c_double()
        rc = L.rwig_get_option(n.encode(), ctypes.byref(v))
        if rc < 0:
            _lib.check(rc)
        out[n] = v.value if rc == 0 else None
    return out


def _apply(L, opts):
    for n, v in opts.items():
        _lib.check(L.rwig_set_option(n.encode(), float("nan") if v is None else float(v)))


def _device_batch(problems, dev):
    """The problems' inputs copied to the device once; returns (keep-alive
    tensors, rwig_problem array).  Same dict format as batch_sinkhorn_log."""
    import torch

    from .api import _cost_or_points, _vec
    keep = []
    arr = (_lib.Problem * len(problems))()
    vp = lambda t: ctypes.c_void_p(t.data_ptr()) if t is not None else None  # noqa: E731
    for i, q in enumerate(problems):
        a, b = _vec(q["a"], "a"), _vec(q["b"], "b")
        C, X, Y = _cost_or_points(q)
        M, N = a.shape[0], b.shape[0]
        ta, tb = torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)
        tC = torch.from_numpy(np.ascontiguousarray(C.T)).to(dev) if C is not None else None
        tX = torch.from_numpy(np.ascontiguousarray(X.T)).to(dev) if X is not None else None
        tY = torch.from_numpy(np.ascontiguousarray(Y.T)).to(dev) if Y is not None else None
        tf = torch.empty(M, dtype=torch.float64, device=dev)
        tg = torch.empty(N, dtype=torch.float64, device=dev)
        keep.append((ta, tb, tC, tX, tY, tf, tg))
        arr[i] = _lib.Problem(vp(ta), vp(tb), vp(tC), M, N, float(q.get("reg", 0.1)), int(q.get("max_iter", 1000)),
                              float(q.get("zero_tol", 1e-6)), None, vp(tf), vp(tg), vp(tX), vp(tY),
                              0 if X is None else X.shape[1])
    return keep, arr


def autotune_batch(problems, space=None, reps: int = 3, min_gain: float = 0.03, apply: bool = True,
                   loss_rtol: float = 1e-9) -> dict:
    """Tune the batch.* options for `problems` (dicts as in
    batch_sinkhorn_log: a, b, C or point clouds x, y, reg, max_iter,
    zero_tol) on cuda:0.  Each trial is `reps` batched calls on device
    buffers, timed with CUDA events; the trial's time is their median.
    space: {option: [values]} (default: default_space for this GPU).  With
    apply, the best setting stays set process-wide; otherwise the options
    are put back as they were.  Returns {"options", "ms", "start_ms",
    "speedup", "trials", "rejected"}."""
    import torch

    problems = list(problems)
    if not problems:
        raise ValueError("autotune_batch needs at least one problem")
    L = _lib.load()
    dev = torch.device("cuda", 0)
    sm = torch.cuda.get_device_properties(dev).multi_processor_count
    space = default_space(sm) if space is None else space
    names = list(space.keys())
    before = _current(L, names)
    base = defaults(sm)
    start = {n: (before[n] if before[n] is not None else base.get(n)) for n in names}
    keep, arr = _device_batch(problems, dev)
    n = len(problems)
    res = (_lib.Result * n)()
    stream = torch.cuda.current_stream(dev)
    sp = ctypes.c_void_p(stream.cuda_stream)
    ref = {}
    rejected = []

    def measure(opts):
        _apply(L, opts)
        _lib.check(L.rwig_batch_sinkhorn_log_dev(arr, n, res, sp))  # warm-up (allocations, first launch)
        ts = []
        for _ in range(max(1, reps)):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            _lib.check(L.rwig_batch_sinkhorn_log_dev(arr, n, res, sp))
            e.record(stream)
            e.synchronize()
            ts.append(s.elapsed_time(e))
        out = [(res[i].iter, res[i].loss) for i in range(n)]
        if not ref:
            ref["r"] = out
        else:
            for (it0, l0), (it, lo) in zip(ref["r"], out):
                if it != it0 or not abs(lo - l0) <= loss_rtol * max(1.0, abs(l0)):
                    rejected.append(dict(opts))
                    return None
        return float(np.median(ts))

    try:
        best, best_ms, trials = coordinate_search(measure, space, start, min_gain)
    except BaseException:
        _apply(L, before)
        raise
    _apply(L, best if apply else before)
    del keep
    return {"options": best, "ms": best_ms, "start_ms": trials[0][1], "speedup": trials[0][1] / best_ms,
            "trials": trials, "rejected": rejected}
