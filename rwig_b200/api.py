"""R-facing API of rwig, restated over the engine's C ABI.

`sinkhorn()` mirrors rwig's R function of the same name (R/sinkhorn.R:85-181):
same control list, defaults, validation messages, automatic method choice and
result fields.  The compute goes through include/rwig_b200.h; there is no CPU
path here.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _lib
from ._lib import RwigError

SINKHORN_ARGS = ("reg", "with_grad", "use_cuda", "n_threads", "method", "threshold", "max_iter",
                 "zero_tol", "verbose")


def check_sinkhorn_args(ctrl: dict | None) -> dict:
    """Fill and validate a sinkhorn control list (R/check_args.R:108-189)."""
    ctrl = dict(ctrl or {})
    bad = [k for k in ctrl if k not in SINKHORN_ARGS]
    if bad:
        raise ValueError(", ".join(bad) + " not matching one of the sinkhorn arguments: " +
                         ", ".join(f'"{a}"' for a in SINKHORN_ARGS))
    defaults = dict(reg=0.1, with_grad=False, use_cuda=True, n_threads=0, method="auto",
                    threshold=0.1, max_iter=1000, zero_tol=1e-6, verbose=10)
    for k, v in defaults.items():
        if ctrl.get(k) is None:
            ctrl[k] = v
    if ctrl["method"] not in ("auto", "vanilla", "log"):
        raise ValueError('method must be from: "auto", "vanilla", or "log"')
    return ctrl


def choose_sinkhorn_method(C: np.ndarray, reg: float, threshold: float) -> str:
    """The "auto" rule of R/sinkhorn.R:124-142."""
    k1 = math.exp(-float(np.min(C)) / reg)
    k2 = math.exp(-float(np.max(C)) / reg)
    return "log" if min(k1, k2) < threshold else "vanilla"


def _vec(x, name):
    a = np.asarray(x, dtype=np.float64)
    if a.ndim != 1:
        raise ValueError(f"{name} must be a numeric vector!")
    return np.ascontiguousarray(a)


def _mat(x, name):
    a = np.asarray(x, dtype=np.float64)
    if a.ndim != 2:
        raise ValueError(f"{name} must be a numeric matrix!")
    return np.asfortranarray(a)


def _dp(a):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def sinkhorn(a, b, C, sinkhorn_control: dict | None = None) -> dict:
    """Entropic OT between histograms a and b under cost C (R/sinkhorn.R:85)."""
    a = _vec(a, "a")
    b = _vec(b, "b")
    C = _mat(C, "C")
    if a.shape[0] != C.shape[0] or b.shape[0] != C.shape[1]:
        raise ValueError("a, b, C don't match in dimension!")
    ctrl = check_sinkhorn_args(sinkhorn_control)
    reg = ctrl["reg"]
    if not isinstance(reg, (int, float)) or isinstance(reg, bool):
        raise ValueError("reg must be a single value")
    reg = float(reg)
    method = ctrl["method"]
    if method == "auto":
        method = choose_sinkhorn_method(C, reg, ctrl["threshold"])
    M, N = C.shape
    with_grad = bool(ctrl["with_grad"])
    P = np.zeros((M, N), order="F")
    x, y = np.zeros(M), np.zeros(N)
    ga = np.zeros(M) if with_grad else None
    loss, err, it = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
    L = _lib.load()
    if method == "log":
        rc = L.rwig_sinkhorn_log(_dp(P), _dp(ga), _dp(x), _dp(y), ctypes.byref(loss), ctypes.byref(it),
                                 ctypes.byref(err), _dp(a), _dp(b), _dp(C), M, N, reg, int(with_grad),
                                 int(ctrl["max_iter"]), float(ctrl["zero_tol"]))
        names = ("f", "g")
    else:
        fn = getattr(L, "rwig_sinkhorn_vanilla", None)
        if fn is None:
            raise RwigError(-6, "vanilla Sinkhorn is not available in this build")
        rc = fn(_dp(P), _dp(ga), _dp(x), _dp(y), ctypes.byref(loss), ctypes.byref(it), ctypes.byref(err),
                _dp(a), _dp(b), _dp(C), M, N, reg, int(with_grad), int(ctrl["max_iter"]),
                float(ctrl["zero_tol"]))
        names = ("u", "v")
    _lib.check(rc)
    out = {"P": P}
    if with_grad:
        out["grad_a"] = ga
    out.update({names[0]: x, names[1]: y, "loss": loss.value, "iter": it.value, "err": err.value,
                "return_status": rc, "method": method})
    return out


BARYCENTER_ARGS = SINKHORN_ARGS


def check_barycenter_args(ctrl: dict | None) -> dict:
    """Fill and validate a barycenter control list (R/check_args.R:193-271)."""
    ctrl = dict(ctrl or {})
    bad = [k for k in ctrl if k not in BARYCENTER_ARGS]
    if bad:
        raise ValueError(", ".join(bad) + " not matching one of the barycenter arguments: " +
                         ", ".join(f'"{a}"' for a in BARYCENTER_ARGS))
    defaults = dict(reg=0.1, with_grad=False, use_cuda=True, n_threads=0, method="auto", threshold=0.1,
                    max_iter=1000, zero_tol=1e-6, verbose=0)
    for k, v in defaults.items():
        if ctrl.get(k) is None:
            ctrl[k] = v
    if ctrl["method"] not in ("auto", "parallel", "log"):
        raise ValueError('method must be from: "auto", "parallel", or "log"')
    return ctrl


def barycenter(A, C, w, b_ext=None, barycenter_control: dict | None = None) -> dict:
    """Wasserstein barycenter of the columns of A (R/barycenter.R:90)."""
    A = np.asfortranarray(np.asarray(A, dtype=np.float64))
    C = np.asfortranarray(np.asarray(C, dtype=np.float64))
    if A.ndim != 2:
        raise ValueError("A must be a numeric matrix!")
    if C.ndim != 2:
        raise ValueError("C must be a numeric matrix!")
    w = np.asarray(w, dtype=np.float64)
    if w.ndim != 1:
        raise ValueError("w must be a numeric vector!")
    if A.shape[0] != C.shape[0]:
        raise ValueError("number of rows of A and C must equal!")
    ctrl = check_barycenter_args(barycenter_control)
    reg = ctrl["reg"]
    if not isinstance(reg, (int, float)) or isinstance(reg, bool):
        raise ValueError("reg must be a single value")
    reg = float(reg)
    with_grad = bool(ctrl["with_grad"])
    if with_grad and b_ext is None:
        raise ValueError("you must supply the `b_ext` with `with_grad = TRUE`!")
    method = ctrl["method"]
    if method == "auto":  # R/barycenter.R:168-182
        method = "log" if choose_sinkhorn_method(C, reg, ctrl["threshold"]) == "log" else "parallel"
    M, S = A.shape
    N = C.shape[1]
    if w.shape[0] != S:
        raise ValueError("w must have one weight per column of A")
    be = np.ascontiguousarray(np.asarray(b_ext, dtype=np.float64).ravel()) if with_grad else None
    if with_grad and be.shape[0] != N:
        raise ValueError("b_ext must have one entry per column of C")
    X1 = np.zeros((M, S), order="F")
    X2 = np.zeros((N, S), order="F")
    b = np.zeros(N)
    gA = np.zeros((M, S), order="F") if with_grad else None
    gw = np.zeros(S) if with_grad else None
    loss, err, it = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
    L = _lib.load()
    fn = L.rwig_barycenter_log if method == "log" else L.rwig_barycenter_parallel
    rc = fn(_dp(X1), _dp(X2), _dp(b), _dp(gA), _dp(gw), ctypes.byref(loss), ctypes.byref(it), ctypes.byref(err),
            _dp(A), _dp(np.ascontiguousarray(w)), _dp(C), _dp(be), M, N, S, reg, int(with_grad),
            int(ctrl["max_iter"]), float(ctrl["zero_tol"]))
    _lib.check(rc)
    names = ("F", "G") if method == "log" else ("U", "V")
    out = {"b": b}
    if with_grad:
        out.update(grad_A=gA, grad_w=gw, loss=loss.value)
    out.update({names[0]: X1, names[1]: X2, "iter": it.value, "err": err.value, "return_status": rc,
                "method": method})
    return out


def batch_barycenter(problems) -> list:
    """Many barycenter problems in one call (rwig_batch_barycenter_dev):
    `problems` is an iterable of dicts with A, C, w, optional b_ext and
    optional control entries as in barycenter() (reg, method "log" or
    "parallel", with_grad, max_iter, zero_tol).  Problems with a fixed
    iteration count (zero_tol <= 0) run side by side on the GPU.  Returns one
    dict per problem with the keys of barycenter()'s result."""
    import torch
    dev = torch.device("cuda", 0)
    problems = list(problems)
    n = len(problems)
    arr = (_lib.BaryProblem * max(n, 1))()
    res = (_lib.BaryResult * max(n, 1))()
    keep, meta = [], []
    t = lambda x: torch.from_numpy(np.ascontiguousarray(x)).to(dev) if x is not None else None  # noqa: E731
    vp = lambda x: ctypes.c_void_p(x.data_ptr()) if x is not None else None  # noqa: E731
    for i, q in enumerate(problems):
        A = np.asfortranarray(np.asarray(q["A"], dtype=np.float64))
        C = np.asfortranarray(np.asarray(q["C"], dtype=np.float64))
        w = np.asarray(q["w"], dtype=np.float64).ravel()
        ctrl = check_barycenter_args({k: v for k, v in q.items() if k not in ("A", "C", "w", "b_ext")})
        method = ctrl["method"]
        if method == "auto":
            method = "log" if choose_sinkhorn_method(C, ctrl["reg"], ctrl["threshold"]) == "log" else "parallel"
        wg = bool(ctrl["with_grad"])
        if A.ndim != 2 or C.ndim != 2 or A.shape[0] != C.shape[0] or w.shape[0] != A.shape[1]:
            raise ValueError(f"problem {i}: A (M x S), C (M x N) and w (S) don't match")
        if wg and q.get("b_ext") is None:
            raise ValueError(f"problem {i}: you must supply the `b_ext` with `with_grad = TRUE`!")
        M, S = A.shape
        N = C.shape[1]
        tA, tC, tw = t(A.T), t(C.T), t(w)  # column-major on the device
        tbe = t(np.asarray(q["b_ext"], dtype=np.float64).ravel()) if wg else None
        X1 = torch.empty((S, M), dtype=torch.float64, device=dev)
        X2 = torch.empty((S, N), dtype=torch.float64, device=dev)
        b = torch.empty(N, dtype=torch.float64, device=dev)
        gA = torch.empty((S, M), dtype=torch.float64, device=dev) if wg else None
        gw = torch.empty(S, dtype=torch.float64, device=dev) if wg else None
        keep.append((tA, tC, tw, tbe, X1, X2, b, gA, gw))
        meta.append((method, wg))
        arr[i] = _lib.BaryProblem(vp(tA), vp(tw), vp(tC), vp(tbe), M, N, S, float(ctrl["reg"]),
                                  1 if method == "log" else 0, int(wg), int(ctrl["max_iter"]), float(ctrl["zero_tol"]),
                                  vp(X1), vp(X2), vp(b), vp(gA), vp(gw))
    _lib.check(_lib.load().rwig_batch_barycenter_dev(arr, n, res, None))
    out = []
    for i in range(n):
        tA, tC, tw, tbe, X1, X2, b, gA, gw = keep[i]
        method, wg = meta[i]
        r = res[i]
        names = ("F", "G") if method == "log" else ("U", "V")
        d = {"b": b.cpu().numpy(), names[0]: np.asfortranarray(X1.cpu().numpy().T),
             names[1]: np.asfortranarray(X2.cpu().numpy().T), "iter": r.iter, "err": r.err,
             "return_status": r.status, "method": method}
        if wg:
            d.update(grad_A=np.asfortranarray(gA.cpu().numpy().T), grad_w=gw.cpu().numpy(), loss=r.loss)
        out.append(d)
    return out


def wdl_cpp(Y, C, reg, S, batch_size, epochs, sinkhorn_mode=1, max_iter=1000, zero_tol=1e-6, optimizer=2,
            eta=0.001, gamma=0.01, beta1=0.9, beta2=0.999, eps=1e-8, verbose=False, seed=42, Alpha0=None,
            Lambda0=None, max_steps=0) -> dict:
    """Wasserstein dictionary learning on a document matrix Y (N x M) and cost
    C (N x N): the numeric core of rwig's wdl(), with wdl_cpp_cuda's argument
    list (src/wdl.cpp:57-65).  Returns {"A": topics N x S, "W": weights S x M,
    "Yhat": barycenters N x M}.  Training runs the batched parallel
    barycenter, as the reference does on every path; the inference
    barycenters are parallel, as on the reference's GPU path (sinkhorn_mode
    is accepted for signature compatibility).  Alpha0 / Lambda0 give the
    initial logits (otherwise N(0, 1) draws from mt19937(seed)); max_steps > 0
    stops training after that many batches."""
    Y = _mat(Y, "Y")
    C = _mat(C, "C")
    N, M = Y.shape
    if C.shape != (N, N):
        raise ValueError("C must be N x N for N rows of Y")
    if optimizer not in (0, 1, 2):
        raise ValueError("optimizer must be 0 (SGD), 1 (Adam) or 2 (AdamW)")
    S = int(S)
    a0 = None if Alpha0 is None else np.asfortranarray(np.asarray(Alpha0, dtype=np.float64))
    l0 = None if Lambda0 is None else np.asfortranarray(np.asarray(Lambda0, dtype=np.float64))
    if a0 is not None and a0.shape != (N, S):
        raise ValueError("Alpha0 must be N x S")
    if l0 is not None and l0.shape != (S, M):
        raise ValueError("Lambda0 must be S x M")
    A = np.zeros((N, S), order="F")
    W = np.zeros((S, M), order="F")
    Yhat = np.zeros((N, M), order="F")
    rc = _lib.load().rwig_wdl(_dp(A), _dp(W), _dp(Yhat), _dp(Y), _dp(C), N, M, S, float(reg), int(max_iter),
                              float(zero_tol), int(batch_size), int(epochs), int(optimizer), float(eta),
                              float(gamma), float(beta1), float(beta2), float(eps), int(seed), int(bool(verbose)),
                              _dp(a0), _dp(l0), int(max_steps))
    _lib.check(rc)
    return {"A": A, "W": W, "Yhat": Yhat}


def wdl_batch_grad(A, W_B, Y_B, K_or_C, reg=0.1, L=20, mode=0):
    """One batched WDL gradient step (WassersteinDictionaryLearning::
    _train_batch_batched, src/wdl_impl.cpp:87-247): returns (g_Alpha (N x S),
    g_lambda (S)).  mode 0: K_or_C is the Gibbs kernel; 1: it is the cost C."""
    A = _mat(A, "A")
    W_B = _mat(W_B, "W_B")
    Y_B = _mat(Y_B, "Y_B")
    KC = _mat(K_or_C, "K_or_C")
    N, S = A.shape
    D = W_B.shape[1]
    if W_B.shape[0] != S or Y_B.shape != (N, D) or KC.shape != (N, N):
        raise ValueError("A (N x S), W_B (S x D), Y_B (N x D) and K_or_C (N x N) do not match")
    gA, gl = np.zeros((N, S), order="F"), np.zeros(S)
    _lib.check(_lib.load().rwig_wdl_batch_grad(_dp(gA), _dp(gl), _dp(A), _dp(W_B), _dp(Y_B), _dp(KC), N, S, D,
                                               float(reg), int(L), int(mode)))
    return gA, gl


def wdl_batch_grad_dp(A, W_B, Y_B, K_or_C, reg=0.1, L=20, mode=0, group=None, grad_fn=None):
    """Data-parallel batched WDL gradient over the ranks of a torch.distributed
    group (one process per GPU).  Every rank passes the whole batch; its D
    documents are split into contiguous shards, rank r taking documents
    [r D / R, (r + 1) D / R), and each rank computes its shard's mean gradient
    with `grad_fn` (default: this engine's wdl_batch_grad on the rank's
    current GPU).  One all-reduce of the shard sums (g_Alpha, N x S, and
    g_lambda, S) then gives every rank the whole batch's mean gradient, as
    WassersteinDictionaryLearning::_train_batch_batched averages it
    (src/wdl_impl.cpp:236-243), so every rank can take the same optimizer step.
    The all-reduce runs on the group's backend: a CUDA buffer for NCCL, a host
    buffer otherwise.  Returns (g_Alpha, g_lambda) as numpy arrays."""
    import torch
    import torch.distributed as dist
    A = _mat(A, "A")
    W_B = _mat(W_B, "W_B")
    Y_B = _mat(Y_B, "Y_B")
    N, S = A.shape
    D = W_B.shape[1]
    if W_B.shape[0] != S or Y_B.shape != (N, D):
        raise ValueError("A (N x S), W_B (S x D) and Y_B (N x D) do not match")
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    lo, hi = rank * D // world, (rank + 1) * D // world
    fn = grad_fn if grad_fn is not None else wdl_batch_grad
    buf = np.zeros(N * S + S)
    if hi > lo:
        gA, gl = fn(A, np.asfortranarray(W_B[:, lo:hi]), np.asfortranarray(Y_B[:, lo:hi]), K_or_C, reg, L, mode)
        buf[:N * S] = np.asarray(gA).ravel(order="F") * (hi - lo)
        buf[N * S:] = np.asarray(gl) * (hi - lo)
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else torch.device("cpu")
    t = torch.from_numpy(buf).to(dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    out = t.cpu().numpy() / D
    return np.asfortranarray(out[:N * S].reshape((N, S), order="F")), out[N * S:].copy()


def wdl_batch_grad_dp_dev(A, W_B, Y_B, K_or_C, reg=0.1, L=20, mode=0, group=None, stream=None):
    """Data-parallel batched WDL gradient on device buffers (one process per
    GPU, torch.distributed group).  Matrices are contiguous float64 CUDA
    tensors in column-major order, i.e. an R x C matrix is a (C, R) tensor:
    A (S, N), W_B (D, S), Y_B (D, N) and K_or_C (N, N), the last resident on
    the device for as long as the caller keeps it (it is not copied per call).
    Rank r computes the mean gradient of documents [r D / R, (r + 1) D / R)
    with rwig_wdl_batch_grad_dev straight into one device buffer, scales it by
    its shard size, and one all-reduce of that buffer (g_Alpha then g_lambda,
    N S + S doubles) on the device gives every rank the whole batch's mean
    (src/wdl_impl.cpp:236-243).  Returns device tensors (g_Alpha as (S, N),
    g_lambda (S,)); nothing passes through host memory."""
    import torch
    import torch.distributed as dist
    S, N = A.shape
    D = W_B.shape[0]
    if W_B.shape[1] != S or Y_B.shape != (D, N) or K_or_C.shape != (N, N):
        raise ValueError("A (S, N), W_B (D, S), Y_B (D, N) and K_or_C (N, N) do not match")
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    lo, hi = rank * D // world, (rank + 1) * D // world
    caller = torch.cuda.current_stream(A.device)
    st = stream if stream is not None else caller
    if st.cuda_stream == 0:
        # the engine reads a null stream as its own stream, unordered with torch's
        # legacy default stream: run on a side stream joined to the caller's
        st = torch.cuda.Stream(A.device)
    with torch.cuda.stream(st):
        st.wait_stream(caller)  # inputs written
        buf = torch.zeros(N * S + S, dtype=torch.float64, device=A.device)
    if hi > lo:
        gA, gl = buf[:N * S], buf[N * S:]
        rc = _lib.load().rwig_wdl_batch_grad_dev(_ptr(gA), _ptr(gl), _ptr(A), _ptr(W_B[lo:hi]), _ptr(Y_B[lo:hi]),
                                                 _ptr(K_or_C), N, S, hi - lo, float(reg), int(L), int(mode),
                                                 ctypes.c_void_p(st.cuda_stream))
        _lib.check(rc)
        with torch.cuda.stream(st):
            buf.mul_(float(hi - lo))
    host_collective = dist.get_backend(group) == "gloo"  # gloo reduces CUDA tensors through host copies
    if host_collective:
        st.synchronize()  # the shard's gradient is complete before the host copy starts
    with torch.cuda.stream(st):
        dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=group)
    if host_collective:
        st.synchronize()  # the reduced buffer is back on the device before any later kernel reads it
    with torch.cuda.stream(st):
        buf.div_(float(D))
    if st.cuda_stream != caller.cuda_stream:
        caller.wait_stream(st)  # the caller's later work sees the reduced gradient
        buf.record_stream(caller)
    return buf[:N * S].view(S, N), buf[N * S:]


def wdl_train_dp_dev(Y, C, S, reg=0.1, L=20, B=64, E=1, optimizer=1, eta=1e-3, gamma=0.01, beta1=0.9,
                     beta2=0.999, eps=1e-8, Alpha0=None, Lambda0=None, max_steps=0, group=None):
    """Data-parallel WDL training on device buffers (one process per GPU,
    torch.distributed group), the training loop of rwig_wdl
    (src/wdl_impl.cpp:254-340) with each batch's documents split over the
    ranks: every rank computes its shard's gradient (rwig_wdl_batch_grad_dev,
    C given, K built on the device and its INT8 residue planes reused across
    batches), one all-reduce gives every rank the batch mean
    (wdl_batch_grad_dp_dev), and every rank takes the same optimizer step and
    softmaxes on the device (rwig_wdl_update_dev), so the parameters stay
    identical on all ranks.  Y (N x M) and C (N x N) are host arrays or
    column-major device tensors ((M, N), (N, N)); Alpha0 (N x S) and Lambda0
    (S x M) the initial logits (required: the ranks must start equal).
    Returns A (N x S) and W (S x M) as host arrays, like wdl_cpp."""
    import torch
    if Alpha0 is None or Lambda0 is None:
        raise ValueError("Alpha0 and Lambda0 are required (every rank must start from the same logits)")
    dev = torch.device("cuda", torch.cuda.current_device())

    def col_major(x, rows, cols):
        if isinstance(x, torch.Tensor):
            t = x.to(device=dev, dtype=torch.float64).contiguous()
        else:
            t = torch.from_numpy(np.ascontiguousarray(np.asarray(x, dtype=np.float64).T)).to(dev)
        if t.shape != (cols, rows):
            raise ValueError(f"expected a {rows} x {cols} matrix")
        return t

    Alpha0 = np.asarray(Alpha0, dtype=np.float64)
    N, S_ = Alpha0.shape
    if S_ != S:
        raise ValueError("Alpha0 must be N x S")
    M = np.asarray(Lambda0).shape[1]
    tY, tC = col_major(Y, N, M), col_major(C, N, N)
    Al, La = col_major(Alpha0, N, S), col_major(Lambda0, S, M)
    A, W = torch.empty_like(Al), torch.empty_like(La)
    mA, vA, mL, vL = (torch.zeros_like(Al), torch.zeros_like(Al), torch.zeros_like(La), torch.zeros_like(La))
    lib = _lib.load()
    # one side stream for every engine call and torch operation of the loop (the
    # engine reads a null stream handle as its own stream)
    st = torch.cuda.Stream(dev)
    st.wait_stream(torch.cuda.current_stream(dev))  # inputs copied
    sp = ctypes.c_void_p(st.cuda_stream)
    with torch.cuda.stream(st):
        zero = torch.zeros(N * S + S, dtype=torch.float64, device=dev)
    # A, W from the initial logits: a step with a zero gradient under SGD leaves them unchanged
    _lib.check(lib.rwig_wdl_update_dev(_ptr(Al), _ptr(La), _ptr(A), _ptr(W), None, None, None, None, _ptr(zero),
                                       _ptr(zero[N * S:]), N, S, M, 0, 0.0, 0.0, 0.0, 0.0, 0.0, 1, sp))
    batches = -(-M // B)
    steps = 0
    for _ in range(E):
        for bi in range(batches):
            if max_steps > 0 and steps >= max_steps:
                break
            b0 = bi * B
            D = (M % B) if (bi == M // B) else B  # src/wdl_impl.cpp:91
            with torch.cuda.stream(st):
                gA, gl = wdl_batch_grad_dp_dev(A, W[b0:b0 + D], tY[b0:b0 + D], tC, reg, L, mode=1, group=group,
                                               stream=st)
            steps += 1
            _lib.check(lib.rwig_wdl_update_dev(_ptr(Al), _ptr(La), _ptr(A), _ptr(W), _ptr(mA), _ptr(vA), _ptr(mL),
                                               _ptr(vL), _ptr(gA), _ptr(gl), N, S, M, int(optimizer), float(eta),
                                               float(gamma), float(beta1), float(beta2), float(eps), steps, sp))
    torch.cuda.synchronize(dev)
    return {"A": A.cpu().numpy().T.copy(), "W": W.cpu().numpy().T.copy(), "steps": steps}


def _cost_or_points(q):
    """(C, None, None) from q["C"], or (None, X, Y) from point clouds q["x"]
    (M x d), q["y"] (N x d), column-major; sizes checked against a, b."""
    M, N = len(q["a"]), len(q["b"])
    if q.get("C") is not None:
        C = _mat(q["C"], "C")
        if C.shape != (M, N):
            raise ValueError("a, b, C don't match in dimension!")
        return C, None, None
    X, Y = _mat(q["x"], "x"), _mat(q["y"], "y")
    if X.shape[0] != M or Y.shape[0] != N or X.shape[1] != Y.shape[1]:
        raise ValueError("points don't match a, b or each other")
    return None, X, Y


def batch_sinkhorn_log(problems, with_plan=False) -> list:
    """Solve many log-stabilised Sinkhorn problems in one call
    (rwig_batch_sinkhorn_log).  `problems`: iterable of dicts with a, b, C
    and optional reg (0.1), max_iter (1000), zero_tol (1e-6), as in
    sinkhorn(..., method="log").  Returns one dict per problem with f, g,
    (P), loss, iter, err, return_status, marginal violations and the path
    taken (0: batched kernel, 1: per-call path)."""
    problems = list(problems)
    n = len(problems)
    arr = (_lib.Problem * max(n, 1))()
    res = (_lib.Result * max(n, 1))()
    keep = []
    for i, q in enumerate(problems):
        a, b = _vec(q["a"], "a"), _vec(q["b"], "b")
        C, X, Y = _cost_or_points(q)
        M, N = a.shape[0], b.shape[0]
        f, g = np.zeros(M), np.zeros(N)
        P = np.zeros((M, N), order="F") if with_plan else None
        keep.append((a, b, C, f, g, P, X, Y))
        vp = lambda x: ctypes.c_void_p(x.ctypes.data) if x is not None else None  # noqa: E731
        arr[i] = _lib.Problem(vp(a), vp(b), vp(C), M, N, float(q.get("reg", 0.1)), int(q.get("max_iter", 1000)),
                              float(q.get("zero_tol", 1e-6)), vp(P), vp(f), vp(g), vp(X), vp(Y),
                              0 if X is None else X.shape[1])
    _lib.check(_lib.load().rwig_batch_sinkhorn_log(arr, n, res))
    out = []
    for i in range(n):
        r = res[i].as_dict()
        d = {"f": keep[i][3], "g": keep[i][4], "loss": r["loss"], "iter": r["iter"], "err": r["err"],
             "return_status": r["status"], "marg_l1_row": r["marg_l1_row"], "marg_l1_col": r["marg_l1_col"],
             "path": r["path"]}
        if with_plan:
            d["P"] = keep[i][5]
        out.append(d)
    return out


class Server:
    """Continuous-batching log-Sinkhorn server (rwig_server_*): submit()
    admits a request into the running service kernel, poll() returns its
    result once finished.  One thread drives a server."""

    def __init__(self, mem_budget_bytes=8e9, idle_ms=50.0):
        self._L = _lib.load()
        h = ctypes.c_void_p()
        _lib.check(self._L.rwig_server_create(ctypes.byref(h), float(mem_budget_bytes), float(idle_ms)))
        self._h = h
        self._pending = {}

    def submit(self, a, b, C=None, reg=0.1, max_iter=1000, zero_tol=1e-6, with_plan=False, x=None, y=None):
        """Returns a ticket (>= 0), or None when the server is full (poll and
        retry).  Give C, or point clouds x (M x d), y (N x d) for a cost built
        on the device.  The arrays must stay alive until the result is polled."""
        a, b = _vec(a, "a"), _vec(b, "b")
        C, X, Y = _cost_or_points({"a": a, "b": b, "C": C, "x": x, "y": y})
        M, N = a.shape[0], b.shape[0]
        f, g = np.zeros(M), np.zeros(N)
        P = np.zeros((M, N), order="F") if with_plan else None
        vp = lambda z: ctypes.c_void_p(z.ctypes.data) if z is not None else None  # noqa: E731
        q = _lib.Problem(vp(a), vp(b), vp(C), M, N, float(reg), int(max_iter), float(zero_tol), vp(P), vp(f), vp(g),
                         vp(X), vp(Y), 0 if X is None else X.shape[1])
        rc = self._L.rwig_server_submit(self._h, ctypes.byref(q))
        if rc == -7:  # RWIG_E_BUSY
            return None
        _lib.check(rc)
        self._pending[rc] = (a, b, C, f, g, P, X, Y)
        return rc

    def poll(self, ticket):
        """The result dict once the request is finished, else None."""
        r = _lib.Result()
        rc = _lib.check(self._L.rwig_server_poll(self._h, int(ticket), ctypes.byref(r)))
        if rc == 0:
            return None
        a, b, C, f, g, P, X, Y = self._pending.pop(ticket)
        d = r.as_dict()
        out = {"f": f, "g": g, "loss": d["loss"], "iter": d["iter"], "err": d["err"], "return_status": d["status"],
               "marg_l1_row": d["marg_l1_row"], "marg_l1_col": d["marg_l1_col"]}
        if P is not None:
            out["P"] = P
        return out

    def close(self):
        if self._h:
            self._L.rwig_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


# ---------------------------------------------------------------------------
# device-resident entry points (torch CUDA tensors as plain device buffers)
# ---------------------------------------------------------------------------
def _ptr(t):
    if t is None:
        return None
    if not (t.is_cuda and t.dtype.is_floating_point and t.element_size() == 8 and t.is_contiguous()):
        raise ValueError("device buffers must be contiguous float64 CUDA tensors")
    return ctypes.c_void_p(t.data_ptr())


def sinkhorn_vanilla_device(a, b, C_cm, reg, max_iter=1000, zero_tol=1e-6, P=None, u=None, v=None,
                            stream=None, grad_a=None) -> dict:
    """Vanilla Sinkhorn on device buffers (layout as sinkhorn_log_device);
    grad_a (M, device) receives the gradient w.r.t. a when given."""
    M, N = a.shape[0], b.shape[0]
    if C_cm.numel() != M * N:
        raise ValueError("C must hold M*N entries")
    loss, err, it = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
    st = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
    rc = _lib.load().rwig_sinkhorn_vanilla_dev(_ptr(P), _ptr(grad_a), _ptr(u), _ptr(v), ctypes.byref(loss),
                                               ctypes.byref(it), ctypes.byref(err), _ptr(a), _ptr(b),
                                               _ptr(C_cm), M, N, float(reg), int(grad_a is not None), int(max_iter),
                                               float(zero_tol), st)
    _lib.check(rc)
    return {"loss": loss.value, "iter": it.value, "err": err.value, "return_status": rc}


def sinkhorn_log_device(a, b, C_cm, reg, max_iter=1000, zero_tol=1e-6, P=None, f=None, g=None,
                        stream=None, grad_a=None) -> dict:
    """Log-Sinkhorn on device buffers.  C_cm is the M x N cost in column-major
    order, i.e. a contiguous (N, M) tensor holding C^T row-major; P likewise.
    grad_a (M, device) receives the gradient w.r.t. a when given."""
    M, N = a.shape[0], b.shape[0]
    if C_cm.numel() != M * N:
        raise ValueError("C must hold M*N entries")
    loss, err, it = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
    st = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
    rc = _lib.load().rwig_sinkhorn_log_dev(_ptr(P), _ptr(grad_a), _ptr(f), _ptr(g), ctypes.byref(loss),
                                           ctypes.byref(it), ctypes.byref(err), _ptr(a), _ptr(b),
                                           _ptr(C_cm), M, N, float(reg), int(grad_a is not None), int(max_iter),
                                           float(zero_tol),
                                           st)
    _lib.check(rc)
    return {"loss": loss.value, "iter": it.value, "err": err.value, "return_status": rc}
