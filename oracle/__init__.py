"""CPU parity oracle for the rwig entropic-OT path -- TEST INFRASTRUCTURE ONLY.

ctypes bindings over ``oracle/_build/librwig_oracle.so`` (built from
``oracle/rwig_oracle.cpp`` by ``oracle/Makefile``), a C++ restatement of rwig's
Armadillo CPU code (src/sinkhorn_impl_*.cpp, src/barycenter_impl_*.cpp,
src/wdl_impl.cpp).  Only tests/, ``__graft_entry__.smoke()`` and ``bench.py``'s
CPU-baseline / reference arm may import this package.  The engine in
``rwig_b200`` never calls it.

Each wrapper returns a dict shaped like the R list the reference returns
(src/sinkhorn.cpp:28-43, src/barycenter.cpp:213-229, :360-376).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "librwig_oracle.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def build(force: bool = False) -> str:
    """Compile the oracle shared library with the committed Makefile."""
    src = os.path.join(_HERE, "rwig_oracle.cpp")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_REF_GPU_PATH = os.path.join(_HERE, "_ref", "librwig_ref_gpu.so")
_ref_gpu = None


def build_ref_gpu(ref_dir: str | None = None) -> str | None:
    """Compile rwig's own GPU vanilla Sinkhorn, parallel barycenter and WDL from
    the reference's sources (``make -C oracle ref REF=<dir>``).  The source tree
    is ``ref_dir`` or the environment variable ``RWIG_REFERENCE_DIR``; with
    neither set nothing is built and the prebuilt library (if any) is used."""
    src = ref_dir or os.environ.get("RWIG_REFERENCE_DIR")
    if src:
        if not os.path.isdir(os.path.join(src, "src")):
            raise RuntimeError(f"not an rwig source tree (no src/): {src}")
        subprocess.run(["make", "-s", "-C", _HERE, "ref", f"REF={src}"], check=True)
    return _REF_GPU_PATH if os.path.exists(_REF_GPU_PATH) else None


def ref_gpu_available() -> bool:
    return os.path.exists(_REF_GPU_PATH)


def ref_gpu():
    """The reference's GPU path (oracle/_ref), loaded on first use."""
    global _ref_gpu
    if _ref_gpu is None:
        if not os.path.exists(_REF_GPU_PATH):
            raise RuntimeError(f"reference GPU library not built: {_REF_GPU_PATH} (make -C oracle ref REF=...)")
        L = ctypes.CDLL(_REF_GPU_PATH)
        i, d = ctypes.c_int, ctypes.c_double
        L.ref_gpu_sinkhorn_vanilla.argtypes = [_dp, _dp, _dp, _dp, _dp, _ip, _dp, _dp, _dp, _dp, i, i, d, i, i, d]
        L.ref_gpu_sinkhorn_vanilla.restype = None
        L.ref_gpu_barycenter_parallel.argtypes = [_dp, _dp, _dp, _dp, _dp, _dp, _ip, _dp, _dp, _dp, _dp, _dp,
                                                  i, i, i, d, i, i, d]
        L.ref_gpu_barycenter_parallel.restype = None
        L.ref_gpu_wdl.argtypes = [_dp, _dp, _dp, _dp, _dp, i, i, i, d, i, d, i, i, i, d, d, d, d, d, i]
        L.ref_gpu_wdl.restype = None
        L.ref_gpu_wdl_batch_grad.argtypes = [_dp, _dp, _dp, _dp, _dp, _dp, i, i, i, d, i, i, i,
                                             ctypes.POINTER(ctypes.c_float)]
        L.ref_gpu_wdl_batch_grad.restype = i
        _ref_gpu = L
    return _ref_gpu


def ref_gpu_wdl_batch_grad(A, WB, YB, K_or_C, reg, L, mode=0, reps=1):
    """rwig's own unrolled GPU WDL batch gradient (wdl_batch, src/cuda_wdl.cu:385)
    on D = WB.shape[1] documents, host buffers.  Returns (g_Alpha, g_lambda,
    mean device ms of one wdl_batch call over `reps` calls)."""
    A, WB, YB, K_or_C = _f64(A), _f64(WB), _f64(YB), _f64(K_or_C)
    N, S = A.shape
    D = WB.shape[1]
    gA, gl = np.zeros((N, S), order="F"), np.zeros(S)
    ms = ctypes.c_float()
    rc = ref_gpu().ref_gpu_wdl_batch_grad(_ptr(gA), _ptr(gl), _ptr(A), _ptr(WB), _ptr(YB), _ptr(K_or_C), N, S, D,
                                          float(reg), int(L), int(mode), int(reps), ctypes.byref(ms))
    if rc != 0:
        raise RuntimeError(f"reference wdl_batch failed with CUDA error {rc}")
    return gA, gl, ms.value


def ref_gpu_wdl(Y, C, S, reg, max_iter, zero_tol, B, E, opt=1, eta=1e-3, gamma=0.01, beta1=0.9, beta2=0.999,
                eps=1e-8, seed=1):
    """rwig's own GPU WDL (cuda_wdl, src/cuda_wdl.cu:539): training from
    mt19937(seed) logits, then inference.  Returns A, W, Yhat."""
    Y, C = _f64(Y), _f64(C)
    N, M = Y.shape
    A, W, Yhat = np.zeros((N, S), order="F"), np.zeros((S, M), order="F"), np.zeros((N, M), order="F")
    ref_gpu().ref_gpu_wdl(_ptr(A), _ptr(W), _ptr(Yhat), _ptr(Y), _ptr(C), N, M, S, float(reg), int(max_iter),
                          float(zero_tol), int(B), int(E), int(opt), float(eta), float(gamma), float(beta1),
                          float(beta2), float(eps), int(seed))
    return dict(A=A, W=W, Yhat=Yhat)


def ref_gpu_sinkhorn_vanilla(a, b, C, reg, max_iter=1000, zero_tol=1e-6):
    """rwig's own GPU vanilla Sinkhorn (src/cuda_sinkhorn.cu:181), host buffers."""
    a, b = _f64(a).ravel(), _f64(b).ravel()
    C = _f64(C)
    M, N = C.shape
    P, u, v = np.zeros((M, N), order="F"), np.zeros(M), np.zeros(N)
    loss, err, it = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
    ref_gpu().ref_gpu_sinkhorn_vanilla(_ptr(P), None, _ptr(u), _ptr(v), ctypes.byref(loss), ctypes.byref(it),
                                       ctypes.byref(err), _ptr(a), _ptr(b), _ptr(C), M, N, float(reg), 0,
                                       int(max_iter), float(zero_tol))
    return {"P": P, "u": u, "v": v, "loss": loss.value, "iter": it.value, "err": err.value}


def ref_gpu_barycenter_parallel(A, C, w, b_ext=None, reg=0.1, with_grad=False, max_iter=1000, zero_tol=1e-6):
    """rwig's own GPU parallel barycenter (src/cuda_barycenter.cu:268), host buffers."""
    A, C = _f64(A), _f64(C)
    w = _f64(w).ravel()
    M, S = A.shape
    N = C.shape[1]
    U, V = np.zeros((M, S), order="F"), np.zeros((N, S), order="F")
    b = np.zeros(N)
    gA = np.zeros((M, S), order="F") if with_grad else None
    gw = np.zeros(S) if with_grad else None
    be = _f64(b_ext).ravel() if b_ext is not None else np.zeros(N)
    loss, err, it = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
    ref_gpu().ref_gpu_barycenter_parallel(_ptr(U), _ptr(V), _ptr(b), _ptr(gA), _ptr(gw), ctypes.byref(loss),
                                          ctypes.byref(it), ctypes.byref(err), _ptr(A), _ptr(w), _ptr(C), _ptr(be),
                                          M, N, S, float(reg), int(bool(with_grad)), int(max_iter), float(zero_tol))
    out = {"b": b, "U": U, "V": V, "iter": it.value, "err": err.value}
    if with_grad:
        out.update(grad_A=gA, grad_w=gw, loss=loss.value)
    return out


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        i, d = ctypes.c_int, ctypes.c_double
        L.oracle_sinkhorn_vanilla.argtypes = [_dp, _dp, _dp, _dp, _dp, _ip, _dp, _dp, _dp, _dp,
                                              i, i, d, i, i, d]
        L.oracle_sinkhorn_vanilla.restype = i
        L.oracle_sinkhorn_log.argtypes = [_dp, _dp, _dp, _dp, _dp, _ip, _dp, _dp, _dp, _dp,
                                          i, i, d, i, i, d, i]
        L.oracle_sinkhorn_log.restype = i
        L.oracle_barycenter_parallel.argtypes = [_dp, _dp, _dp, _dp, _dp, _dp, _ip, _dp, _dp, _dp,
                                                 _dp, _dp, i, i, i, d, i, i, d]
        L.oracle_barycenter_parallel.restype = i
        L.oracle_barycenter_log.argtypes = [_dp, _dp, _dp, _dp, _dp, _dp, _ip, _dp, _dp, _dp,
                                            _dp, _dp, i, i, i, d, i, i, d, i]
        L.oracle_barycenter_log.restype = i
        L.oracle_wdl_batch_grad.argtypes = [_dp, _dp, _dp, _dp, _dp, _dp, i, i, i, i]
        L.oracle_wdl_batch_grad.restype = None
        L.oracle_last_raw_b.argtypes = [_dp, i]
        L.oracle_last_raw_b.restype = i
        L.oracle_col_softmax.argtypes = [_dp, _dp, i, i]
        L.oracle_col_softmax.restype = None
        L.oracle_optimizer_step.argtypes = [_dp, _dp, _dp, _dp, ctypes.c_size_t, i, i, d, d, d, d, d]
        L.oracle_optimizer_step.restype = None
        L.oracle_wdl_train.argtypes = [_dp, _dp, _dp, _dp, _dp, _dp, i, i, i, d, i, i, i, i,
                                       d, d, d, d, d, i]
        L.oracle_wdl_train.restype = i
        _lib = L
    return _lib


def _f64(x, shape=None):
    a = np.asarray(x, dtype=np.float64)
    if shape is not None:
        a = a.reshape(shape)
    return np.asfortranarray(a)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_dp)


def sinkhorn_vanilla(a, b, C, reg, with_grad=False, max_iter=1000, zero_tol=1e-6):
    a, b, C = _f64(a).ravel(), _f64(b).ravel(), _f64(C)
    M, N = C.shape
    P = np.zeros((M, N), order="F")
    u, v, ga = np.zeros(M), np.zeros(N), np.zeros(M)
    loss, err, it = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
    rc = lib().oracle_sinkhorn_vanilla(_ptr(P), _ptr(ga), _ptr(u), _ptr(v), ctypes.byref(loss),
                                       ctypes.byref(it), ctypes.byref(err), _ptr(a), _ptr(b),
                                       _ptr(C), M, N, float(reg), int(bool(with_grad)),
                                       int(max_iter), float(zero_tol))
    out = dict(P=P, u=u, v=v, loss=loss.value, iter=it.value, err=err.value, return_status=rc)
    if with_grad:
        out["grad_a"] = ga
    return out


def sinkhorn_log(a, b, C, reg, with_grad=False, n_threads=0, max_iter=1000, zero_tol=1e-6,
                 want_P=True):
    a, b, C = _f64(a).ravel(), _f64(b).ravel(), _f64(C)
    M, N = C.shape
    P = np.zeros((M, N), order="F") if want_P else None
    f, g, ga = np.zeros(M), np.zeros(N), np.zeros(M)
    loss, err, it = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
    rc = lib().oracle_sinkhorn_log(_ptr(P), _ptr(ga), _ptr(f), _ptr(g), ctypes.byref(loss),
                                   ctypes.byref(it), ctypes.byref(err), _ptr(a), _ptr(b), _ptr(C),
                                   M, N, float(reg), int(bool(with_grad)), int(max_iter),
                                   float(zero_tol), int(n_threads))
    out = dict(P=P, f=f, g=g, loss=loss.value, iter=it.value, err=err.value, return_status=rc)
    if with_grad:
        out["grad_a"] = ga
    return out


def _raw_b(N):
    out = np.zeros(N)
    lib().oracle_last_raw_b(_ptr(out), N)
    return out


def barycenter_parallel(A, C, w, b_ext=None, reg=0.1, with_grad=False, max_iter=1000,
                        zero_tol=1e-6):
    A, C, w = _f64(A), _f64(C), _f64(w).ravel()
    M, S = A.shape
    N = C.shape[1]
    be = _f64(b_ext).ravel() if b_ext is not None else np.zeros(N)
    U, V = np.zeros((M, S), order="F"), np.zeros((N, S), order="F")
    b, gA, gw = np.zeros(N), np.zeros((M, S), order="F"), np.zeros(S)
    loss, err, it = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
    rc = lib().oracle_barycenter_parallel(_ptr(U), _ptr(V), _ptr(b), _ptr(gA), _ptr(gw),
                                          ctypes.byref(loss), ctypes.byref(it), ctypes.byref(err),
                                          _ptr(A), _ptr(w), _ptr(C), _ptr(be), M, N, S, float(reg),
                                          int(bool(with_grad)), int(max_iter), float(zero_tol))
    out = dict(b=b, U=U, V=V, iter=it.value, err=err.value, return_status=rc, b_raw=_raw_b(N))
    if with_grad:
        out.update(grad_A=gA, grad_w=gw, loss=loss.value)
    return out


def barycenter_log(A, C, w, b_ext=None, reg=0.1, with_grad=False, n_threads=0, max_iter=1000,
                   zero_tol=1e-6):
    A, C, w = _f64(A), _f64(C), _f64(w).ravel()
    M, S = A.shape
    N = C.shape[1]
    be = _f64(b_ext).ravel() if b_ext is not None else np.zeros(N)
    F, G = np.zeros((M, S), order="F"), np.zeros((N, S), order="F")
    b, gA, gw = np.zeros(N), np.zeros((M, S), order="F"), np.zeros(S)
    loss, err, it = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
    rc = lib().oracle_barycenter_log(_ptr(F), _ptr(G), _ptr(b), _ptr(gA), _ptr(gw),
                                     ctypes.byref(loss), ctypes.byref(it), ctypes.byref(err),
                                     _ptr(A), _ptr(w), _ptr(C), _ptr(be), M, N, S, float(reg),
                                     int(bool(with_grad)), int(max_iter), float(zero_tol),
                                     int(n_threads))
    out = dict(b=b, F=F, G=G, iter=it.value, err=err.value, return_status=rc, b_raw=_raw_b(N))
    if with_grad:
        out.update(grad_A=gA, grad_w=gw, loss=loss.value)
    return out


def wdl_batch_grad(A, WB, YB, K, L):
    A, WB, YB, K = _f64(A), _f64(WB), _f64(YB), _f64(K)
    N, S = A.shape
    D = WB.shape[1]
    gA, gl = np.zeros((N, S), order="F"), np.zeros(S)
    lib().oracle_wdl_batch_grad(_ptr(gA), _ptr(gl), _ptr(A), _ptr(WB), _ptr(YB), _ptr(K), N, S, D,
                                int(L))
    return gA, gl


def col_softmax(X):
    X = _f64(X)
    out = np.zeros_like(X, order="F")
    lib().oracle_col_softmax(_ptr(out), _ptr(X), X.shape[0], X.shape[1])
    return out


def wdl_train(Y, C, S, reg, L, B, E, Alpha0, Lambda0, opt=1, eta=1e-3, gamma=0.01, beta1=0.9,
              beta2=0.999, eps=1e-8, max_steps=0):
    Y, C = _f64(Y), _f64(C)
    N, M = Y.shape
    Alpha = _f64(Alpha0).copy(order="F")
    Lambda = _f64(Lambda0).copy(order="F")
    A, W = np.zeros((N, S), order="F"), np.zeros((S, M), order="F")
    steps = lib().oracle_wdl_train(_ptr(A), _ptr(W), _ptr(Alpha), _ptr(Lambda), _ptr(Y), _ptr(C),
                                   N, M, S, float(reg), int(L), int(B), int(E), int(opt),
                                   float(eta), float(gamma), float(beta1), float(beta2), float(eps),
                                   int(max_steps))
    return dict(A=A, W=W, Alpha=Alpha, Lambda=Lambda, steps=steps)
