"""ctypes loader for the engine's C ABI (include/rwig_b200.h).

The shared library is built in-tree (rwig_b200/librwig_b200.so).  There is no
fallback: when the library is missing or no sm_100 device is present, calls
fail loudly with RwigError.
"""
from __future__ import annotations

import ctypes
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librwig_b200.so")
HEADER = os.path.join(HERE, "..", "include", "rwig_b200.h")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_vp = ctypes.c_void_p
_i, _d = ctypes.c_int, ctypes.c_double

ERRORS = {
    -1: "RWIG_E_INVALID",
    -2: "RWIG_E_CUDA",
    -3: "RWIG_E_NODEVICE",
    -4: "RWIG_E_NOMEM",
    -5: "RWIG_E_TIMEOUT",
    -6: "RWIG_E_UNSUPPORTED",
    -7: "RWIG_E_BUSY",
}


class RwigError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class Report(ctypes.Structure):
    _fields_ = [
        ("iter", _i),
        ("status", _i),
        ("err", _d),
        ("marg_l1_row", _d),
        ("marg_l1_col", _d),
        ("marg_l2_row", _d),
        ("marg_l2_col", _d),
        ("device_ms", _d),
        ("kernel_ms", _d),
        ("sweep_ms", _d),
        ("sweep_iters", _i),
        ("fallback_events", _i),
        ("kernel_launches", _i),
        ("support_m", _i),
        ("support_n", _i),
        ("bary_norm", _d),
        ("grad_ms", _d),
        ("gemm_ms", _d),
        ("gemm_launches", _i),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Problem(ctypes.Structure):
    """rwig_problem (include/rwig_b200.h)."""
    _fields_ = [("a", _vp), ("b", _vp), ("C", _vp), ("M", _i), ("N", _i), ("reg", _d), ("max_iter", _i),
                ("zero_tol", _d), ("P", _vp), ("f", _vp), ("g", _vp), ("X", _vp), ("Y", _vp), ("d", _i)]


class BaryProblem(ctypes.Structure):
    """rwig_bary_problem (include/rwig_b200.h)."""
    _fields_ = [("A", _vp), ("w", _vp), ("C", _vp), ("b_ext", _vp), ("M", _i), ("N", _i), ("S", _i), ("reg", _d),
                ("method", _i), ("withgrad", _i), ("max_iter", _i), ("zero_tol", _d), ("X1", _vp), ("X2", _vp),
                ("b", _vp), ("grad_A", _vp), ("grad_w", _vp)]


class BaryResult(ctypes.Structure):
    """rwig_bary_result (include/rwig_b200.h)."""
    _fields_ = [("loss", _d), ("err", _d), ("iter", _i), ("status", _i)]


class Result(ctypes.Structure):
    """rwig_result (include/rwig_b200.h)."""
    _fields_ = [("loss", _d), ("err", _d), ("iter", _i), ("status", _i), ("marg_l1_row", _d),
                ("marg_l1_col", _d), ("device_us", _d), ("path", _i), ("reserved", _i)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


# name -> (restype, argtypes)
SIGNATURES = {
    "rwig_init": (_i, [_i]),
    "rwig_shutdown": (None, []),
    "rwig_last_error": (ctypes.c_char_p, []),
    "rwig_version": (_i, []),
    "rwig_last_report": (_i, [ctypes.POINTER(Report)]),
    "rwig_set_option": (_i, [ctypes.c_char_p, _d]),
    "rwig_get_option": (_i, [ctypes.c_char_p, ctypes.POINTER(_d)]),
    "rwig_sinkhorn_vanilla": (_i, [_dp, _dp, _dp, _dp, _dp, _ip, _dp, _dp, _dp, _dp, _i, _i, _d, _i, _i, _d]),
    "rwig_sinkhorn_vanilla_dev": (_i, [_vp, _vp, _vp, _vp, _dp, _ip, _dp, _vp, _vp, _vp, _i, _i, _d, _i, _i,
                                       _d, _vp]),
    "rwig_sinkhorn_log": (_i, [_dp, _dp, _dp, _dp, _dp, _ip, _dp, _dp, _dp, _dp, _i, _i, _d, _i, _i, _d]),
    "rwig_sinkhorn_log_dev": (_i, [_vp, _vp, _vp, _vp, _dp, _ip, _dp, _vp, _vp, _vp, _i, _i, _d, _i, _i,
                                   _d, _vp]),
    "rwig_barycenter_parallel": (_i, [_dp, _dp, _dp, _dp, _dp, _dp, _ip, _dp, _dp, _dp, _dp, _dp, _i, _i, _i,
                                      _d, _i, _i, _d]),
    "rwig_barycenter_log": (_i, [_dp, _dp, _dp, _dp, _dp, _dp, _ip, _dp, _dp, _dp, _dp, _dp, _i, _i, _i, _d, _i,
                                 _i, _d]),
    "rwig_barycenter_parallel_dev": (_i, [_vp, _vp, _vp, _vp, _vp, _dp, _ip, _dp, _vp, _vp, _vp, _vp, _i, _i,
                                          _i, _d, _i, _i, _d, _vp]),
    "rwig_barycenter_log_dev": (_i, [_vp, _vp, _vp, _vp, _vp, _dp, _ip, _dp, _vp, _vp, _vp, _vp, _i, _i, _i, _d,
                                     _i, _i, _d, _vp]),
    "rwig_selftest_exp": (_i, [_vp, _vp, _vp, _i, _vp]),
    "rwig_selftest_dgemm": (_i, [_vp, ctypes.c_longlong, _i, _i, _i, _i, _vp, ctypes.c_longlong, _vp,
                                 ctypes.c_longlong, _i, _vp]),
    "rwig_selftest_i8gemm": (_i, [_vp, _vp, _i, _i, _i, _vp, _vp]),
    "rwig_selftest_ozaki": (_i, [_vp, ctypes.c_longlong, _i, _i, _vp, ctypes.c_longlong, _i, _vp, ctypes.c_longlong,
                                 _vp]),
    "rwig_sinkhorn_log_noalloc": (_i, [_vp, _vp, _vp, _dp, _ip, _dp, _vp, _vp, _vp, _i, _i, _d, _i, _d, _vp]),
    "rwig_wdl": (_i, [_dp, _dp, _dp, _dp, _dp, _i, _i, _i, _d, _i, _d, _i, _i, _i, _d, _d, _d, _d, _d, _i, _i,
                      _dp, _dp, _i]),
    "rwig_wdl_batch_grad": (_i, [_dp, _dp, _dp, _dp, _dp, _dp, _i, _i, _i, _d, _i, _i]),
    "rwig_wdl_batch_grad_dev": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _i, _i, _i, _d, _i, _i, _vp]),
    "rwig_wdl_update_dev": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i, _i, _i, _i, _d, _d, _d, _d,
                                 _d, _i, _vp]),
    "rwig_batch_sinkhorn_log": (_i, [ctypes.POINTER(Problem), _i, ctypes.POINTER(Result)]),
    "rwig_batch_sinkhorn_log_dev": (_i, [ctypes.POINTER(Problem), _i, ctypes.POINTER(Result), _vp]),
    "rwig_batch_barycenter_dev": (_i, [ctypes.POINTER(BaryProblem), _i, ctypes.POINTER(BaryResult), _vp]),
    "rwig_server_create": (_i, [ctypes.POINTER(_vp), _d, _d]),
    "rwig_server_submit": (_i, [_vp, ctypes.POINTER(Problem)]),
    "rwig_server_poll": (_i, [_vp, _i, ctypes.POINTER(Result)]),
    "rwig_server_destroy": (_i, [_vp]),
}

_lib = None


def header_symbols(path: str = HEADER):
    """Names of every function the public header declares."""
    src = open(path).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(rwig_[a-z0-9_]+)\s*\(", src)))


def load(build_if_missing: bool = False):
    """Load (once) and type the shared library."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        if build_if_missing:
            from . import build as _build
            _build.build()
        else:
            raise RwigError(-3, f"engine library not built: {LIB_PATH} (run python -m rwig_b200.build)")
    L = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def check(rc: int) -> int:
    if rc < 0:
        msg = load().rwig_last_error()
        raise RwigError(rc, msg.decode() if msg else "")
    return rc


def last_report() -> dict:
    r = Report()
    check(load().rwig_last_report(ctypes.byref(r)))
    return r.as_dict()
