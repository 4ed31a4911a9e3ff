"""rwig_b200 -- B200-native (sm_100a) engine for rwig's entropic optimal transport.

Public Python surface (mirrors rwig's R API over the C ABI in include/rwig_b200.h):
    sinkhorn(a, b, C, sinkhorn_control)
    barycenter(A, C, w, b_ext, barycenter_control)
The compute path is the CUDA library rwig_b200/librwig_b200.so; importing this
package does not load it until the first call.
"""
from ._lib import RwigError, last_report, load  # noqa: F401
from .api import (barycenter, check_barycenter_args, check_sinkhorn_args, choose_sinkhorn_method,  # noqa: F401
                  sinkhorn, sinkhorn_log_device, sinkhorn_vanilla_device)

__all__ = ["sinkhorn", "barycenter", "sinkhorn_log_device", "sinkhorn_vanilla_device", "RwigError", "last_report", "load"]
