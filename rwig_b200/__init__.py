"""rwig_b200 -- B200-native (sm_100a) engine for rwig's entropic optimal transport.

Public Python surface (mirrors rwig's R API over the C ABI in include/rwig_b200.h):
    sinkhorn(a, b, C, sinkhorn_control)
    barycenter(A, C, w, b_ext, barycenter_control), batch_barycenter(problems)
    wdl_cpp(Y, C, reg, S, batch_size, epochs, ...), wdl_batch_grad(A, W_B, Y_B, K_or_C, reg, L, mode)
    wdl_batch_grad_dp(...): the same gradient with the batch split over torch.distributed ranks
    wdl_batch_grad_dp_dev(...): the same on device buffers, all-reduced on the device
    wdl_train_dp_dev(...): data-parallel WDL training on the device (gradient shards,
                           all-reduce, the same optimizer step on every rank)
    batch_sinkhorn_log(problems), Server: batched and served log-Sinkhorn
    autotune_batch(problems): picks the batched kernel's team shapes and schedule
The compute path is the CUDA library rwig_b200/librwig_b200.so; importing this
package does not load it until the first call.
"""
from ._lib import RwigError, last_report, load  # noqa: F401
from .autotune import autotune_batch  # noqa: F401
from .api import (Server, barycenter, batch_barycenter, batch_sinkhorn_log, check_barycenter_args, check_sinkhorn_args, choose_sinkhorn_method,  # noqa: F401
                  sinkhorn, sinkhorn_log_device, sinkhorn_vanilla_device, wdl_batch_grad, wdl_batch_grad_dp, wdl_batch_grad_dp_dev, wdl_cpp, wdl_train_dp_dev)

__all__ = ["autotune_batch", "batch_barycenter", "sinkhorn", "barycenter", "wdl_cpp", "wdl_batch_grad", "wdl_batch_grad_dp", "wdl_batch_grad_dp_dev", "wdl_train_dp_dev", "batch_sinkhorn_log", "Server", "sinkhorn_log_device", "sinkhorn_vanilla_device", "RwigError", "last_report", "load"]
