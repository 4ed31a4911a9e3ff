"""Host-side logic of the R-mirroring API: control lists, validation messages,
automatic method choice (R/sinkhorn.R, R/check_args.R).  No device work."""
import numpy as np
import pytest

import rwig_b200 as rw


def test_defaults_filled():
    c = rw.check_sinkhorn_args({})
    assert c["reg"] == 0.1 and c["max_iter"] == 1000 and c["zero_tol"] == 1e-6
    assert c["method"] == "auto" and c["threshold"] == 0.1 and c["with_grad"] is False


def test_unknown_control_argument():
    with pytest.raises(ValueError, match="not matching one of the sinkhorn arguments"):
        rw.check_sinkhorn_args({"regg": 1})


def test_bad_method():
    with pytest.raises(ValueError, match="method must be from"):
        rw.check_sinkhorn_args({"method": "exact"})


def test_auto_method_rule():
    C = np.array([[0.0, 1.0], [1.0, 0.0]])
    # exp(-1/0.1) = 4.5e-5 < 0.1 -> log
    assert rw.choose_sinkhorn_method(C, 0.1, 0.1) == "log"
    # exp(-1/10) = 0.9 >= 0.1 -> vanilla
    assert rw.choose_sinkhorn_method(C, 10.0, 0.1) == "vanilla"


@pytest.mark.parametrize("a,b,C,msg", [
    (np.ones((2, 2)), np.ones(2), np.ones((2, 2)), "a must be a numeric vector"),
    (np.ones(2), np.ones((2, 1)), np.ones((2, 2)), "b must be a numeric vector"),
    (np.ones(2), np.ones(2), np.ones(4), "C must be a numeric matrix"),
    (np.ones(3), np.ones(2), np.ones((2, 2)), "don't match in dimension"),
])
def test_input_validation(a, b, C, msg):
    with pytest.raises(ValueError, match=msg):
        rw.sinkhorn(a, b, C)


def test_reg_must_be_scalar():
    with pytest.raises(ValueError, match="reg must be a single value"):
        rw.sinkhorn(np.ones(2) / 2, np.ones(2) / 2, np.eye(2), {"reg": [0.1, 0.2]})


def test_dp_training_needs_common_initial_logits():
    """Every rank must start from the same logits: the data-parallel training
    refuses to draw them itself (checked before any device work)."""
    import numpy as np
    with pytest.raises(ValueError, match="Alpha0 and Lambda0"):
        rw.wdl_train_dp_dev(np.ones((5, 3)), np.zeros((5, 5)), 2)


def test_update_entry_validates_before_any_device_work(engine):
    """rwig_wdl_update_dev rejects null buffers, sizes and step counts below 1
    and unknown optimizers with RWIG_E_INVALID, without a GPU."""
    import ctypes
    buf = (ctypes.c_double * 16)()
    p = ctypes.cast(buf, ctypes.c_void_p)
    args = [p] * 10 + [2, 2, 2, 1, 1e-3, 0.01, 0.9, 0.999, 1e-8, 1, None]
    bad = list(args)
    bad[0] = None
    assert engine.rwig_wdl_update_dev(*bad) == -1
    bad = list(args)
    bad[19] = 0  # step
    assert engine.rwig_wdl_update_dev(*bad) == -1
    bad = list(args)
    bad[13] = 3  # optimizer
    assert engine.rwig_wdl_update_dev(*bad) == -1
