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
