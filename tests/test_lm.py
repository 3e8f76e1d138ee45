"""LevenbergMarquardtStrategy through the C ABI (host state only, no GPU): the reference's known
answer (test/unit/optimization/block_schur_test.cpp:550-569), clamping and option validation
(include/plamatrix/optimization/levenberg_marquardt.h:36-55)."""
import numpy as np
import pytest
import torch

from plamatrix_b200 import _native as N
from plamatrix_b200 import lm as LM


def test_accepted_and_rejected_steps_update_damping_and_counters():
    s = LM.LevenbergMarquardtStrategy(LM.LevenbergMarquardtOptions(1e-3, 1e-8, 1e4, 0.25, 8.0))
    s.accept_step()
    assert s.damping() == 2.5e-4 and s.accepted_steps() == 1 and s.rejected_steps() == 0
    s.reject_step()
    assert s.damping() == 2e-3 and s.accepted_steps() == 1 and s.rejected_steps() == 1


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_damping_is_clamped_and_follows_the_scalar_type(dtype):
    o = LM.LevenbergMarquardtOptions(1e-3, 1e-6, 1e2, 0.3, 10.0)
    s = LM.LevenbergMarquardtStrategy(o, dtype)
    scalar = np.float32 if dtype == torch.float32 else np.float64
    d = scalar(1e-3)
    for _ in range(20):
        s.accept_step()
        d = max(scalar(1e-6), d * scalar(0.3))
        assert s.damping() == float(d)
    assert s.damping() == float(scalar(1e-6))
    for _ in range(20):
        s.reject_step()
        d = min(scalar(1e2), d * scalar(10.0))
        assert s.damping() == float(d)
    assert s.damping() == float(scalar(1e2)) and s.accepted_steps() == 20 and s.rejected_steps() == 20


def test_default_options():
    s = LM.LevenbergMarquardtStrategy()
    assert s.damping() == 1e-3
    s.reject_step()
    assert s.damping() == 1e-2


@pytest.mark.parametrize("kw", [dict(minimum_damping=0.0), dict(maximum_damping=1e-14),
                                dict(initial_damping=1e-13), dict(initial_damping=1e13),
                                dict(decrease_factor=1.0), dict(decrease_factor=0.0),
                                dict(increase_factor=1.0), dict(minimum_damping=float("nan")),
                                dict(maximum_damping=float("inf"))])
def test_invalid_options_are_rejected(kw):
    with pytest.raises(N.InvalidArgument, match="invalid damping options"):
        LM.LevenbergMarquardtStrategy(LM.LevenbergMarquardtOptions(**kw))
