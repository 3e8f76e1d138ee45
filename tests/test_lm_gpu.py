"""Device robust cost of an LM trial step against evaluateHuberLoss restated in numpy
(robust_loss.h:27-51: 0.5 s inside delta, delta sqrt(s) - 0.5 delta^2 outside), and its use in
an accept / reject decision with the strategy."""
import numpy as np
import pytest
import torch

from plamatrix_b200 import _native as N
from plamatrix_b200 import lm as LM
from plamatrix_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _costs(res, delta):
    s = np.zeros(res.shape[0], dtype=res.dtype)
    for k in range(res.shape[1]):  # the device's order: rounded square, rounded add
        s = s + res[:, k] * res[:, k]
    d = res.dtype.type(delta)
    inside = (d == 0) | (s <= d * d)
    with np.errstate(invalid="ignore"):
        outside = d * np.sqrt(s) - (res.dtype.type(0.5) * d) * d
    return np.where(inside, res.dtype.type(0.5) * s, outside)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("m", [1, 2, 3])
def test_huber_cost_matches_evaluate_huber_loss(dtype, m):
    prob = W.bundle_problem(50, 3000, per_eliminated=4, residual_size=m, seed=m, dtype=dtype)
    res = prob["residual"].reshape(len(prob["obs_primary"]), m)
    expected = float(np.sum(_costs(res, prob["huber_delta"]).astype(np.float64)))
    t = torch.as_tensor(res).cuda()
    a = LM.huber_cost(t, prob["huber_delta"]).item()
    b = LM.huber_cost(t, prob["huber_delta"]).item()
    assert a == b  # fixed reduction order
    assert abs(a - expected) <= 1e-12 * abs(expected)
    # delta 0: plain least squares
    ls = float(np.sum(_costs(res, 0.0).astype(np.float64)))
    assert abs(LM.huber_cost(t, 0.0).item() - ls) <= 1e-12 * ls


def test_huber_cost_edge_cases_and_lm_decision():
    z = torch.zeros((0, 2), dtype=torch.float64, device="cuda")
    assert LM.huber_cost(z, 1.0).item() == 0.0
    r = torch.tensor([[3.0, 4.0], [0.1, 0.2]], dtype=torch.float64, device="cuda")
    # |r0| = 5 > delta 1: 5 - 0.5; |r1|^2 = 0.05 inside: 0.025
    assert abs(LM.huber_cost(r, 1.0).item() - (4.5 + 0.025)) < 1e-15
    bad = r.clone()
    bad[1, 0] = float("nan")
    assert not np.isfinite(LM.huber_cost(bad, 1.0).item())
    with pytest.raises(N.InvalidArgument):
        LM.huber_cost(r, -1.0)
    # an LM step: accept when the trial cost is finite and lower, else reject
    s = LM.LevenbergMarquardtStrategy()
    current = LM.huber_cost(r, 1.0).item()
    for trial in (r * 0.5, bad, r * 2.0):
        c = LM.huber_cost(trial, 1.0).item()
        if np.isfinite(c) and c < current:
            s.accept_step()
            current = c
        else:
            s.reject_step()
    assert s.accepted_steps() == 1 and s.rejected_steps() == 2
    assert s.damping() == pytest.approx(1e-3 * 0.3 * 10.0 * 10.0)
