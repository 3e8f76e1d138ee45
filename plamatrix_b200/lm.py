"""Caller side of the LM loop: LevenbergMarquardtOptions / LevenbergMarquardtStrategy
(include/plamatrix/optimization/levenberg_marquardt.h:13-95) and the robust cost of a set of
device residuals (evaluateHuberLoss per residual, robust_loss.h:27-51, summed on the device)."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import torch

from . import _native as N
from .sparse import _ptr, _stream_handle

HUBER_COST_SCRATCH = 1024  # doubles of device scratch per cost evaluation (PM_HUBER_COST_SCRATCH)


class _Options(C.Structure):
    _fields_ = [("initial_damping", C.c_double), ("minimum_damping", C.c_double), ("maximum_damping", C.c_double),
                ("decrease_factor", C.c_double), ("increase_factor", C.c_double)]


N.register("pm_lm_options_default", [C.c_void_p], None)
N.register("pm_lm_strategy_create_f32", [C.c_void_p, C.c_void_p])
N.register("pm_lm_strategy_create_f64", [C.c_void_p, C.c_void_p])
N.register("pm_lm_strategy_destroy", [C.c_void_p], None)
N.register("pm_lm_accept_step", [C.c_void_p])
N.register("pm_lm_reject_step", [C.c_void_p])
N.register("pm_lm_strategy_state", [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p])
N.register("pm_huber_cost_f32", [C.c_void_p, C.c_int64, C.c_int64, C.c_void_p, C.c_float, C.c_void_p, C.c_void_p])
N.register("pm_huber_cost_f64", [C.c_void_p, C.c_int64, C.c_int64, C.c_void_p, C.c_double, C.c_void_p,
                                 C.c_void_p])


@dataclass
class LevenbergMarquardtOptions:
    initial_damping: float = 1e-3
    minimum_damping: float = 1e-12
    maximum_damping: float = 1e12
    decrease_factor: float = 0.3
    increase_factor: float = 10.0


class LevenbergMarquardtStrategy:
    """Damping and accepted / rejected step counts; the damping is updated in the strategy's
    scalar type (`dtype` float32 or float64, the reference's template argument)."""

    def __init__(self, options: LevenbergMarquardtOptions | None = None, dtype=torch.float64):
        o = options or LevenbergMarquardtOptions()
        c = _Options(o.initial_damping, o.minimum_damping, o.maximum_damping, o.decrease_factor, o.increase_factor)
        h = C.c_void_p()
        sfx = "f32" if dtype == torch.float32 else "f64"
        N.call(f"pm_lm_strategy_create_{sfx}", C.byref(c), C.byref(h))
        self._h = h

    def accept_step(self) -> None:
        N.call("pm_lm_accept_step", self._h)

    def reject_step(self) -> None:
        N.call("pm_lm_reject_step", self._h)

    def _state(self):
        d, a, r = C.c_double(), C.c_int(), C.c_int()
        N.call("pm_lm_strategy_state", self._h, C.byref(d), C.byref(a), C.byref(r))
        return d.value, a.value, r.value

    def damping(self) -> float:
        return self._state()[0]

    def accepted_steps(self) -> int:
        return self._state()[1]

    def rejected_steps(self) -> int:
        return self._state()[2]

    def __del__(self):
        h = getattr(self, "_h", None)
        try:
            if h is not None and N._lib is not None:
                N._lib.pm_lm_strategy_destroy(h)
        except (AttributeError, TypeError):  # interpreter shutdown
            pass
        self._h = None


def huber_cost(residual: torch.Tensor, delta: float, out: torch.Tensor | None = None,
               scratch: torch.Tensor | None = None, stream=None) -> torch.Tensor:
    """Sum over residual rows (count x m, row-major) of evaluateHuberLoss(|r|^2, delta).cost,
    as a 0-d float64 device tensor; non-finite when a residual's squared norm is not finite."""
    if not residual.is_cuda or not residual.is_contiguous() or residual.dtype not in (torch.float32, torch.float64):
        raise N.InvalidArgument("residual must be a contiguous float32 or float64 CUDA tensor")
    count = residual.shape[0] if residual.dim() > 0 else 0
    m = residual.numel() // count if count else 1
    cost = torch.empty((), dtype=torch.float64, device=residual.device) if out is None else out
    work = torch.empty(HUBER_COST_SCRATCH, dtype=torch.float64, device=residual.device) if scratch is None else scratch
    if work.numel() < HUBER_COST_SCRATCH or work.dtype != torch.float64:
        raise N.InvalidArgument(f"scratch must hold {HUBER_COST_SCRATCH} float64 values")
    sfx = "f32" if residual.dtype == torch.float32 else "f64"
    N.call(f"pm_huber_cost_{sfx}", _stream_handle(stream), count, m, _ptr(residual), float(delta), _ptr(work),
           _ptr(cost))
    return cost
