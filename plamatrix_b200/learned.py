"""Training and evaluation protocol of the learned block-Jacobi correction (no counterpart in
the reference).

An LM sequence of a two-block problem: iteration k perturbs the Jacobian blocks by 10% relative
N(0,1) noise and moves lambda by a factor drawn from {0.5, 2} (starting at 1e-3).  Every
iteration's system is assembled and solved with plain FP64 block-Jacobi PCG; its reduced
solution x and right-hand side b train the network (Adam steps of
LearnedPreconditioner.train_step).  Evaluation solves held-out iterations and unseen seeds both
ways and reports iterations and time to the FP64 true relative residual.
"""
from __future__ import annotations

import time
from dataclasses import dataclass

import numpy as np
import torch

from . import schur as SC


@dataclass
class LMSystem:
    lam: float
    jp: torch.Tensor
    jl: torch.Tensor


def lm_sequence(problem: dict, iterations: int, seed: int, noise: float = 0.1, lam0: float = 1e-3):
    """Perturbed Jacobians and lambdas of `iterations` LM steps (device tensors)."""
    g = torch.Generator(device="cuda")
    g.manual_seed(int(seed) + 7919)
    jp0 = problem["jp"] if torch.is_tensor(problem["jp"]) else torch.from_numpy(problem["jp"]).cuda()
    jl0 = problem["jl"] if torch.is_tensor(problem["jl"]) else torch.from_numpy(problem["jl"]).cuda()
    lam = lam0
    for _ in range(iterations):
        lam *= 0.5 if torch.rand((), generator=g, device="cuda").item() < 0.5 else 2.0
        jp = jp0 * (1.0 + noise * torch.randn(jp0.shape, generator=g, device="cuda", dtype=jp0.dtype))
        jl = jl0 * (1.0 + noise * torch.randn(jl0.shape, generator=g, device="cuda", dtype=jl0.dtype))
        yield LMSystem(lam, jp, jl)


def _device(problem: dict, key: str) -> torch.Tensor:
    v = problem[key]
    return v if torch.is_tensor(v) else torch.from_numpy(np.ascontiguousarray(v)).cuda()


class LMRunner:
    """Normal equations, workspace and indices of one problem, reused across its LM systems."""

    def __init__(self, problem: dict):
        self.problem = problem
        self.ne = SC.DeviceNormalEquations(problem["P"], problem["L"], 6, 3)
        self.ws = SC.SchurComplementSolverWorkspace()
        self.op = _device(problem, "obs_primary")
        self.ol = _device(problem, "obs_eliminated")
        self.res = _device(problem, "residual")
        n, m = problem["P"] * 6, problem["L"] * 3
        self.dp = torch.zeros(n, dtype=torch.float64, device="cuda")
        self.dl = torch.zeros(m, dtype=torch.float64, device="cuda")

    def solve(self, system: LMSystem, options: SC.SchurComplementSolverOptions):
        self.ne.accumulate_observations(self.op, self.ol, system.jp, system.jl, self.res, self.problem["huber_delta"])
        return SC.solve_damped_schur_complement(self.ne, system.lam, options, self.ws, self.dp, self.dl)


def train(net: SC.LearnedPreconditioner, runners: list, sequences: list, steps_per_system: int = 20,
          learning_rate: float = 2e-3, tolerance: float = 1e-8, max_iterations: int = 500) -> list:
    """Train on every system of every sequence; returns the mean loss of each system's first
    and last Adam step, in order."""
    plain = SC.SchurComplementSolverOptions(max_iterations=max_iterations, relative_tolerance=tolerance)
    history = []
    for runner, seq in zip(runners, sequences):
        for system in seq:
            dp, _, rep = runner.solve(system, plain)
            if not rep["converged"]:
                continue
            b = runner.ws.export()["rhs"]
            x = dp.clone()
            first = net.train_step(runner.ws, x, b, learning_rate)
            for _ in range(steps_per_system - 1):
                last = net.train_step(runner.ws, x, b, learning_rate)
            history.append((first, last))
    return history


def evaluate(net: SC.LearnedPreconditioner, runners: list, sequences: list, tolerance: float = 1e-8,
             max_iterations: int = 500, precision: str = "mixed") -> list:
    """Each held-out system solved with plain FP64 block Jacobi and with the learned correction
    (`precision` pipeline): iterations, solve time (ms) and true relative residual of both."""
    plain = SC.SchurComplementSolverOptions(max_iterations=max_iterations, relative_tolerance=tolerance)
    learned = SC.SchurComplementSolverOptions(max_iterations=max_iterations, relative_tolerance=tolerance,
                                              precision=precision, learned=net)
    rows = []
    for runner, seq in zip(runners, sequences):
        for system in seq:
            out = {"lambda": system.lam}
            for name, opts in (("plain", plain), ("learned", learned)):
                runner.solve(system, opts)  # warm (pattern, buffers)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                _, _, rep = runner.solve(system, opts)
                torch.cuda.synchronize()
                out[name] = {"iterations": rep["iterations"], "ms": (time.perf_counter() - t0) * 1e3,
                             "converged": rep["converged"], "true_relative_residual": rep["true_relative_residual"],
                             "fallback": rep.get("learned_fallback", False)}
            rows.append(out)
    return rows
