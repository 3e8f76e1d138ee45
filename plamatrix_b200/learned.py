"""Training and evaluation protocol of the learned block-Jacobi correction (no counterpart in
the reference).

An LM sequence of a two-block problem: iteration k perturbs the Jacobian blocks by 10% relative
N(0,1) noise and moves lambda by a factor drawn from {0.5, 2} (starting at 1e-3).  Every
iteration's system is assembled and trains the network.  Two losses are offered:
  - probe_train: the preconditioned operator along Rademacher probes v,
    ||(I - M S) v||^2 / ||v||^2 with S v from the device SpMV (LearnedPreconditioner.train_probe_step);
    it needs no solve, and it measures what PCG convergence depends on;
  - train: the block-diagonal fit sum_p ||A_p x_p - b_p||^2 / ||b||^2 along each system's solved
    step x (LearnedPreconditioner.train_step).
Evaluation solves held-out iterations and unseen seeds both ways and reports iterations and time
to the FP64 true relative residual.
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


def assemble(runner: "LMRunner", system: LMSystem) -> None:
    """Accumulate and assemble one LM system in the runner's workspace (a one-iteration plain
    solve: the assembled FP64 system stays in the workspace)."""
    runner.solve(system, SC.SchurComplementSolverOptions(max_iterations=1, relative_tolerance=1e-30))


def probe_train(net: SC.LearnedPreconditioner, systems, probes_per_system: int = 4, epochs: int = 1,
                learning_rate: float = 1e-3, seed: int = 0) -> list:
    """Probe-loss training.  `systems` yields (workspace, block rows) pairs whose workspaces hold an
    assembled FP64 system (callable: re-assembles before use); one Adam step per Rademacher probe.
    Returns the mean loss of every epoch."""
    g = torch.Generator(device="cuda")
    g.manual_seed(int(seed) + 104729)
    history = []
    for _ in range(epochs):
        losses = []
        for item in systems():
            ws, P = item
            for _ in range(probes_per_system):
                v = torch.randint(0, 2, (6 * P,), generator=g, device="cuda").to(torch.float64) * 2.0 - 1.0
                losses.append(net.train_probe_step(ws, v, ws.spmv(v), learning_rate))
        history.append(float(np.mean(losses)) if losses else float("nan"))
    return history


def lm_probe_systems(runners: list, sequences: list):
    """Callable for probe_train over LM sequences: assembles each system in turn."""
    def gen():
        for runner, seq in zip(runners, sequences):
            for system in seq:
                assemble(runner, system)
                yield runner.ws, runner.problem["P"]
    return gen


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


def c3_protocol(net: SC.LearnedPreconditioner, P: int, L: int, train_seeds=range(8), unseen_seeds=range(100, 104),
                train_iterations: int = 20, test_iterations: int = 10, probes_per_system: int = 4, epochs: int = 2,
                learning_rate: float = 1e-3, tolerance: float = 1e-8, precision: str = "mixed_fp32_assembly") -> dict:
    """The learned-preconditioner protocol on the large windowed LM problem: LM sequences of
    train_iterations + test_iterations systems per seed (Jacobians x (1 + 0.1 N(0,1)), lambda x
    {0.5, 2} from 1e-3); probe-loss training on the first train_iterations systems of every training
    seed (`epochs` passes, `probes_per_system` Rademacher probes each); evaluation on the remaining
    test_iterations systems of every training seed and of every unseen seed, block Jacobi (FP64)
    against the learned correction (`precision` pipeline).  Problems are drawn on the device and
    dropped after use, one seed at a time."""
    from . import workloads as W

    total = train_iterations + test_iterations
    t0 = time.perf_counter()
    losses = []
    for epoch in range(epochs):
        epoch_losses = []
        for seed in train_seeds:
            prob = W.bundle_problem_device(P, L, per_eliminated="2+poisson4", window=40, seed=seed)
            runner = LMRunner(prob)
            seq = list(lm_sequence(prob, total, seed=seed))[:train_iterations]
            epoch_losses += probe_train(net, lm_probe_systems([runner], [seq]), probes_per_system, 1, learning_rate,
                                        seed=1000 * epoch + seed)
            del runner, prob, seq
        losses.append(float(np.mean(epoch_losses)))
    train_s = time.perf_counter() - t0
    rows = []
    for group, seeds in (("held_out_iterations", train_seeds), ("unseen_seeds", unseen_seeds)):
        for seed in seeds:
            prob = W.bundle_problem_device(P, L, per_eliminated="2+poisson4", window=40, seed=seed)
            runner = LMRunner(prob)
            seq = list(lm_sequence(prob, total, seed=seed))[train_iterations:]
            for r in evaluate(net, [runner], [seq], tolerance=tolerance, precision=precision):
                r["group"], r["seed"] = group, int(seed)
                rows.append(r)
            del runner, prob, seq
    plain_it = [r["plain"]["iterations"] for r in rows]
    learned_it = [r["learned"]["iterations"] for r in rows]
    return {"train_seconds": round(train_s, 2), "epoch_losses": losses, "systems_evaluated": len(rows),
            "mean_plain_iterations": float(np.mean(plain_it)) if rows else None,
            "mean_learned_iterations": float(np.mean(learned_it)) if rows else None,
            "fallbacks": int(sum(bool(r["learned"]["fallback"]) for r in rows)),
            "all_converged": all(r["plain"]["converged"] and r["learned"]["converged"] for r in rows),
            "rows": rows}
