"""Benchmark of the LM normal-equation / Schur / block-Jacobi-PCG hot path on B200.

Step (the unit timed): one Levenberg-Marquardt linear step of the large Schur LM
workload -- P=4,000 primary 6-dof blocks, L=2,000,000 eliminated 3-dof blocks, each
observed by 2+Poisson(4) distinct primaries from a wrapped window of 40 (about 12.0M
2-dim residuals, Jacobians N(0,1), residuals N(0,0.5^2) with 5% N(0,20^2) outliers,
Huber delta 1, LM lambda 1e-3).  From device-resident Jacobians the step computes the
Huber-weighted normal equations, the damped Schur complement and its block-Jacobi
preconditioner, solves the reduced system to an FP64 true relative residual of 1e-8
and back-substitutes the eliminated step.  The headline pipeline is mixed precision
(FP64 assembly, FP32 inner PCG with FP64 dots, FP64 refinement); the plain FP64
pipeline is timed beside it.  Synthetic, seeded inputs (no dataset).

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Under torchrun (N>1) every rank solves its own system (replicas: the path has no
exchange step), time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

P_FULL, L_FULL = 4000, 2_000_000
LAMBDA, TOL = 1e-3, 1e-8
WORKLOAD = ("schur_lm_P4000_L2000000: P=4,000 x 6-dof, L=2,000,000 x 3-dof, 2+Poisson(4) primaries "
            "per eliminated block from a wrapped window of 40, 2-dim residuals, Huber delta 1, "
            "lambda 1e-3, FP64 true relative residual 1e-8")
METRIC = "Schur-PCG ms to 1e-8 FP64 rel. residual: learned+mixed vs plain; SpMV HBM GB/s"
# DRAM bytes (read + write) of one assembly (assemble_diag6 + assemble_upper6) per cross block,
# from an ncu capture of the two kernels on the P=4,000, L=200,000 case, scaled by the cross count
# (the traffic grows with the crosses): see the profile summary of the assembly
ASSEMBLY_TRAFFIC_BYTES_PER_CROSS = 632.66e6 / 1_200_542
ASSEMBLY_TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of assemble_diag6 + assemble_upper6 on "
                           "P=4,000, L=200,000 (632.7 MB for 1,200,542 crosses), scaled by the cross count")
BATCH_SYSTEMS = 512


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--eliminated", type=int, default=L_FULL, help="L (eliminated blocks)")
    ap.add_argument("--no-extras", action="store_true", help="skip SpMV / e2e / CPU-baseline legs")
    ap.add_argument("--sparse-only", action="store_true", help="only the Laplacian SpMV / COO->CSR leg")
    ap.add_argument("--dense-only", action="store_true", help="only the dense-backend vs PCG leg (n = 3,072)")
    ap.add_argument("--learned-protocol", default="full", choices=["full", "short"],
                    help="full: train on LM iterations 1-20 of 8 seeds, test on 21-30 and 4 unseen seeds")
    return ap.parse_args()


# ------------------------------------------------------------------ clocks during the timed region
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    INTERVAL_MS = 50

    def __init__(self, device_index: int):
        self.device_index = device_index
        self.proc = None
        self.lines = []
        self.first = 0

    def start(self):
        """Start sampling and return once the first sample has arrived (at most 3 s), so that the
        samples kept -- those after this call -- fall inside the timed region that follows."""
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", str(self.INTERVAL_MS), "-i", str(self.device_index)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
            return
        deadline = time.time() + 3.0
        while not self.lines and time.time() < deadline and self.proc.poll() is None:
            time.sleep(0.01)
        self.first = len(self.lines)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        # samples taken during the timed region; if it was shorter than one interval, the sample
        # taken just before it
        window = self.lines[self.first:] or self.lines[max(0, self.first - 1):self.first]
        for line in window:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm), "interval_ms": self.INTERVAL_MS,
                "samples_in_timed_region": len(self.lines) - self.first}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return d["hbm_gbs"], "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


# ------------------------------------------------------------------ reference arm / CPU baseline
def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown CPU"


def reference_step_ms(prob: dict):
    """One LM linear step through the reference CPU library (oracle/_ref, compiled from the
    reference sources): Huber-weighted BlockNormalEquations accumulation of every observation,
    then solveDampedSchurComplement (Cpu backend, tol 1e-8, lambda 1e-3).  Returns (ms, report)."""
    import oracle
    t0 = time.perf_counter()
    ne = oracle.normal_equations_from_observations(prob, impl="ref")
    _, _, rep = ne.solve(LAMBDA, relative_tolerance=TOL, max_iterations=200)
    ms = (time.perf_counter() - t0) * 1e3
    del ne
    return ms, rep


def reference_sample_text(prob: dict, steps: int) -> str:
    return (f"reference CPU library (oracle/_ref, compiled from the reference sources with g++ -O2): "
            f"Huber-weighted BlockNormalEquations accumulation of all {len(prob['obs_primary']):,} observations + "
            f"solveDampedSchurComplement(Cpu backend, tol 1e-8) on the full P=4,000, L=2,000,000 system, "
            f"{steps} step(s), each timed on its own (no scaling); 1 thread of {os.cpu_count()} "
            f"({cpu_model()}); the reference's path has no threading")


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle
    if not oracle.available("ref"):
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU library oracle/_ref not built"}))
        return
    from plamatrix_b200 import workloads as W
    # warm-up: the same code path on the small P=20, L=2,000 workload (CPU code has no device
    # caches or JIT to warm; a full-size warm-up step would only add a minute per step)
    small = W.small_bundle(seed=0)
    for _ in range(args.warmup):
        reference_step_ms(small)
    prob = W.large_bundle(seed=0, P=P_FULL, L=args.eliminated)  # generated once, outside the timed steps
    times, reps = [], []
    for k in range(args.steps):
        ms, rep = reference_step_ms(prob)
        times.append(ms)
        reps.append(rep)
        print(f"reference step {k + 1}/{args.steps}: {ms / 1e3:.2f} s, {rep['iterations']} iterations",
              file=sys.stderr, flush=True)
    value = statistics.mean(times)
    sample = reference_sample_text(prob, args.steps)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "ms", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(value, 3), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_dict(args.gpus, args.eliminated),
        "iterations": [r["iterations"] for r in reps], "converged": all(r["converged"] for r in reps),
        "step_ms_min_median_max": [round(min(times), 1), round(statistics.median(times), 1), round(max(times), 1)],
        "warmup_workload": "P=20, L=2,000 (same code path)",
        "cpu_baseline": {"value": round(value, 3), "unit": "ms", "cores": 1, "kind": "reference", "sample": sample},
        "e2e": {"value": round(value, 3), "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def config_dict(world: int, L: int) -> dict:
    """The workload of every arm's line (the same dict for ours and the reference); a run with
    another eliminated-block count names its own L."""
    workload = WORKLOAD if L == L_FULL else WORKLOAD.replace("L2000000", f"L{L}").replace(
        "L=2,000,000", f"L={L:,}")
    return {"workload": workload, "primary_blocks": P_FULL, "eliminated_blocks": L,
            "parallelism": f"replicas x{world} (no exchange step)",
            "l2": "inputs larger than L2 (observations 1.9 GB FP64)" if L == L_FULL else
            "observations %.2f GB FP64" % (L * 6 * 160 / 1e9)}


# ------------------------------------------------------------------ our arm
def run_ours(args):
    import torch
    import torch.distributed as dist

    from plamatrix_b200 import replicas

    world, rank = replicas.world_and_rank()
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))

    from plamatrix_b200 import _native as N
    from plamatrix_b200 import schur as SC
    from plamatrix_b200 import sparse as S
    from plamatrix_b200 import workloads as W

    L = args.eliminated
    prob = W.large_bundle(seed=rank, P=P_FULL, L=L)
    nobs = len(prob["obs_primary"])
    host = {k: torch.from_numpy(prob[k]).pin_memory() for k in ("obs_primary", "obs_eliminated", "jp", "jl",
                                                                   "residual")}
    dev = {k: v.cuda() for k, v in host.items()}
    ne = SC.DeviceNormalEquations(P_FULL, L, 6, 3)
    ws = SC.SchurComplementSolverWorkspace()
    n, m = P_FULL * 6, L * 3
    dp = torch.zeros(n, dtype=torch.float64, device="cuda")
    dl = torch.zeros(m, dtype=torch.float64, device="cuda")
    # mixed precision as specified: FP32 assembly products, SpMV and preconditioner apply; FP64
    # dots, factorisations and matrix-free true residual.  mixed64: FP64 assembly, FP32 inner PCG
    mixed = SC.SchurComplementSolverOptions(max_iterations=200, relative_tolerance=TOL,
                                            precision="mixed_fp32_assembly")
    mixed64 = SC.SchurComplementSolverOptions(max_iterations=200, relative_tolerance=TOL, precision="mixed")
    plain = SC.SchurComplementSolverOptions(max_iterations=200, relative_tolerance=TOL, precision="native")
    stream = torch.cuda.current_stream()

    def step(opts):
        ne.accumulate_observations(dev["obs_primary"], dev["obs_eliminated"], dev["jp"], dev["jl"],
                                   dev["residual"], 1.0)
        return SC.solve_damped_schur_complement(ne, LAMBDA, opts, ws, dp, dl)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def timed(fn, steps):
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        last = None
        for _ in range(steps):
            last = fn()
        e1.record(stream)
        barrier()
        ms = replicas.max_over_ranks(e0.elapsed_time(e1) / steps)
        return ms, last

    # ---- learned block-Jacobi correction: the LM-sequence protocol (device kernels: features,
    # tensor-core MLP forward/backward, Adam), probe loss of the preconditioned operator; held-out
    # LM iterations and unseen seeds evaluated against plain block Jacobi
    from plamatrix_b200 import learned as LR
    net = SC.LearnedPreconditioner(seed=rank)
    if args.learned_protocol == "full":
        c3 = LR.c3_protocol(net, P_FULL, L, train_seeds=range(8), unseen_seeds=range(100, 104), train_iterations=20,
                            test_iterations=10, epochs=2)
    else:
        c3 = LR.c3_protocol(net, P_FULL, L, train_seeds=range(2), unseen_seeds=range(100, 101), train_iterations=4,
                            test_iterations=2, epochs=1)
    learned_mixed = SC.SchurComplementSolverOptions(max_iterations=200, relative_tolerance=TOL,
                                                    precision="mixed_fp32_assembly", learned=net)

    for _ in range(args.warmup):
        step(learned_mixed)
        step(mixed)
        step(mixed64)
        step(plain)
    torch.cuda.synchronize()
    # the upper-block assembly launch shape, timed on this system (FP64 products: the last warm-up
    # step was plain) before the timed region; the fastest is kept for every arm
    tune = ws.autotune_assembly(ne, repeats=3)
    tune["shapes"] = ["%d streams x %d lanes" % ws.assembly_shape_info(k) for k in range(len(tune["shape_ms"]))]
    tune["shape_ms"] = [round(t, 4) for t in tune["shape_ms"]]
    tune["ms"] = round(tune["ms"], 4)
    step(plain)
    torch.cuda.synchronize()

    clocks = ClockSampler(local)
    clocks.start()
    launches0 = N.load().pm_kernel_launches()
    ms_learned, (_, _, rep_learned) = timed(lambda: step(learned_mixed), args.steps)
    launches = (N.load().pm_kernel_launches() - launches0) / args.steps
    ms_mixed, (_, _, rep_mixed) = timed(lambda: step(mixed), args.steps)
    ms_mixed64, (_, _, rep_mixed64) = timed(lambda: step(mixed64), args.steps)
    ms_plain, (_, _, rep_plain) = timed(lambda: step(plain), args.steps)
    clock = clocks.stop()

    # accumulation alone (for the phase table)
    ms_accum, _ = timed(lambda: ne.accumulate_observations(dev["obs_primary"], dev["obs_eliminated"], dev["jp"],
                                                           dev["jl"], dev["residual"], 1.0), args.steps)
    # the 6x6 block-CSR SpMV of the PCG on the system the plain step assembled
    schur_spmv = schur_spmv_leg(torch, ws, n, stream) if rank == 0 else None
    out = {}
    if rank == 0 and not args.no_extras:
        out = extras(args, torch, SC, S, W, ne, ws, host, dev, dp, dl, learned_mixed, n, m, net, prob)
    if not args.no_extras:
        # every rank takes part: the 512 independent systems are sharded across the ranks
        batched = batched_leg(torch, SC, W, net)
        if rank == 0:
            out["batched"] = batched
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return

    hbm, peak_kind = peaks()
    # dominant kernel: the Schur assembly (one CTA per block row); algorithmic bytes per launch =
    # cross blocks read (C x 18 x 8) + eliminated inverses (L x 9 x 8) + y (L x 3 x 8) + primary
    # blocks (P x 42 x 8) + topology (C x 8 + L x 4) + Schur blocks written (B x 36 x 8) +
    # RHS + preconditioner (P x 42 x 8)
    C_, _, _ = ne.counts()
    _, _, B = ws.dims()
    assembly_bytes = C_ * 18 * 8 + L * 12 * 8 + P_FULL * 42 * 8 + C_ * 8 + L * 4 + B * 36 * 8 + P_FULL * 42 * 8
    asm_ms = rep_plain["assembly_ms"]
    achieved = assembly_bytes / (asm_ms * 1e-3) / 1e9
    phases = ("pattern_ms", "eliminated_inverse_ms", "assembly_ms", "solve_ms", "back_substitution_ms", "total_ms")
    def group_summary(group):
        rows = [r for r in c3["rows"] if r["group"] == group]
        return {"systems": len(rows),
                "mean_plain_iterations": round(float(np.mean([r["plain"]["iterations"] for r in rows])), 3) if rows else None,
                "mean_learned_iterations": round(float(np.mean([r["learned"]["iterations"] for r in rows])), 3) if rows else None,
                "plain_learned_iterations": [[r["plain"]["iterations"], r["learned"]["iterations"]] for r in rows]}

    line = {
        "metric": METRIC, "value": round(ms_learned, 4), "unit": "ms", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_learned, 4), "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None,
        "dtype": ("f64 result (FP32 assembly products, SpMV and preconditioner apply; FP64 dots, alpha/beta, "
                  "Cholesky factors, matrix-free true residual and refinement; BF16 tensor-core MLP)"),
        "data": "synthetic",
        "config": config_dict(world, L),
        "workload_counts": {"observations": nobs, "schur_blocks": B, "cross_blocks": C_, "systems_per_step": world},
        "plain_fp64_ms": round(ms_plain, 4),
        "mixed_ms": round(ms_mixed, 4),
        "mixed_fp64_assembly_ms": round(ms_mixed64, 4),
        "learned_mixed_over_plain_speedup": round(ms_plain / ms_learned, 3),
        "mixed_over_plain_speedup": round(ms_plain / ms_mixed, 3),
        "pcg_phase_speedup": {"learned_mixed_over_plain": round(rep_plain["solve_ms"] / rep_learned["solve_ms"], 3),
                              "mixed_over_plain": round(rep_plain["solve_ms"] / rep_mixed["solve_ms"], 3)},
        "accumulation_ms": round(ms_accum, 4),
        "phases_learned_mixed": {k: round(rep_learned[k], 4) for k in phases},
        "phases_mixed": {k: round(rep_mixed[k], 4) for k in phases},
        "phases_mixed_fp64_assembly": {k: round(rep_mixed64[k], 4) for k in phases},
        "phases_plain": {k: round(rep_plain[k], 4) for k in phases},
        "iterations": {"learned_mixed_inner": rep_learned["iterations"],
                       "learned_mixed_refinements": rep_learned["refinement_steps"],
                       "learned_fallback": bool(rep_learned["learned_fallback"]),
                       "mixed_inner": rep_mixed["iterations"], "mixed_refinements": rep_mixed["refinement_steps"],
                       "mixed_fp64_assembly_inner": rep_mixed64["iterations"], "plain": rep_plain["iterations"]},
        "true_relative_residual": {"learned_mixed": rep_learned["true_relative_residual"],
                                   "mixed": rep_mixed["true_relative_residual"],
                                   "mixed_fp64_assembly": rep_mixed64["true_relative_residual"],
                                   "plain": rep_plain["true_relative_residual"]},
        "converged": bool(rep_learned["converged"] and rep_mixed["converged"] and rep_mixed64["converged"] and
                          rep_plain["converged"]),
        "learned": {
            "protocol": ("LM sequences of the large problem (Jacobians x (1 + 0.1 N(0,1)), lambda x{0.5,2} from 1e-3); "
                         + ("training on iterations 1-20 of seeds 0-7 (2 passes, 4 Rademacher probes per system, "
                            "probe loss ||(I - M S) v||^2 / ||v||^2, Adam lr 1e-3); tested on iterations 21-30 of "
                            "those seeds and of 4 unseen seeds" if args.learned_protocol == "full" else
                            "short form: training on iterations 1-4 of seeds 0-1 (1 pass, 4 probes per system); "
                            "tested on iterations 5-6 of those seeds and of 1 unseen seed; --learned-protocol full "
                            "runs iterations 1-20 x 8 seeds / 21-30 + 4 unseen seeds")),
            "train_seconds": c3["train_seconds"], "epoch_losses": [round(x, 6) for x in c3["epoch_losses"]],
            "held_out_iterations": group_summary("held_out_iterations"),
            "unseen_seeds": group_summary("unseen_seeds"),
            "fallbacks": c3["fallbacks"], "all_converged": c3["all_converged"],
        },
        "roofline": {"bound": "hbm", "kernel": "assemble_diag6_kernel + assemble_upper6_kernel (FP64, plain step)",
                     "achieved": round(achieved, 1),
                     "peak": hbm, "unit": "GB/s", "frac": round(achieved / hbm, 4),
                     "traffic": (round(ASSEMBLY_TRAFFIC_BYTES_PER_CROSS * C_) if ASSEMBLY_TRAFFIC_BYTES_PER_CROSS
                                 else None),
                     "traffic_source": ASSEMBLY_TRAFFIC_SOURCE,
                     "peak_kind": peak_kind, "algorithmic_bytes_per_launch": assembly_bytes},
        "schur_spmv_fp64": schur_spmv,
        "assembly_autotune": tune,
        "gpu_launches": launches,
        "clocks": clock,
    }
    line.update(out)
    print(json.dumps(line))


def extras(args, torch, SC, S, W, ne, ws, host, dev, dp, dl, opts, n, m, net=None, prob=None):
    out = {}
    # ---- end to end through the public API with host buffers
    dp_h = torch.empty(n, dtype=torch.float64).pin_memory()
    dl_h = torch.empty(m, dtype=torch.float64).pin_memory()
    stream = torch.cuda.current_stream()

    def e2e_step():
        for k in ("obs_primary", "obs_eliminated", "jp", "jl", "residual"):
            dev[k].copy_(host[k], non_blocking=True)
        ne.accumulate_observations(dev["obs_primary"], dev["obs_eliminated"], dev["jp"], dev["jl"],
                                   dev["residual"], 1.0)
        SC.solve_damped_schur_complement(ne, LAMBDA, opts, ws, dp, dl)
        dp_h.copy_(dp, non_blocking=True)
        dl_h.copy_(dl, non_blocking=True)

    e2e_step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        e2e_step()
    e1.record(stream)
    torch.cuda.synchronize()
    h2d = sum(v.numel() * v.element_size() for v in host.values())
    out["e2e"] = {"value": round(e0.elapsed_time(e1) / args.steps, 3), "unit": "ms", "h2d_bytes_per_step": h2d,
                  "d2h_bytes_per_step": (n + m) * 8}
    out["spmv"] = sparse_leg(torch, S, W, stream)
    out["c1_jacobi_pcg"] = c1_pcg_leg(torch, S, W, stream)
    out["c0"] = c0_leg(torch, SC, W, stream)
    out["dense_c4_max"] = dense_leg(torch, SC, W)
    # ---- CPU baseline: one full-size LM linear step of the reference's own CPU library (the
    # same host problem the device arm was built from), timed on its own, no scaling
    try:
        import oracle
        if oracle.available("ref") and prob is not None:
            ms, rep = reference_step_ms(prob)
            out["cpu_baseline"] = {
                "value": round(ms, 1), "unit": "ms", "cores": 1, "kind": "reference",
                "sample": reference_sample_text(prob, 1) + f"; {rep['iterations']} PCG iterations"}
    except Exception as exc:  # noqa: BLE001
        out["cpu_baseline"] = {"value": None, "unit": "ms", "cores": 1, "kind": "reference", "sample": str(exc)}
    return out


L2_FLUSH = "flushed before each timed call: 512 MiB written, then read back so no dirty line drains in the timed call"


def flushed_ms(torch, fn, flush, stream, reps=10):
    """Median device time of fn() with L2 flushed before each call (CUDA events on `stream`).
    The flush writes a buffer of 4x the L2 and then reads it back: the read evicts the lines the
    write left dirty, so their write-back to DRAM happens before the timed call instead of
    competing with its reads (the L2 then holds clean lines of the flush buffer only)."""
    times = []
    words = flush.view(torch.float64)
    for _ in range(reps):
        flush.zero_()
        words.sum()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b))
    return statistics.median(times)


def same_size_read_ms(torch, nbytes, flush, stream):
    """A plain device reduction (torch.sum) over nbytes, L2 flushed: what a streaming kernel of
    this size reaches on this GPU (the long-copy peak needs GBs in flight)."""
    ref = torch.ones(max(1, nbytes // 8), dtype=torch.float64, device="cuda")
    out = torch.empty((), dtype=torch.float64, device="cuda")
    t = flushed_ms(torch, lambda: torch.sum(ref, dim=(0,), out=out), flush, stream)
    del ref
    return t


def schur_spmv_leg(torch, ws, n, stream):
    """y = S x on the assembled 6x6 block-CSR Schur system (FP64), L2 flushed before each call."""
    hbm, _ = peaks()
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    dim, nnz, blocks = ws.dims()
    x = torch.randn(n, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    t = flushed_ms(torch, lambda: ws.spmv(x, out=y, stream=stream), flush, stream)
    byts = blocks * 36 * 8 + (n // 6 + 1) * 4 + blocks * 4 + 2 * n * 8
    tr = same_size_read_ms(torch, byts, flush, stream)
    return {"l2": L2_FLUSH, "ms": round(t, 4), "GBps": round(byts / (t * 1e-3) / 1e9, 1),
            "frac_of_hbm": round(byts / (t * 1e-3) / 1e9 / hbm, 3),
            "same_size_read_GBps": round(byts / (tr * 1e-3) / 1e9, 1), "frac_of_same_size_read": round(tr / t, 3),
            "algorithmic_bytes": byts, "blocks": blocks}


def sparse_leg(torch, S, W, stream):
    """CSR SpMV and COO -> CSR of the 128^3 Laplacian (16.04M triplets), FP64 and FP32, L2 flushed
    between timed calls."""
    hbm, _ = peaks()
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    spmv = {}
    lap = W.laplacian_coo(128, seed=0, dtype=np.float64)
    for dt, name in ((torch.float64, "f64"), (torch.float32, "f32")):
        csr = S.coo_to_csr(lap["rows"], lap["cols"], torch.from_numpy(lap["row_indices"]).cuda(),
                           torch.from_numpy(lap["col_indices"]).cuda(),
                           torch.from_numpy(lap["values"]).to(dt).cuda())
        op = S.CsrOperand(csr)
        x = torch.randn(lap["rows"], dtype=dt, device="cuda")
        y = torch.empty_like(x)
        t = flushed_ms(torch, lambda: op.spmv(x, y), flush, stream)
        s = 4 if dt == torch.float32 else 8
        nn = lap["rows"]
        byts = csr.nnz * (s + 4) + (nn + 1) * 4 + 2 * nn * s
        tr = same_size_read_ms(torch, byts, flush, stream)
        spmv[f"csr_laplacian128_{name}"] = {"l2": L2_FLUSH, "ms": round(t, 4),
                                            "GBps": round(byts / (t * 1e-3) / 1e9, 1),
                                            "frac_of_hbm": round(byts / (t * 1e-3) / 1e9 / hbm, 3),
                                            "same_size_read_GBps": round(byts / (tr * 1e-3) / 1e9, 1),
                                            "frac_of_same_size_read": round(tr / t, 3),
                                            "algorithmic_bytes": byts}
        # the autotuner's pick for this operand (timed with warm caches), then flushed again
        chosen = op.autotune(x, y, stream)
        ta = flushed_ms(torch, lambda: op.spmv(x, y), flush, stream)
        spmv[f"csr_laplacian128_{name}"]["autotuned"] = {"kernel": S.CsrOperand.KERNELS[chosen], "ms": round(ta, 4),
                                                         "GBps": round(byts / (ta * 1e-3) / 1e9, 1)}
        # COO -> CSR of the same matrix (16.04M triplets)
        ws_coo = S.SparseOpsWorkspace()
        r_d = torch.from_numpy(lap["row_indices"]).cuda()
        c_d = torch.from_numpy(lap["col_indices"]).cuda()
        v_d = torch.from_numpy(lap["values"]).to(dt).cuda()
        out_csr = S.CSRMatrix.empty(lap["rows"], lap["cols"], csr.nnz, dt)
        S.coo_to_csr_async(lap["rows"], lap["cols"], r_d, c_d, v_d, out_csr, ws_coo)
        torch.cuda.synchronize()
        ws_coo.check_status()
        ct = []
        for _ in range(5):
            flush.zero_()
            flush.view(torch.float64).sum()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            S.coo_to_csr_async(lap["rows"], lap["cols"], r_d, c_d, v_d, out_csr, ws_coo)
            b.record(stream)
            torch.cuda.synchronize()
            ws_coo.check_status()
            ct.append(a.elapsed_time(b))
        trip = len(lap["values"])
        cbytes = trip * (16 + s) + csr.nnz * (4 + s) + (nn + 1) * 4
        tc = statistics.median(ct)
        spmv[f"coo_to_csr_laplacian128_{name}"] = {"ms": round(tc, 4), "GBps": round(cbytes / (tc * 1e-3) / 1e9, 1),
                                                   "triplets": trip, "algorithmic_bytes": cbytes}
    return spmv


def c1_pcg_leg(torch, S, W, stream):
    """Jacobi PCG to a relative residual of 1e-8 on the 128^3 Laplacian (+ 1e-2 shift), FP64 and
    FP32, b ~ U(-1, 1): device time (CUDA events, median of 3 after a warm solve), iterations and
    the FP64 true relative residual of the solution; the reference CPU library's pcg (its
    iterative_solver_cpu.cpp, one thread) on the same matrix and right-hand side beside it."""
    out = {}
    lap = W.laplacian_coo(128, seed=0, dtype=np.float64)
    n = lap["rows"]
    r_d, c_d = torch.from_numpy(lap["row_indices"]).cuda(), torch.from_numpy(lap["col_indices"]).cuda()
    csr64 = S.coo_to_csr(n, n, r_d, c_d, torch.from_numpy(lap["values"]).cuda())
    op64 = S.CsrOperand(csr64)
    for dt, name in ((torch.float64, "f64"), (torch.float32, "f32")):
        csr = csr64 if dt == torch.float64 else S.coo_to_csr(n, n, r_d, c_d, torch.from_numpy(lap["values"]).to(dt).cuda())
        b = torch.from_numpy(lap["rhs"]).to(dt).cuda()
        opts = S.IterativeSolverOptions(relative_tolerance=1e-8, max_iterations=2000)
        op = op64 if dt == torch.float64 else S.CsrOperand(csr)
        sws = S.IterativeSolverWorkspace()
        times, rep = [], None
        for k in range(4):
            x = torch.zeros(n, dtype=dt, device="cuda")
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            rep = S.pcg(op, b, x, workspace=sws, options=opts)
            e1.record(stream)
            torch.cuda.synchronize()
            if k > 0:
                times.append(e0.elapsed_time(e1))
        x64 = x.to(torch.float64)
        b64 = b.to(torch.float64)
        res = b64 - op64.spmv(x64, torch.empty_like(x64))
        entry = {"ms": round(statistics.median(times), 3), "iterations": rep["iterations"],
                 "converged": bool(rep["converged"]),
                 "true_relative_residual": float(torch.linalg.norm(res) / torch.linalg.norm(b64))}
        try:
            import oracle
            if oracle.available("ref"):
                ro, ci, v = csr.cpu()
                t0 = time.perf_counter()
                _, rref = oracle.pcg(ro, ci, v, lap["rhs"].astype(v.dtype), relative_tolerance=1e-8,
                                     max_iterations=2000, impl="ref")
                entry["reference_cpu"] = {"ms": round((time.perf_counter() - t0) * 1e3, 1),
                                          "iterations": rref["iterations"], "converged": bool(rref["converged"]),
                                          "cores": 1}
        except Exception as exc:  # noqa: BLE001
            entry["reference_cpu"] = {"error": str(exc)}
        out[name] = entry
    return out


def c0_leg(torch, SC, W, stream):
    """The small Schur workload (P=20, L=2,000, 8,000 observations, tol 1e-10): one device LM linear
    step from device observations (accumulation, assembly, block-Jacobi PCG, back-substitution;
    median of 10 after 3 warm steps, CUDA events) against the reference CPU library's accumulation
    + solveDampedSchurComplement with the Cpu backend and with DenseCpu (its OpenMP dense Cholesky,
    all host threads), median of 5."""
    prob = W.small_bundle(seed=1)
    dev = {k: torch.from_numpy(prob[k]).cuda() for k in ("obs_primary", "obs_eliminated", "jp", "jl", "residual")}
    ne = SC.DeviceNormalEquations(prob["P"], prob["L"], 6, 3)
    ws = SC.SchurComplementSolverWorkspace()
    opts = SC.SchurComplementSolverOptions(max_iterations=500, relative_tolerance=1e-10)
    times = []
    for k in range(13):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ne.accumulate_observations(dev["obs_primary"], dev["obs_eliminated"], dev["jp"], dev["jl"], dev["residual"],
                                   prob["huber_delta"])
        _, _, rep = SC.solve_damped_schur_complement(ne, 1e-3, opts, ws)
        e1.record(stream)
        torch.cuda.synchronize()
        if k >= 3:
            times.append(e0.elapsed_time(e1))
    out = {"workload": "P=20, L=2,000, 4 distinct uniform primaries per eliminated block, tol 1e-10",
           "device_ms": round(statistics.median(times), 3), "device_iterations": rep["iterations"]}
    try:
        import oracle
        if oracle.available("ref"):
            for backend, key in (("cpu", "reference_cpu"), ("dense_cpu", "reference_dense_cpu")):
                t = []
                for _ in range(6):
                    t0 = time.perf_counter()
                    ref_ne = oracle.normal_equations_from_observations(prob, impl="ref")
                    _, _, rrep = ref_ne.solve(1e-3, backend=backend, relative_tolerance=1e-10, max_iterations=500)
                    t.append((time.perf_counter() - t0) * 1e3)
                    del ref_ne
                out[key] = {"ms": round(statistics.median(t[1:]), 3), "iterations": rrep["iterations"],
                            "converged": bool(rrep["converged"]),
                            "threads": os.cpu_count() if backend == "dense_cpu" else 1}
    except Exception as exc:  # noqa: BLE001
        out["reference_error"] = str(exc)
    return out


def dense_leg(torch, SC, W):
    """The largest C4 system size (P=512, L=50,000; n = 3,072 primary unknowns): the dense backend
    (device Cholesky, DenseCpu's counterpart) against block-Jacobi PCG, whole solve each."""
    prob = W.bundle_problem(512, 50000, per_eliminated=4, window=40, seed=5)
    ne = SC.DeviceNormalEquations(512, 50000, 6, 3)
    ne.accumulate_observations(*[torch.from_numpy(prob[k]).cuda() for k in ("obs_primary", "obs_eliminated", "jp",
                                                                            "jl", "residual")], prob["huber_delta"])
    out = {"primary_unknowns": 512 * 6}
    for name, backend in (("pcg", "pcg"), ("dense", "dense")):
        ws = SC.SchurComplementSolverWorkspace()
        opts = SC.SchurComplementSolverOptions(max_iterations=1000, relative_tolerance=1e-8, linear_backend=backend)
        SC.solve_damped_schur_complement(ne, 1e-3, opts, ws)
        times = []
        for _ in range(5):
            torch.cuda.synchronize()
            _, _, rep = SC.solve_damped_schur_complement(ne, 1e-3, opts, ws)
            times.append(rep["total_ms"])
        out[name] = {"ms": round(statistics.median(times), 3), "solve_ms": round(rep["solve_ms"], 3),
                     "iterations": rep["iterations"], "converged": bool(rep["converged"]),
                     "true_relative_residual": rep["true_relative_residual"]}
    return out


def batched_leg(torch, SC, W, net, systems=BATCH_SYSTEMS):
    """Independent systems P ~ U{8..512}, L ~ U{500..50,000}, 4 uniform distinct primaries per
    eliminated block, split across the ranks by estimated cost (contiguous shards, no collective on
    the data path): each rank solves its shard as one batched launch sequence (union accumulation,
    pattern, assembly, graph-replayed per-system PCG, back-substitution) and as a plain per-system
    loop.  Times are device times, the job's the maximum over ranks.  Latency is reported two ways:
    a system's own duration, and the time from the start of the job to its solution."""
    from plamatrix_b200 import replicas
    world, rank = replicas.world_and_rank()
    sizes = W.uneven_family_sizes(systems)
    costs = [P * 36 + 4 * L for P, L in sizes]
    mine = replicas.shard_by_cost(costs, rank, world)
    probs = [W.uneven_family_system(i, *sizes[i]) for i in mine]
    P_off = np.cumsum([0] + [p["P"] for p in probs]).astype(np.int64)
    L_off = np.cumsum([0] + [p["L"] for p in probs]).astype(np.int64)
    union = {
        "obs_primary": torch.cat([p["obs_primary"] + int(P_off[i]) for i, p in enumerate(probs)]),
        "obs_eliminated": torch.cat([p["obs_eliminated"] + int(L_off[i]) for i, p in enumerate(probs)]),
        "jp": torch.cat([p["jp"] for p in probs]), "jl": torch.cat([p["jl"] for p in probs]),
        "residual": torch.cat([p["residual"] for p in probs])}
    opts = SC.SchurComplementSolverOptions(max_iterations=500, relative_tolerance=TOL)
    stream = torch.cuda.current_stream()
    res = {"systems": systems, "ranks": world, "shard": "contiguous by estimated cost (36 P + 4 L per system)",
           "config": "P~U{8..512}, L~U{500..50000}, 4 uniform distinct primaries per eliminated block, tol 1e-8"}

    def run_batched(options):
        ne_u = SC.DeviceNormalEquations(int(P_off[-1]), int(L_off[-1]), 6, 3)
        ws_u = SC.SchurComplementSolverWorkspace()
        tune = None
        for k in range(2):  # the first call builds the topology and the pattern
            if k == 1:
                # the union's assembly launch shape, timed on the system the first call solved
                tune = ws_u.autotune_assembly(ne_u, repeats=2)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ne_u.accumulate_observations(union["obs_primary"], union["obs_eliminated"], union["jp"], union["jl"],
                                         union["residual"], 1.0)
            e1.record(stream)
            _, _, rep, per = SC.solve_batched_schur_complement(ne_u, LAMBDA, P_off, options, ws_u)
            torch.cuda.synchronize()
            t_acc = e0.elapsed_time(e1)
            total = t_acc + rep["total_ms"]
        # a system's solution is available once the shared prefix (accumulation, pattern check,
        # eliminated inverses, assembly), its own PCG and the shared back-substitution are done
        prefix = t_acc + rep["pattern_ms"] + rep["eliminated_inverse_ms"] + rep["assembly_ms"]
        done = [prefix + s["time_ms"] + rep["back_substitution_ms"] for s in per if s["converged"]]
        job_ms = replicas.max_over_ranks(total)
        done_all = replicas.gather_reports(done)
        conv = replicas.gather_reports([int(s["converged"]) for s in per])
        fb = replicas.gather_reports([int(s["learned_fallback"]) for s in per])
        its = replicas.gather_reports([s["iterations"] for s in per])
        if rank != 0:
            return None
        return {"ms": round(job_ms, 3), "systems_per_s": round(systems / (job_ms * 1e-3), 1),
                "assembly_shape_rank0": "%d streams x %d lanes" % ws_u.assembly_shape_info(tune["shape"]),
                "assembly_shape_ms_rank0": [round(t, 3) for t in tune["shape_ms"]],
                "converged": sum(conv), "fallbacks": sum(fb), "max_iterations": max(its),
                "mean_iterations": round(float(np.mean(its)), 2),
                "phases_ms_rank0": {"accumulation": round(t_acc, 3), "pattern": round(rep["pattern_ms"], 3),
                                    "eliminated_inverse": round(rep["eliminated_inverse_ms"], 3),
                                    "assembly": round(rep["assembly_ms"], 3), "pcg": round(rep["solve_ms"], 3),
                                    "back_substitution": round(rep["back_substitution_ms"], 3)},
                "time_to_solution_from_job_start_p50_ms": round(float(np.percentile(done_all, 50)), 3),
                "time_to_solution_from_job_start_p99_ms": round(float(np.percentile(done_all, 99)), 3),
                "own_duration_p50_ms": round(float(np.percentile(done_all, 50)), 3),
                "own_duration_p99_ms": round(float(np.percentile(done_all, 99)), 3)}

    res["batched_plain"] = run_batched(opts)
    # mixed precision: FP64 assembly, iterations on the FP32 values and blocks, FP64 checks
    res["batched_mixed"] = run_batched(SC.SchurComplementSolverOptions(max_iterations=500, relative_tolerance=TOL,
                                                                       precision="mixed"))
    if net is not None:
        res["batched_learned"] = run_batched(SC.SchurComplementSolverOptions(max_iterations=500, relative_tolerance=TOL,
                                                                             learned=net))
        res["batched_learned_mixed"] = run_batched(SC.SchurComplementSolverOptions(
            max_iterations=500, relative_tolerance=TOL, learned=net, precision="mixed"))
    # per-system launch loop on the same shard (each system with its own normal equations and
    # workspace, warmed once); its own duration and its time from the start of the loop
    own, from_start, t = [], [], 0.0
    nes = []
    for p in probs:
        ne_s = SC.DeviceNormalEquations(p["P"], p["L"], 6, 3)
        ws_s = SC.SchurComplementSolverWorkspace()
        ne_s.accumulate_observations(p["obs_primary"], p["obs_eliminated"], p["jp"], p["jl"], p["residual"], 1.0)
        SC.solve_damped_schur_complement(ne_s, LAMBDA, opts, ws_s)
        nes.append((ne_s, ws_s))
    torch.cuda.synchronize()
    for p, (ne_s, ws_s) in zip(probs, nes):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ne_s.accumulate_observations(p["obs_primary"], p["obs_eliminated"], p["jp"], p["jl"], p["residual"], 1.0)
        SC.solve_damped_schur_complement(ne_s, LAMBDA, opts, ws_s)
        e1.record(stream)
        torch.cuda.synchronize()
        dt = e0.elapsed_time(e1)
        t += dt
        own.append(dt)
        from_start.append(t)
    loop_ms = replicas.max_over_ranks(t)
    own_all = replicas.gather_reports(own)
    start_all = replicas.gather_reports(from_start)
    if rank != 0:
        return None
    res["per_system_loop"] = {"ms": round(loop_ms, 3), "systems_per_s": round(systems / (loop_ms * 1e-3), 1),
                              "own_duration_p50_ms": round(float(np.percentile(own_all, 50)), 3),
                              "own_duration_p99_ms": round(float(np.percentile(own_all, 99)), 3),
                              "time_to_solution_from_job_start_p50_ms": round(float(np.percentile(start_all, 50)), 3),
                              "time_to_solution_from_job_start_p99_ms": round(float(np.percentile(start_all, 99)), 3)}
    return res


if __name__ == "__main__":
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    elif a.sparse_only:
        import torch
        from plamatrix_b200 import sparse as S_
        from plamatrix_b200 import workloads as W_
        print(json.dumps({"spmv": sparse_leg(torch, S_, W_, torch.cuda.current_stream())}))
    elif a.dense_only:
        import torch
        from plamatrix_b200 import schur as SC_
        from plamatrix_b200 import workloads as W_
        print(json.dumps({"dense_c4_max": dense_leg(torch, SC_, W_)}))
    else:
        run_ours(a)
