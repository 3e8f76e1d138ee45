"""Multi-GPU layout of the normal-equation / Schur / PCG path: replicas only.

One solve has no exchange step worth sharding (its reduced system is a few MB and block-Jacobi
PCG converges in a handful of iterations), so N GPUs run N independent problems, one process per
GPU. Two pieces of host logic are shared by every multi-rank run:

- the step time of the job is the maximum over ranks of each rank's device time (a slow rank sets
  the pace of the whole job);
- independent systems (the batched workload) are partitioned into contiguous, disjoint ranges,
  one per rank -- by count, or balanced by an estimated cost per system -- with no collective on
  the data path; their per-system reports are gathered on rank 0 afterwards.

The collectives here run on whatever process group the caller initialised: NCCL on GPUs, gloo on
CPU (the tests).
"""
from __future__ import annotations

import math
import os
from typing import Sequence

import torch
import torch.distributed as dist


def world_and_rank() -> tuple[int, int]:
    """(WORLD_SIZE, RANK) as set by torchrun; (1, 0) for a single process."""
    return int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0"))


def _collective_device() -> torch.device:
    if dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def max_over_ranks(value: float) -> float:
    """The maximum of `value` over all ranks (every rank gets it); `value` itself without a
    process group or with one rank."""
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=_collective_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shard(count: int, rank: int, world: int) -> range:
    """The contiguous range of `count` independent systems that `rank` of `world` solves: sizes
    differ by at most one, lower ranks take the larger ranges, and the ranges partition
    0..count-1 in rank order."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    if count < 0:
        raise ValueError("count must be non-negative")
    base, extra = divmod(count, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def shard_by_cost(costs: Sequence[float], rank: int, world: int) -> range:
    """The contiguous range of systems that `rank` of `world` solves when system i has estimated
    cost costs[i] >= 0: system i goes to the rank whose share [r, r + 1) x total / world holds
    the midpoint of i's cost interval in the prefix sum. The ranges are contiguous, disjoint,
    in rank order, and as even in cost as a contiguous split allows; with a zero total the
    split is by count."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    c = [float(x) for x in costs]
    if any(not (math.isfinite(x) and x >= 0.0) for x in c):
        raise ValueError("costs must be finite and non-negative")
    total = sum(c)
    if total <= 0.0:
        return shard(len(c), rank, world)
    owners, prefix = [], 0.0
    for x in c:
        owners.append(min(world - 1, int((prefix + 0.5 * x) * world / total)))
        prefix += x
    # owners is non-decreasing: this rank's systems are the run of entries equal to `rank`
    start = sum(1 for o in owners if o < rank)
    stop = sum(1 for o in owners if o <= rank)
    return range(start, stop)


def gather_reports(local: list) -> list | None:
    """Every rank's per-system reports, concatenated in rank order, on rank 0 (None on the other
    ranks); `local` itself without a process group or with one rank."""
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return list(local)
    rank, world = dist.get_rank(), dist.get_world_size()
    parts = [None] * world if rank == 0 else None
    dist.gather_object(list(local), parts, dst=0)
    if rank != 0:
        return None
    return [item for part in parts for item in part]
