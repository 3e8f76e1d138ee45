"""Multi-rank host logic of the replica layout, on CPU: two gloo ranks agree on the job's step
time (the maximum over ranks) and split a set of independent systems into disjoint, complete,
rank-ordered ranges; a single process needs no process group."""
import os
import socket
from datetime import timedelta

import pytest
import torch.multiprocessing as mp

from plamatrix_b200 import replicas

# estimated per-system costs of an uneven batch (P x L of each system, arbitrary units)
COSTS = [512.0, 8.0, 64.0, 300.0, 12.0, 12.0, 450.0, 40.0, 9.0]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        w, r = replicas.world_and_rank()
        step_ms = replicas.max_over_ranks(1.5 + 2.0 * rank)
        systems = list(replicas.shard(11, r, w))
        # uneven systems, balanced by estimated cost; reports gathered on rank 0 in rank order
        mine = list(replicas.shard_by_cost(COSTS, r, w))
        gathered = replicas.gather_reports([{"system": i, "rank": r} for i in mine])
        dist.barrier()
        out.put((rank, w, r, step_ms, systems, mine, gathered))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_gloo_ranks_take_the_max_time_and_partition_the_systems(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    try:
        results = sorted(q.get(timeout=120) for _ in range(world))
    finally:
        for p in procs:
            p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs)
    assert [r[:3] for r in results] == [(k, world, k) for k in range(world)]
    # every rank reports the slowest rank's time
    assert all(r[3] == 1.5 + 2.0 * (world - 1) for r in results)
    # the ranges cover 0..10 once, in rank order
    joined = [s for r in results for s in r[4]]
    assert joined == list(range(11))
    assert [len(r[4]) for r in results] == [6, 5]
    # cost-balanced ranges: complete, disjoint, in order, and within one system's cost of even
    assert [s for r in results for s in r[5]] == list(range(len(COSTS)))
    loads = [sum(COSTS[i] for i in r[5]) for r in results]
    assert abs(loads[0] - loads[1]) <= max(COSTS)
    # rank 0 holds every report in rank (= system) order; the others hold none
    assert [rep["system"] for rep in results[0][6]] == list(range(len(COSTS)))
    assert [rep["rank"] for rep in results[0][6]] == [r for r in range(world) for _ in results[r][5]]
    assert all(r[6] is None for r in results[1:])


def test_single_process_needs_no_group():
    assert replicas.max_over_ranks(3.25) == 3.25
    assert replicas.world_and_rank() == (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")))


def test_cost_shards_are_contiguous_complete_and_balanced():
    for world in (1, 2, 3, 4, 9, 12):
        parts = [replicas.shard_by_cost(COSTS, r, world) for r in range(world)]
        assert [i for p in parts for i in p] == list(range(len(COSTS)))
        assert all(p.start <= p.stop for p in parts)
    two = [list(replicas.shard_by_cost(COSTS, r, 2)) for r in range(2)]
    assert two == [[0, 1, 2], [3, 4, 5, 6, 7, 8]]
    # zero total cost: by count; invalid costs and ranks are rejected
    assert [list(replicas.shard_by_cost([0.0] * 3, r, 2)) for r in range(2)] == [[0, 1], [2]]
    with pytest.raises(ValueError):
        replicas.shard_by_cost([1.0, -1.0], 0, 2)
    with pytest.raises(ValueError):
        replicas.shard_by_cost([1.0, float("inf")], 0, 2)
    with pytest.raises(ValueError):
        replicas.shard_by_cost([1.0], 3, 2)
    assert replicas.gather_reports([1, 2]) == [1, 2]


def test_shard_edges():
    assert [list(replicas.shard(3, r, 4)) for r in range(4)] == [[0], [1], [2], []]
    assert [list(replicas.shard(0, r, 2)) for r in range(2)] == [[], []]
    assert list(replicas.shard(8, 0, 1)) == list(range(8))
    with pytest.raises(ValueError):
        replicas.shard(4, 2, 2)
    with pytest.raises(ValueError):
        replicas.shard(-1, 0, 1)
