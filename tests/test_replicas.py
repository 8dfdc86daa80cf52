"""The multi-rank host logic on CPU: colonies shared out across ranks once
each, and timings combined as the maximum over ranks, with world_size-2 gloo
process groups."""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from microsimulator_b200 import replicas, workloads


def test_shard_covers_every_colony_once_and_balances_cells():
    sizes, _, _ = workloads.sweep_sizes(256, 500, 50_000, seed=42)
    for world in (1, 2, 4, 8):
        parts = [replicas.shard(sizes, r, world) for r in range(world)]
        joined = np.sort(np.concatenate(parts))
        assert np.array_equal(joined, np.arange(len(sizes)))
        loads = [int(sizes[p].sum()) for p in parts]
        assert max(loads) - min(loads) <= int(sizes.max())
    with pytest.raises(ValueError):
        replicas.shard(sizes, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, queue):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sizes, _, _ = workloads.sweep_sizes(64, 500, 50_000, seed=1)
        mine = replicas.shard(sizes, rank, world)
        # Each rank times its own share; the job's time is the slowest rank's.
        elapsed = 1.0 + rank
        total = replicas.max_over_ranks(elapsed, dist)
        cells = replicas.max_over_ranks(float(sizes[mine].sum()), dist)
        queue.put((rank, total, sorted(mine.tolist()), cells))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_with_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, queue)) for r in range(2)]
    for p in procs:
        p.start()
    results = [queue.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    results.sort()
    assert [r[1] for r in results] == [2.0, 2.0]
    assert sorted(results[0][2] + results[1][2]) == list(range(64))
    assert results[0][3] == results[1][3]


def test_max_over_ranks_without_a_group():
    assert replicas.max_over_ranks(3.5) == 3.5
