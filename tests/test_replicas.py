"""Multi-process host logic on CPU: two `gloo` ranks, no GPU.

The GPU path shards without a data-path collective (replicas of one workload,
or whole scenes per rank), so what crosses ranks is host logic: the scene
partition every rank computes on its own, and the max / sum reductions of the
measurement.  These run here as two spawned processes over 127.0.0.1.
"""
import ast
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from physbam_b200 import replicas


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, counts, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist = replicas.init("gloo", timeout_s=60)
    try:
        assert replicas.rank_env() == (world, rank, rank)
        parts = replicas.partition_scenes(counts, world)
        gathered = [None] * world
        dist.all_gather_object(gathered, parts)
        mine = parts[rank]
        units = float(sum(counts[i] for i in mine))
        total = replicas.sum_over_ranks(units, dist)
        slowest = replicas.max_over_ranks(1.0 + rank, dist)
        dist.barrier()
        with open(os.path.join(out_dir, "rank%d.txt" % rank), "w") as f:
            same = all(g == parts for g in gathered)
            f.write("%d %r %r %r\n" % (same, total, slowest, mine))
    finally:
        dist.destroy_process_group()


def test_partition_single_rank_is_identity():
    assert replicas.partition_scenes([5, 3, 9], 1) == [[0, 1, 2]]
    assert replicas.partition_scenes([], 3) == [[], [], []]
    with pytest.raises(ValueError):
        replicas.partition_scenes([1], 0)
    with pytest.raises(ValueError):
        replicas.partition_scenes([-1], 2)


@pytest.mark.parametrize("world", [2, 3, 8])
def test_partition_covers_and_balances(world):
    rng = np.random.default_rng(world)
    counts = rng.integers(1_000, 450_000, 256).tolist()
    parts = replicas.partition_scenes(counts, world)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(256))
    loads = [sum(counts[i] for i in p) for p in parts]
    # LPT bound: max load <= 4/3 optimum + largest job; the optimum is >= the mean
    assert max(loads) <= 4 / 3 * sum(counts) / world + max(counts)
    assert all(p == sorted(p) for p in parts)
    assert replicas.partition_scenes(counts, world) == parts     # deterministic


def test_two_gloo_ranks(tmp_path):
    rng = np.random.default_rng(3)
    counts = rng.integers(1_000, 450_000, 64).tolist()
    world = 2
    mp.spawn(_worker, args=(world, free_port(), counts, str(tmp_path)), nprocs=world, join=True)
    lines = [open(tmp_path / ("rank%d.txt" % r)).read().split(" ", 3) for r in range(world)]
    parts = replicas.partition_scenes(counts, world)
    for r, (same, total, slowest, mine) in enumerate(lines):
        assert same == "1"
        assert float(total) == float(sum(counts))
        assert float(slowest) == float(world)
        assert ast.literal_eval(mine) == parts[r]
