"""Host side of multi-GPU runs: one process per GPU, no data-path collective.

The explicit substep does not exchange anything between independent scenes, so
N GPUs run either N replicas of one workload (weak scaling) or one batch of
scenes split into N disjoint partitions.  The only cross-rank traffic is on the
host side of the measurement: a barrier before the timed region and the max of
the ranks' device times after it.

The reference runs one process with OpenMP threads and has no multi-process
path (PhysBAM Hybrid_Methods MPM_DRIVER); the scene partition here plays the
part of its per-thread particle ranges (GATHER_SCATTER::Prepare_Scatter,
Hybrid_Methods/Iterators/GATHER_SCATTER.cpp:33-87) one level up: whole scenes
per GPU instead of x-slabs per thread.
"""
from __future__ import annotations

import datetime
import os
from typing import List, Sequence, Tuple


def rank_env() -> Tuple[int, int, int]:
    """(world size, rank, local rank) from the launcher's environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: float = 120.0):
    """Join the process group when more than one rank runs; returns the
    torch.distributed module or None for a single process."""
    world, _, _ = rank_env()
    if world <= 1:
        return None
    import torch.distributed as dist
    if not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def partition_scenes(particle_counts: Sequence[int], world: int) -> List[List[int]]:
    """Split scenes into `world` disjoint sets of similar particle totals.

    Longest-processing-time greedy: scenes in decreasing particle count (ties by
    index) each go to the rank with the smallest total so far (ties by rank).
    Every rank computes the same answer from the same counts, so no message is
    needed.  Each rank's list is in increasing scene order.  The largest total
    is at most 4/3 of the optimum plus one scene."""
    if world < 1:
        raise ValueError("world size must be positive")
    counts = [int(c) for c in particle_counts]
    if any(c < 0 for c in counts):
        raise ValueError("negative particle count")
    load = [0] * world
    parts: List[List[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(counts)), key=lambda k: (-counts[k], k)):
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += counts[i]
    return [sorted(p) for p in parts]


def max_over_ranks(value: float, dist=None, device="cpu") -> float:
    """The largest `value` over all ranks (device timings: the job ends when
    the slowest rank does)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, dist=None, device="cpu") -> float:
    """Total of `value` over all ranks (units processed by the whole job)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
