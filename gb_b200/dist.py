"""Multi-GPU plumbing: one process per GPU, no data-path collective.

A single Macaulay matrix does not shard (its echelon needs every pivot), so
several GPUs either run replicas of the same reduction (benchmark weak
scaling) or split a batch of independent matrices between them.  The only
communication is the timing reduction (max over ranks) and, for batches,
nothing at all: every rank reduces its own share and keeps its answers.
"""
from __future__ import annotations

import heapq
import os
from typing import List, Sequence

from .matrix import MacaulayMatrix


def env_rank() -> tuple:
    """(world_size, rank, local_rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of a per-rank scalar (e.g. device milliseconds) over all ranks
    of the default process group; the value itself when not distributed."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64,
                     device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def work_estimate(m: MacaulayMatrix) -> float:
    """Relative cost of reducing one matrix: nonzeros of the rows to reduce
    times the width of the right block (the Schur update dominates)."""
    nru, nrl = m.split_counts()
    return float(max(m.nnz, 1)) * float(max(m.ncr, 1)) * (1.0 + nrl / max(m.nr, 1))


def shard_batch(mats: Sequence[MacaulayMatrix], world_size: int) -> List[List[int]]:
    """Greedy largest-first assignment of matrices to ranks by estimated work;
    returns the matrix indices of every rank (deterministic)."""
    order = sorted(range(len(mats)), key=lambda i: (-work_estimate(mats[i]), i))
    heap = [(0.0, r) for r in range(world_size)]
    heapq.heapify(heap)
    shards: List[List[int]] = [[] for _ in range(world_size)]
    for i in order:
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + work_estimate(mats[i]), r))
    for s in shards:
        s.sort()
    return shards
