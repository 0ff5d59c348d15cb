"""Several GPUs: whole structures per rank, one gather at the end.

Rays, replicate blocks and structures are independent, so the work shards
without any data-path exchange: each rank (one process per GPU) traces the
structures assigned to it, and the only communication is one gather of the
per-structure results to rank 0 (integer block sums and their summaries, a
few hundred bytes per structure).  Structures are assigned by longest
processing time first on an estimated cost (rays x log2(atoms)), which keeps
the ranks' work within one structure of each other.
"""
from __future__ import annotations

import heapq
import math


def estimated_cost(n_atoms, rays):
    return float(rays) * (1.0 + math.log2(max(2, int(n_atoms))))


def shard(costs, world):
    """Rank of each item (LPT: largest first onto the least-loaded rank)."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    owner = [0] * len(costs)
    for i in order:
        load, r = heapq.heappop(heap)
        owner[i] = r
        heapq.heappush(heap, (load + costs[i], r))
    return owner


def run_sharded(structures, log2s, seeds, run_local, rank, world, group=None):
    """Each rank runs its shard with run_local(indices) -> {index: result};
    rank 0 receives every structure's result (None on other ranks)."""
    import torch.distributed as dist
    costs = [estimated_cost(len(r), (1 << lg)) for (_, r), lg in zip(structures, log2s)]
    owner = shard(costs, world)
    mine = [i for i, o in enumerate(owner) if o == rank]
    local = run_local(mine) if mine else {}
    if world == 1:
        return [local[i] for i in range(len(structures))]
    gathered = [None] * world if rank == 0 else None
    dist.gather_object(local, gathered, dst=0, group=group)
    if rank != 0:
        return None
    merged = {}
    for part in gathered:
        merged.update(part)
    return [merged[i] for i in range(len(structures))]
