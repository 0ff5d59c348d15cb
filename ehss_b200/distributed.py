"""Several GPUs, one process per GPU: two ways to split one job.

Rays, replicate blocks and structures are independent, so nothing crosses
between GPUs while they trace.  The one exchange is the block results: every
block's totals are integers (fixed-point angle sums, counts, histograms), so
partial results add up exactly, whichever GPU traced which rays.

* Structure shards (``ShardedBatch``, ``run_sharded``): a batch of many
  structures is assigned to ranks by longest processing time first on an
  estimated cost, rays x (1 + log2 atoms); each rank builds and traces only
  its own structures.  One all-reduce (sum) of a global integer result buffer
  (or one gather of per-structure summaries) completes the job.
* Ray windows (``trace_window_split``): the blocks of one large structure
  (or any plan) are cut into contiguous windows of the chunk list of about
  equal estimated cost; every rank holds the scenes and traces its window;
  one all-reduce (sum) of the packed block results gives every rank the
  totals of the whole plan, equal to a single launch's bit for bit.

This is the reference's parallel loop over rays (prange,
src/support_exchange_transport/ehss_cpu.py:72; OpenMP,
src/native/ehss_cpu.cpp:49-53) carried across devices.  The exchange is a
few KB per structure; NCCL carries it (gloo in the CPU tests).
"""
from __future__ import annotations

import heapq
import math

import numpy as np


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


def chunk_windows(costs, world):
    """Cut a chunk list with per-chunk ``costs`` into ``world`` contiguous
    windows [first, end) of about equal total cost (window r ends where the
    running cost first exceeds (r + 1) / world of the total)."""
    c = np.cumsum(np.asarray(costs, dtype=np.float64))
    n = len(c)
    total = float(c[-1]) if n else 0.0
    cuts = [0]
    for r in range(1, world):
        cut = int(np.searchsorted(c, total * r / world, side='right')) if total > 0 else n * r // world
        cuts.append(min(max(cut, cuts[-1]), n))
    cuts.append(n)
    return [(cuts[r], cuts[r + 1]) for r in range(world)]


def trace_window_split(plan, rank, world, group=None):
    """Rank ``rank`` of ``world`` traces its window of ``plan``'s chunks; the
    packed integer results are summed over the ranks, so afterwards every
    rank's ``plan.fetch()``/``readout`` hold the whole plan's totals.
    Returns the windows."""
    windows = chunk_windows(plan.chunk_costs(), world)
    plan.window = windows[rank]
    plan.enqueue()
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(plan.packed, op=dist.ReduceOp.SUM, group=group)
    return windows


def global_index(mine, S, R, W, H1):
    """Positions, in a whole batch's packed result buffer (S structures x R
    replicates: W result words per block, then H1 histogram entries and H1
    ledger entries per block), of the elements of a plan that holds only the
    structures ``mine`` (in that order, R replicates each)."""
    if not len(mine):
        return np.zeros(0, dtype=np.int64)
    blocks = np.array([s * R + k for s in mine for k in range(R)], dtype=np.int64)
    res = (blocks[:, None] * W + np.arange(W)[None, :]).ravel()
    hist = (blocks[:, None] * H1 + np.arange(H1)[None, :]).ravel()
    return np.concatenate([res, S * R * W + hist, S * R * W + S * R * H1 + hist])


class ShardedBatch:
    """One batch of structures (``BatchCCS`` arguments) split over ranks by
    structure.  Each rank builds and traces its LPT share; ``exchange``
    scatters the rank's packed block results into a buffer laid out for the
    whole batch (block b = structure * repeats + replicate; cap + 1
    histogram and ledger entries per block) and sums it over the ranks, so
    every rank ends with every block's totals."""

    def __init__(self, structures, log2s, seeds, rank, world, group=None, repeats=3, cap=64, batch_factory=None,
                 **batch_kw):
        from .blocks import _RESULT_WORDS
        from .device import torch
        t = torch()
        self.rank, self.world, self.group = rank, world, group
        self.repeats, self.cap = int(repeats), int(cap)
        costs = [estimated_cost(len(r), 1 << int(lg)) for (_, r), lg in zip(structures, log2s)]
        owner = shard(costs, world)
        self.mine = [i for i, o in enumerate(owner) if o == rank]
        self.n_structures = len(structures)
        S, R, H1, W = len(structures), self.repeats, self.cap + 1, _RESULT_WORDS
        self.batch = None
        if self.mine:
            if batch_factory is None:
                from .batch import BatchCCS as batch_factory
            self.batch = batch_factory([structures[i] for i in self.mine], [log2s[i] for i in self.mine],
                                       [seeds[i] for i in self.mine], repeats=repeats, cap=cap, **batch_kw)
            device = self.batch.device
        else:
            device = t.device('cuda', t.cuda.current_device()) if t.cuda.is_available() else t.device('cpu')
        # where each element of the local packed buffer goes in the global one
        self.global_words = S * R * W + 2 * S * R * H1
        idx = global_index(self.mine, S, R, W, H1)
        if self.mine and len(idx) != self.batch.plan.packed.numel():
            raise ValueError('every block of the batch must have the same cap (the global layout assumes cap + 1 '
                             'histogram entries per block)')
        self.index = t.as_tensor(idx, device=device)
        self.packed = t.zeros(self.global_words, dtype=t.int64, device=device)
        self.rays = sum((1 << int(log2s[i])) * R for i in range(S))
        self._structures, self._log2s = structures, [int(x) for x in log2s]
        self.local_rays = self.batch.rays if self.batch is not None else 0

    def upload(self):
        if self.batch is not None:
            self.batch.upload()

    def build(self):
        if self.batch is not None:
            self.batch.build()

    def trace(self):
        if self.batch is not None:
            self.batch.trace()

    def scatter(self):
        """This rank's block results placed in the whole batch's layout."""
        self.packed.zero_()
        if self.batch is not None:
            self.packed.index_copy_(0, self.index, self.batch.plan.packed)
        return self.packed

    def exchange(self):
        self.scatter()
        if self.world > 1:
            import torch.distributed as dist
            dist.all_reduce(self.packed, op=dist.ReduceOp.SUM, group=self.group)
        return self.packed

    def step(self):
        self.build()
        self.trace()
        return self.exchange()

    def summaries(self):
        """Every structure's EHSS over its replicates (mean, sd, sem), mean
        tail bound and unresolved rays, from the exchanged integers: the same
        numbers on every rank, and the same as one GPU's BatchCCS.  The block
        weights need each structure's impact-disk radius, so every
        structure's real coordinates must have been passed in."""
        from . import _lib
        from .batch import enclosing_radius, summarize
        from .blocks import _RESULT_WORDS
        S, R, W = self.n_structures, self.repeats, _RESULT_WORDS
        packed = self.packed.cpu().numpy().view(np.uint64)
        res = packed[:S * R * W].reshape(S * R, W)
        out = []
        for s, ((c, r), lg) in enumerate(zip(self._structures, self._log2s)):
            radius = enclosing_radius(c, r)
            w = np.pi * radius * radius / float(1 << lg)
            rows = res[s * R:(s + 1) * R]
            ehss = w * (rows[:, 0].astype(np.float64) * _lib.FX_SCALE)
            out.append(dict(structure=s, ehss_angstrom2=summarize(ehss),
                            ehss_tail_bound_mean_angstrom2=float(np.mean(2 * w * rows[:, 2].astype(np.float64))),
                            ehss_unresolved_rays_total=int(rows[:, 2].sum())))
        return out
