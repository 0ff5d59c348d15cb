"""Served form: continuous batching of cross-section requests.

Requests (one structure each) arrive over time.  The server admits them while
their device-memory footprint fits the budget, builds the LBVHs of every
newly admitted structure in one pass, and then runs *rounds*: one persistent
launch that traces one new replicate block (2^block_log2 rays) for every
active request at once.  After each round a request whose replicate values
reach relative RMSE = SEM / mean <= target (after at least min_blocks blocks)
completes and frees its memory; requests that arrived meanwhile are admitted
into the next round, so their work overlaps on the device with the requests
already running.  Each block's result is an integer sum that does not depend
on what else shares the launch, so a request's answer is the same alone and
in any mix.

Replicate seeds follow the reference CLI: seed_k = (seed + 104729 k) mod 2^32
(ccs_cli.py:190); statistics follow ccs_cli.summarize (ccs_cli.py:163-167).

The scheduling logic (``CCSServer``) is independent of the device: the
``executor`` argument supplies build/trace/release, which the tests replace
with a CPU fake.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from .blocks import seed_schedule


@dataclass
class CCSRequest:
    rid: object
    centers: np.ndarray
    radii: np.ndarray
    seed: int = 190003
    arrival: float = 0.0            # seconds on the server clock

    @classmethod
    def from_xyz(cls, rid, path, frame=1, probe_radius=1.4, units='angstrom', exclude_hydrogen=False,
                 radii_json=None, seed=190003, arrival=0.0):
        """A request for one frame of an XYZ file, read and prepared as the
        command line does (same dialect, radii table, probe radius, units and
        recentring; the same ValueError messages for bad input)."""
        from .ccs_cli import prepare_frame, radius_table, read_xyz
        frames = read_xyz(path)
        if not 1 <= int(frame) <= len(frames):
            raise ValueError(f"{Path(path).name}: --frame {frame} exceeds {len(frames)} frames")
        spheres, _ = prepare_frame(frames[int(frame) - 1], radius_table(radii_json), probe_radius, units,
                                   exclude_hydrogen)
        return cls(rid, spheres.centers, spheres.radii, seed=seed, arrival=arrival)


@dataclass
class BuildGroup:
    """Requests admitted together share one device allocation (one batched
    build), which is freed only when the last of them finishes; the group's
    bytes stay counted against the budget until then."""
    bytes: int
    members: int


@dataclass
class RequestState:
    req: CCSRequest
    footprint: int
    handle: object = None
    group: BuildGroup = None
    values: list = field(default_factory=list)
    tails: list = field(default_factory=list)
    admitted_at: float = None
    done_at: float = None
    rounds: int = 0


def rel_rmse(values):
    a = np.asarray(values, dtype=float)
    if len(a) < 2 or a.mean() == 0:
        return math.inf
    return float(a.std(ddof=1) / math.sqrt(len(a)) / abs(a.mean()))


class CCSServer:
    def __init__(self, executor, budget_bytes=8 << 30, block_log2=15, target=0.01, min_blocks=2, max_blocks=256,
                 clock=None):
        self.ex = executor
        self.budget = int(budget_bytes)
        self.block_log2 = int(block_log2)
        self.target = float(target)
        self.min_blocks = int(min_blocks)
        self.max_blocks = int(max_blocks)
        self.clock = clock or time.perf_counter
        self.t0 = self.clock()
        self.pending = []            # not yet admitted, in arrival order
        self.active = []
        self.done = {}
        self.used = 0
        self.rounds = 0
        self.rays = 0

    def now(self):
        return self.clock() - self.t0

    def submit(self, req):
        fp = self.ex.footprint(len(req.radii))
        if fp > self.budget:
            raise ValueError(f'request {req.rid!r} needs {fp} bytes of device memory, the budget is {self.budget}')
        self.pending.append(RequestState(req, fp))

    def _admit(self):
        now = self.now()
        admitted = []
        keep = []
        for st in self.pending:
            if st.req.arrival <= now and self.used + st.footprint <= self.budget:
                self.used += st.footprint
                st.admitted_at = now
                admitted.append(st)
            else:
                keep.append(st)
        self.pending = keep
        if admitted:
            handles = self.ex.build([(s.req.centers, s.req.radii) for s in admitted])
            group = BuildGroup(sum(s.footprint for s in admitted), len(admitted))
            for s, h in zip(admitted, handles):
                s.handle = h
                s.group = group
            self.active.extend(admitted)
        return admitted

    def _finish(self, s):
        """A finished request drops its handle; its group's memory returns to
        the budget when the group's last member has finished."""
        self.ex.release(s.handle)
        s.handle = None
        s.group.members -= 1
        if s.group.members == 0:
            self.used -= s.group.bytes

    def step(self):
        """Admit what has arrived and fits, then run one round; returns requests completed."""
        self._admit()
        if not self.active:
            return []
        jobs = []
        for s in self.active:
            k = len(s.values)
            # the first round of a request traces min_blocks blocks so that its RMSE is defined
            n_new = self.min_blocks if k == 0 else 1
            seeds = seed_schedule(s.req.seed, k + n_new)[k:]
            jobs.extend((s.handle, self.block_log2, seed, s) for seed in seeds)
        results = self.ex.trace([(h, lg, seed) for h, lg, seed, _ in jobs])
        self.rounds += 1
        self.rays += len(jobs) << self.block_log2
        for (_, _, _, s), (omega, tail) in zip(jobs, results):
            s.values.append(omega)
            s.tails.append(tail)
        finished = []
        now = self.now()
        still = []
        for s in self.active:
            s.rounds += 1
            if (len(s.values) >= self.min_blocks and rel_rmse(s.values) <= self.target) or \
                    len(s.values) >= self.max_blocks:
                s.done_at = now
                self._finish(s)
                a = np.asarray(s.values)
                self.done[s.req.rid] = dict(rid=s.req.rid, atoms=len(s.req.radii), ehss_mean_angstrom2=float(a.mean()),
                                            sd=float(a.std(ddof=1)) if len(a) > 1 else None, rel_rmse=rel_rmse(a),
                                            blocks=len(a), values=list(s.values),
                                            tail_bound_mean_angstrom2=float(np.mean(s.tails)),
                                            latency_s=s.done_at - s.req.arrival, admitted_s=s.admitted_at,
                                            converged=rel_rmse(a) <= self.target)
                finished.append(s.req.rid)
            else:
                still.append(s)
        self.active = still
        return finished

    def run(self, until_idle=True, timeout_s=600.0):
        """Serve until every submitted request is done (waiting for future arrivals)."""
        start = self.now()
        while self.pending or self.active:
            if not self.active and self.pending:
                nxt = min(s.req.arrival for s in self.pending)
                wait = nxt - self.now()
                if wait > 0:
                    # sleep until about 1 ms before the next arrival, then poll: a sleep
                    # overshoots by up to a scheduler tick, which would land in that
                    # request's latency
                    if wait > 2e-3:
                        time.sleep(min(wait - 1e-3, 0.05))
                    if self.now() - start > timeout_s:
                        raise TimeoutError('serving did not finish in time')
                    continue
            self.step()
            if self.now() - start > timeout_s:
                raise TimeoutError('serving did not finish in time')
        return self.done

    def latency_percentiles(self):
        lat = np.array([d['latency_s'] for d in self.done.values()])
        return dict(p50_ms=float(np.percentile(lat, 50) * 1e3), p99_ms=float(np.percentile(lat, 99) * 1e3),
                    mean_ms=float(lat.mean() * 1e3), requests=len(lat))


class DeviceExecutor:
    """The device side of the server: batched scene builds and fused block rounds."""

    def __init__(self, leaf_size=None, cap=64, precision='fp32', launch=None, device=None):
        from . import _lib
        from .device import require_cuda
        self.device = require_cuda(device)
        self.leaf_size = _lib.DEFAULT_LEAF if leaf_size is None else int(leaf_size)
        self.cap, self.launch = cap, launch
        self.precision = {'fp64': _lib.PREC_FP64, 'fp32': _lib.PREC_FP32}[precision]

    def warmup(self, sizes=(64, 4096, 12000)):
        """Build and trace one synthetic structure per builder path (per-structure
        key sorts of up to 2048 and 8192 atoms, the device-wide sort above) so
        that the first requests of each size do not wait for kernels to load."""
        rng = np.random.default_rng(0)
        for n in sizes:
            side = int(np.ceil(n ** (1. / 3.)))
            grid = np.stack(np.meshgrid(*[np.arange(side)] * 3, indexing='ij'), -1).reshape(-1, 3)[:n] * 2.5
            structure = (grid + rng.normal(0., 0.05, grid.shape), np.full(n, 1.6))
            handle = self.build([structure])[0]
            self.trace([(handle, 12, 1)])

    def footprint(self, n_atoms):
        """Device bytes one request may hold: its scene, its share of the
        build workspace and its coordinates and radii (32 B per atom).  The
        server counts them for every member of a batched build until the
        batch's last request finishes, so the budget bounds what is allocated."""
        import ctypes as ct
        from . import _lib
        sb, wb = ct.c_uint64(), ct.c_uint64()
        _lib.check(_lib.load().ehss_scene_bytes(int(n_atoms), self.leaf_size, ct.byref(sb), ct.byref(wb)))
        return int(sb.value + wb.value + 32 * int(n_atoms) + 512)

    def build(self, structures):
        from .batch import BatchScenes
        # every block ray starts on the impact disk: exterior scenes give the same outcomes
        scenes = BatchScenes(structures, leaf_size=self.leaf_size, device=self.device, exterior=True)
        scenes.build()
        scenes.drop_build_buffers()
        return [(scenes, i) for i in range(len(structures))]

    def trace(self, jobs):
        from .blocks import BlockJob, BlockPlan
        plan = BlockPlan([BlockJob(h[0].scenes[h[1]], lg, seed, cap=self.cap, precision=self.precision, tag=i)
                          for i, (h, lg, seed) in enumerate(jobs)], launch=self.launch, device=self.device)
        plan.enqueue()
        res = plan.collect()
        return [(r['ehss_angstrom2'], r['tail_bound_angstrom2']) for r in res]

    def release(self, handle):
        pass    # the batch's scene buffer goes with the last handle into it (the server drops each handle)
