"""Fused Sobol -> impact disk -> EHSS/PA -> reduction over many blocks.

One *block* is one replicate of one structure: 2**log2_rays rays drawn from
Sobol(4, seed) on that structure's impact disk, traced and reduced on the
device with no per-ray HBM traffic (the body of the reference's repeat loop,
ccs_cli.solve_frame, src/support_exchange_transport/ccs_cli.py:189-219).
A ``BlockPlan`` holds the device descriptors of any mix of structures and
replicates and runs them in one persistent launch; ``capture()`` records that
launch in a CUDA graph so repeated runs cost one graph replay.

Totals come back as integers (fixed point for angle sums), so every block's
result is independent of what else shares the launch:
    omega = w * angle_fx * 2^-40,  pa = w * hits,  tail = 2 * w * unresolved,
with w = pi R^2 / 2**log2_rays.
"""
from __future__ import annotations

import ctypes as ct
import math
from dataclasses import dataclass

import numpy as np

from . import _lib
from .device import empty, ptr, stream_handle, torch

DEFAULT_LAUNCH = dict(block_threads=128, ctas_per_sm=6, chunk_rays=256, resolve_batch=24, smem_stack=8,
                      count_tests=False)


@dataclass
class BlockJob:
    scene: object                 # engine.Scene
    log2_rays: int
    seed: int
    cap: int = 64
    precision: int = _lib.PREC_FP32
    ehss: bool = True
    pa: bool = False
    tag: object = None


class BlockPlan:
    def __init__(self, jobs, launch=None, device=None):
        if not jobs:
            raise ValueError('at least one block required')
        lib = _lib.load()
        t = torch()
        self.jobs = list(jobs)
        self.device = jobs[0].scene.device if device is None else device
        L = dict(DEFAULT_LAUNCH)
        L.update(launch or {})
        precisions = 0
        for j in jobs:
            precisions |= 1 << int(j.precision)
        self.launch = _lib.Launch(int(L['block_threads']), int(L['ctas_per_sm']), int(L['chunk_rays']),
                                  int(L['resolve_batch']), precisions,
                                  _lib.LAUNCH_COUNT_TESTS if L['count_tests'] else 0, int(L['smem_stack']), 0)
        n = len(self.jobs)
        host = (_lib.Block * n)()
        seeds = (ct.c_uint64 * n)()
        offset = 0
        for i, j in enumerate(self.jobs):
            if type(j.cap) is not int or j.cap < 1:
                raise ValueError('Positive integer cap required')
            b = host[i]
            b.scene = j.scene.ptr
            b.log2_rays = int(j.log2_rays)
            b.cap = int(j.cap)
            b.precision = int(j.precision)
            b.flags = (_lib.BLOCK_EHSS if j.ehss else 0) | (_lib.BLOCK_PA if j.pa else 0)
            b.hist_offset = offset
            offset += j.cap + 1
            seeds[i] = int(j.seed)
        total = ct.c_int64()
        _lib.check(lib.ehss_blocks_prepare(host, n, seeds, self.launch.chunk_rays, ct.byref(total)), 'blocks')
        self.total_chunks = total.value
        self.hist_entries = offset
        raw = np.frombuffer(bytes(host), dtype=np.uint8)
        self.blocks_dev = t.from_numpy(raw.copy()).to(self.device)
        self.results = t.zeros(n * ct.sizeof(_lib.BlockResult), dtype=t.uint8, device=self.device)
        self.hist = t.zeros(max(offset, 1), dtype=t.int64, device=self.device)
        self.ledger = t.zeros(max(offset, 1), dtype=t.int64, device=self.device)
        wb = ct.c_uint64()
        _lib.check(lib.ehss_blocks_workspace_bytes(n, ct.byref(wb)), 'blocks')
        self.work = t.zeros(int(wb.value) // 8 + 1, dtype=t.int64, device=self.device)
        self.graph = None
        self.rays = sum(1 << j.log2_rays for j in self.jobs)

    def enqueue(self, stream=None):
        """Enqueue the launch on the current (or given) CUDA stream."""
        lib = _lib.load()
        s = stream_handle(self.device) if stream is None else stream
        _lib.check(lib.ehss_trace_blocks(ptr(self.blocks_dev), len(self.jobs), self.total_chunks, ptr(self.results),
                                         ptr(self.hist), ptr(self.ledger), self.hist_entries, ptr(self.work),
                                         self.work.numel() * 8, ct.byref(self.launch), s), 'trace blocks')

    def capture(self):
        """Record the launch (resets + persistent kernel) in a CUDA graph."""
        t = torch()
        side = t.cuda.Stream(self.device)
        side.wait_stream(t.cuda.current_stream(self.device))
        with t.cuda.stream(side):
            self.enqueue()          # warm-up outside capture (module load, first-launch costs)
        t.cuda.current_stream(self.device).wait_stream(side)
        g = t.cuda.CUDAGraph()
        with t.cuda.graph(g):
            self.enqueue()
        self.graph = g
        return g

    def run(self):
        if self.graph is not None:
            self.graph.replay()
        else:
            self.enqueue()

    def collect(self):
        """Copy results to the host; returns one dict per block (synchronises)."""
        raw = self.results.cpu().numpy().tobytes()
        res = (_lib.BlockResult * len(self.jobs)).from_buffer_copy(raw)
        hist = self.hist.cpu().numpy().astype(np.int64)
        ledger = self.ledger.cpu().numpy().astype(np.uint64)
        out = []
        offset = 0
        for j, r in zip(self.jobs, res):
            n = 1 << j.log2_rays
            R = j.scene.radius
            w = np.pi * R * R / n
            stats = np.array(r.stats[:], dtype=np.uint64)
            if stats[_lib.STAT_ERRORS]:
                raise _lib.EHSSDeviceError(f'block {j.tag!r}: {int(stats[_lib.STAT_ERRORS])} bounded device failures')
            h = hist[offset:offset + j.cap + 1]
            lg = ledger[offset:offset + j.cap + 1].astype(np.float64) * _lib.FX_SCALE * w
            offset += j.cap + 1
            angle = r.angle_fx * _lib.FX_SCALE
            d = dict(tag=j.tag, rays=n, weight=w, radius=R, stats=stats)
            if j.ehss:
                d.update(ehss_angstrom2=w * angle, pa_from_same_rays_angstrom2=w * r.hits,
                         tail_bound_angstrom2=2 * w * r.unresolved, unresolved_rays=int(r.unresolved),
                         escaped_rays=int(r.escaped), collision_histogram=h.tolist(),
                         collision_contribution_angstrom2=lg.tolist(),
                         sphere_tests=int(stats[_lib.STAT_SPHERE]), box_tests=int(stats[_lib.STAT_BOX]),
                         grazing_queries=int(stats[_lib.STAT_GRAZING]),
                         fp64_fallback_queries=int(stats[_lib.STAT_FALLBACK]), queries=int(stats[_lib.STAT_QUERIES]))
            if j.pa:
                d.update(pa_angstrom2=w * r.pa_blocked, pa_blocked_rays=int(r.pa_blocked))
            out.append(d)
        return out


def seed_schedule(seed, repeats):
    """Replicate seeds of the reference CLI: (seed + 104729 k) mod 2^32 (ccs_cli.py:190)."""
    return [(int(seed) + 104729 * k) % (2 ** 32) for k in range(int(repeats))]


def log2_exact(n):
    k = int(n).bit_length() - 1
    if n < 1 or (1 << k) != n:
        raise ValueError('ray count must be a power of two')
    return k


def ceil_log2(x):
    return int(math.ceil(math.log2(x)))
