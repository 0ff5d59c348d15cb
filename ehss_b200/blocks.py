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

_RESULT_WORDS = ct.sizeof(_lib.BlockResult) // 8
_STATS0 = _lib.BlockResult.stats.offset // 8
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
        # block totals, histograms and ledgers in one buffer: one copy back to the host
        H = max(offset, 1)
        nw = n * _RESULT_WORDS
        self.packed = t.zeros(nw + 2 * H, dtype=t.int64, device=self.device)
        self.results, self.hist, self.ledger = self.packed[:nw], self.packed[nw:nw + H], self.packed[nw + H:]
        self.hist_len = H
        self.d2h_bytes = self.packed.numel() * 8
        self._radius = [float(j.scene.radius) for j in self.jobs]
        self._w = np.array([np.pi * R * R / (1 << j.log2_rays) for R, j in zip(self._radius, self.jobs)])
        self._offsets = [int(host[i].hist_offset) for i in range(n)]
        self._w_entry = np.zeros(H)
        for i, j in enumerate(self.jobs):
            self._w_entry[self._offsets[i]:self._offsets[i] + j.cap + 1] = self._w[i]
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
        """Copy results to the host; returns one dict per block (synchronises).

        One device-to-host copy brings the block totals, histograms and
        ledgers; the read-out is vectorised over blocks.
        """
        packed = self.packed.cpu().numpy().view(np.uint64)
        n = len(self.jobs)
        nw = n * _RESULT_WORDS
        res = packed[:nw].reshape(n, _RESULT_WORDS)
        stats = res[:, _STATS0:_STATS0 + _lib.NSTATS]
        errors = stats[:, _lib.STAT_ERRORS]
        if errors.any():
            i = int(np.flatnonzero(errors)[0])
            raise _lib.EHSSDeviceError(f'block {self.jobs[i].tag!r}: {int(errors[i])} bounded device failures')
        H = self.hist_len
        hist = packed[nw:nw + H].astype(np.int64).tolist()
        ledger = (packed[nw + H:nw + 2 * H].astype(np.float64) * _lib.FX_SCALE * self._w_entry).tolist()
        w = self._w
        ehss = (w * (res[:, 0].astype(np.float64) * _lib.FX_SCALE)).tolist()
        hits, unres, esc, pab = (res[:, k].tolist() for k in (1, 2, 3, 4))
        cols = {k: stats[:, k].tolist() for k in (_lib.STAT_SPHERE, _lib.STAT_BOX, _lib.STAT_GRAZING,
                                                  _lib.STAT_FALLBACK, _lib.STAT_QUERIES)}
        wl = w.tolist()
        pa_same = (w * res[:, 1].astype(np.float64)).tolist()
        tail = (2 * w * res[:, 2].astype(np.float64)).tolist()
        pa_area = (w * res[:, 4].astype(np.float64)).tolist()
        sph, box, graz, fall, qry = (cols[k] for k in (_lib.STAT_SPHERE, _lib.STAT_BOX, _lib.STAT_GRAZING,
                                                      _lib.STAT_FALLBACK, _lib.STAT_QUERIES))
        out = []
        for i, j in enumerate(self.jobs):
            d = {'tag': j.tag, 'rays': 1 << j.log2_rays, 'weight': wl[i], 'radius': self._radius[i], 'stats': stats[i]}
            if j.ehss:
                o = self._offsets[i]
                e = o + j.cap + 1
                d.update({'ehss_angstrom2': ehss[i], 'pa_from_same_rays_angstrom2': pa_same[i],
                          'tail_bound_angstrom2': tail[i], 'unresolved_rays': unres[i], 'escaped_rays': esc[i],
                          'collision_histogram': hist[o:e], 'collision_contribution_angstrom2': ledger[o:e],
                          'sphere_tests': sph[i], 'box_tests': box[i], 'grazing_queries': graz[i],
                          'fp64_fallback_queries': fall[i], 'queries': qry[i]})
            if j.pa:
                d['pa_angstrom2'] = pa_area[i]
                d['pa_blocked_rays'] = pab[i]
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
