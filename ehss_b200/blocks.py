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
    omega = w * angle_fx * 2^-36,  pa = w * hits,  tail = 2 * w * unresolved,
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
# chunk_rays 0: sized to the work (auto_chunk)
DEFAULT_LAUNCH = dict(block_threads=128, ctas_per_sm=8, chunk_rays=0, resolve_batch=30, smem_stack=5,
                      count_tests=False)


_SM_COUNT = {}


def _sm_count(device):
    """Multiprocessors of ``device`` (cached: the served form makes a plan per round)."""
    t = torch()
    key = t.device(device).index
    if key not in _SM_COUNT:
        _SM_COUNT[key] = t.cuda.get_device_properties(device).multi_processor_count if t.cuda.is_available() else 148
    return _SM_COUNT[key]


def auto_chunk(rays, launch, sm_count):
    """Rays per work item: 256 when every warp of the persistent grid gets
    several chunks (large batches), smaller for small jobs so that a single
    structure's blocks spread over all warps instead of queueing behind a
    few long chunks (power of two in 32..256)."""
    warps = sm_count * int(launch['ctas_per_sm']) * (int(launch['block_threads']) // 32)
    target = max(1, int(rays) // (4 * warps))
    chunk = 32
    while chunk < 256 and chunk * 2 <= target:
        chunk *= 2
    return chunk


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
    boundary: object = None       # compact.CompactBoundary: its rays and weights instead of the impact disk


class BlockPlan:
    """Device descriptors, buffers and the launch for a list of blocks.

    ``residual_capacity`` > 0 saves every ray left unresolved at its block's
    cap (position, direction, incoming direction, last collider, bounces) so
    that ``extend_caps`` can continue exactly those rays at larger caps.
    """

    def __init__(self, jobs, launch=None, device=None, residual_capacity=0):
        if not jobs:
            raise ValueError('at least one block required')
        lib = _lib.load()
        t = torch()
        self.jobs = list(jobs)
        self.device = jobs[0].scene.device if device is None else device
        L = dict(DEFAULT_LAUNCH)
        L.update(launch or {})
        if not L['chunk_rays']:
            L['chunk_rays'] = auto_chunk(sum(1 << j.log2_rays for j in self.jobs), L, _sm_count(self.device))
        precisions = 0
        for j in jobs:
            precisions |= 1 << int(j.precision)
        options = _lib.LAUNCH_COUNT_TESTS if L['count_tests'] else 0
        n_boundary = sum(j.boundary is not None for j in jobs)
        if n_boundary:
            options |= _lib.LAUNCH_RAY_BLOCKS | (_lib.LAUNCH_NO_DISK_BLOCKS if n_boundary == len(jobs) else 0)
        self.launch = _lib.Launch(int(L['block_threads']), int(L['ctas_per_sm']), int(L['chunk_rays']),
                                  int(L['resolve_batch']), precisions, options, int(L['smem_stack']), 0)
        n = len(self.jobs)
        self._ray_buffers = []
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
            if j.boundary is not None:
                # rays of an enclosing boundary, generated once on the device; weights are
                # summed relative to the largest possible one (ray_scale)
                if residual_capacity:
                    raise ValueError('cap extension needs impact-disk blocks; boundary blocks keep their cap')
                nr = 1 << int(j.log2_rays)
                buf = t.empty(7 * nr, dtype=t.float64, device=self.device)
                j.boundary.fill_ray_buffer(int(j.log2_rays), int(j.seed), buf)
                self._ray_buffers.append(buf)
                b.flags |= _lib.BLOCK_RAYS
                b.rays = buf.data_ptr()
                b.ray_scale = nr / j.boundary.max_projected_area()
            b.hist_offset = offset
            offset += j.cap + 1
            seeds[i] = int(j.seed)
        total = ct.c_int64()
        _lib.check(lib.ehss_blocks_prepare(host, n, seeds, self.launch.chunk_rays, ct.byref(total)), 'blocks')
        self.total_chunks = total.value
        self.chunk_begin = [int(host[i].chunk_begin) for i in range(n)]
        self.window = None          # (first, end): trace only these chunks (one GPU's share)
        self.hist_entries = offset
        # descriptors through pinned memory: the upload does not wait for earlier work on the stream
        self._blocks_host = t.empty(ct.sizeof(host), dtype=t.uint8,
                                    pin_memory=t.device(self.device).type == 'cuda')
        ct.memmove(self._blocks_host.data_ptr(), ct.addressof(host), ct.sizeof(host))
        self.blocks_dev = self._blocks_host.to(self.device, non_blocking=True)
        # block totals, histograms and ledgers in one buffer: one copy back to the host
        H = max(offset, 1)
        nw = n * _RESULT_WORDS
        self.packed = t.zeros(nw + 2 * H, dtype=t.int64, device=self.device)
        self.results, self.hist, self.ledger = self.packed[:nw], self.packed[nw:nw + H], self.packed[nw + H:]
        self.hist_len = H
        self.d2h_bytes = self.packed.numel() * 8
        self._radius = [float(j.scene.radius) for j in self.jobs]
        # weight per ray (impact disk) or the reference weight of a boundary block's weighted sums
        self._w = np.array([1.0 / host[i].ray_scale if j.boundary is not None else np.pi * R * R / (1 << j.log2_rays)
                            for i, (R, j) in enumerate(zip(self._radius, self.jobs))])
        self._weighted = np.array([j.boundary is not None for j in self.jobs])
        self._offsets = [int(host[i].hist_offset) for i in range(n)]
        self._w_entry = np.zeros(H)
        for i, j in enumerate(self.jobs):
            self._w_entry[self._offsets[i]:self._offsets[i] + j.cap + 1] = self._w[i]
        wb = ct.c_uint64()
        _lib.check(lib.ehss_blocks_workspace_bytes(n, ct.byref(wb)), 'blocks')
        self.work = t.zeros(int(wb.value) // 8 + 1, dtype=t.int64, device=self.device)
        self.graph = None
        self.rays = sum(1 << j.log2_rays for j in self.jobs)
        self.residual = None
        self.residual_capacity = 0
        self.residual_count = t.zeros(1, dtype=t.int64, device=self.device)
        if residual_capacity:
            self._alloc_residual(int(residual_capacity))

    def _alloc_residual(self, capacity):
        t = torch()
        self.residual_capacity = max(1, int(capacity))
        self.residual = t.empty(self.residual_capacity * ct.sizeof(_lib.Residual), dtype=t.uint8, device=self.device)
        self.graph = None           # a captured launch holds the old buffer

    def enqueue(self, stream=None):
        """Enqueue the launch on the current (or given) CUDA stream."""
        lib = _lib.load()
        s = stream_handle(self.device) if stream is None else stream
        if self.window is not None:
            if self.residual is not None:
                raise ValueError('a chunk window traces part of each block: no residual rays are saved')
            first, end = self.window
            _lib.check(lib.ehss_trace_blocks_window(ptr(self.blocks_dev), len(self.jobs), self.total_chunks, int(first),
                                                    int(end), ptr(self.results), ptr(self.hist), ptr(self.ledger),
                                                    self.hist_entries, ptr(self.work), self.work.numel() * 8,
                                                    ct.byref(self.launch), s), 'trace blocks (window)')
        elif self.residual is None:
            _lib.check(lib.ehss_trace_blocks(ptr(self.blocks_dev), len(self.jobs), self.total_chunks,
                                             ptr(self.results), ptr(self.hist), ptr(self.ledger), self.hist_entries,
                                             ptr(self.work), self.work.numel() * 8, ct.byref(self.launch), s),
                       'trace blocks')
        else:
            _lib.check(lib.ehss_trace_blocks_residual(ptr(self.blocks_dev), len(self.jobs), self.total_chunks,
                                                      ptr(self.results), ptr(self.hist), ptr(self.ledger),
                                                      self.hist_entries, ptr(self.work), self.work.numel() * 8,
                                                      ct.byref(self.launch), ptr(self.residual),
                                                      self.residual_capacity, ptr(self.residual_count), s),
                       'trace blocks')

    def chunk_costs(self):
        """Estimated cost of every chunk (rays x (1 + log2 atoms) of its block),
        in chunk order: the weights for cutting the chunk list into windows."""
        out = np.zeros(self.total_chunks)
        cr = self.launch.chunk_rays
        for j, begin in zip(self.jobs, self.chunk_begin):
            n = 1 << j.log2_rays
            k = -(-n // cr)
            per_ray = 1.0 + math.log2(max(2, int(j.scene.n_atoms)))
            out[begin:begin + k] = per_ray * np.minimum(cr, n - cr * np.arange(k))
        return out

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

    def fetch(self):
        """One device-to-host copy of every block's totals, histogram and
        ledger (synchronises); raises if a block reported a device failure."""
        packed = self.packed.cpu().numpy().view(np.uint64)
        n = len(self.jobs)
        res = packed[:n * _RESULT_WORDS].reshape(n, _RESULT_WORDS)
        errors = res[:, _STATS0 + _lib.STAT_ERRORS]
        if errors.any():
            i = int(np.flatnonzero(errors)[0])
            raise _lib.EHSSDeviceError(f'block {self.jobs[i].tag!r}: {int(errors[i])} bounded device failures')
        return packed

    def totals(self, packed):
        """Per-block EHSS, tail bound and PA (float64 arrays, same arithmetic as
        ``readout``) and unresolved counts from a ``fetch`` result."""
        n = len(self.jobs)
        res = packed[:n * _RESULT_WORDS].reshape(n, _RESULT_WORDS)
        w = self._w
        _, unres_w, pa_w = self._weighted_counts(res)
        return dict(ehss=w * (res[:, 0].astype(np.float64) * _lib.FX_SCALE), tail=2 * w * unres_w,
                    pa=w * pa_w, unresolved=res[:, 2].astype(np.int64))

    def _weighted_counts(self, res):
        """Hits, unresolved and PA hits as float64: counts for impact-disk blocks,
        weighted sums (in units of the reference weight) for boundary blocks."""
        out = []
        for cnt, fx in ((1, 5), (2, 6), (4, 7)):
            c = res[:, cnt].astype(np.float64)
            if self._weighted.any():
                c = np.where(self._weighted, res[:, fx].astype(np.float64) * _lib.FX_SCALE, c)
            out.append(c)
        return out

    def collect(self):
        """Copy results to the host; returns one dict per block (synchronises)."""
        return self.readout(self.fetch())

    def readout(self, packed):
        """One dict per block from a ``fetch`` result (vectorised over blocks)."""
        n = len(self.jobs)
        nw = n * _RESULT_WORDS
        res = packed[:nw].reshape(n, _RESULT_WORDS)
        stats = res[:, _STATS0:_STATS0 + _lib.NSTATS]
        H = self.hist_len
        hist = packed[nw:nw + H].astype(np.int64).tolist()
        ledger = (packed[nw + H:nw + 2 * H].astype(np.float64) * _lib.FX_SCALE * self._w_entry).tolist()
        w = self._w
        ehss = (w * (res[:, 0].astype(np.float64) * _lib.FX_SCALE)).tolist()
        hits, unres, esc, pab = (res[:, k].tolist() for k in (1, 2, 3, 4))
        cols = {k: stats[:, k].tolist() for k in (_lib.STAT_SPHERE, _lib.STAT_BOX, _lib.STAT_GRAZING,
                                                  _lib.STAT_FALLBACK, _lib.STAT_QUERIES)}
        wl = w.tolist()
        hits_w, unres_w, pa_w = self._weighted_counts(res)
        pa_same = (w * hits_w).tolist()
        tail = (2 * w * unres_w).tolist()
        pa_area = (w * pa_w).tolist()
        sph, box, graz, fall, qry = (cols[k] for k in (_lib.STAT_SPHERE, _lib.STAT_BOX, _lib.STAT_GRAZING,
                                                      _lib.STAT_FALLBACK, _lib.STAT_QUERIES))
        out = []
        for i, j in enumerate(self.jobs):
            d = {'tag': j.tag, 'rays': 1 << j.log2_rays, 'weight': wl[i], 'radius': self._radius[i], 'stats': stats[i],
                 'sphere_tests': sph[i], 'box_tests': box[i]}
            if j.ehss:
                o = self._offsets[i]
                e = o + j.cap + 1
                d.update({'ehss_angstrom2': ehss[i], 'pa_from_same_rays_angstrom2': pa_same[i],
                          'tail_bound_angstrom2': tail[i], 'unresolved_rays': unres[i], 'escaped_rays': esc[i],
                          'collision_histogram': hist[o:e], 'collision_contribution_angstrom2': ledger[o:e],
                          'grazing_queries': graz[i],
                          'fp64_fallback_queries': fall[i], 'queries': qry[i]})
            if j.pa:
                d['pa_angstrom2'] = pa_area[i]
                d['pa_blocked_rays'] = pab[i]
            out.append(d)
        return out


    def extend_caps(self, caps, tail_fraction=5e-4, results=None):
        """Cap-extension ladder: continue the unresolved rays of every block
        whose sampled tail bound exceeds ``tail_fraction`` of its CCS at each
        cap of ``caps`` in turn (the reference's production rule: 512, then
        1024, 2048 and 4096 while the bound exceeds 0.05 %).  Only the saved
        unresolved rays are traced again, from their exact state, so each
        block's totals equal a run at its final cap.  Returns the block dicts
        of ``collect`` updated to the final caps, each with ``cap`` and the
        list ``cap_attempts`` (cap, CCS, tail bound, unresolved and continued
        rays, seconds)."""
        import time
        if self.residual is None:
            raise ValueError('the plan was built without residual_capacity: nothing was saved to extend')
        t = torch()
        lib = _lib.load()
        res = self.collect() if results is None else results
        count = int(self.residual_count.item())
        if count > self.residual_capacity:
            # the saved rays overflowed: trace again with room for all of them (same results)
            self._alloc_residual(count)
            self.enqueue()
            res = self.collect()
            count = int(self.residual_count.item())
        n = len(self.jobs)
        H, nw = self.hist_len, n * _RESULT_WORDS
        packed = self.packed.cpu().numpy().view(np.uint64)
        raw = packed[:nw].reshape(n, _RESULT_WORDS)
        state = []
        for i, j in enumerate(self.jobs):
            o = self._offsets[i]
            state.append(dict(cap=j.cap, angle_fx=int(raw[i, 0]), escaped=int(raw[i, 3]), unresolved=int(raw[i, 2]),
                              hist=[int(x) for x in packed[nw + o:nw + o + j.cap + 1]],
                              ledger=[int(x) for x in packed[nw + H + o:nw + H + o + j.cap + 1]]))
        attempts = [[dict(cap=j.cap, ehss_angstrom2=r.get('ehss_angstrom2'), tail_bound_angstrom2=r.get(
            'tail_bound_angstrom2'), unresolved_rays=r.get('unresolved_rays'), continued_rays=0, seconds=0.0)]
                    for j, r in zip(self.jobs, res)]
        queue, n_in = self.residual, min(count, self.residual_capacity)
        stream = stream_handle(self.device)
        for new_cap in caps:
            new_cap = int(new_cap)
            need = [i for i, (j, st) in enumerate(zip(self.jobs, state))
                    if j.ehss and st['unresolved'] and st['cap'] < new_cap and
                    2 * self._w[i] * st['unresolved'] > tail_fraction * self._w[i] * st['angle_fx'] * _lib.FX_SCALE]
            if not need or n_in == 0:
                break
            tick = time.perf_counter()
            rows = len(need)
            row_of = np.full(n, -1, dtype=np.int32)
            row_of[need] = np.arange(rows, dtype=np.int32)
            row_dev = t.from_numpy(row_of).to(self.device)
            ext = t.zeros(rows * ct.sizeof(_lib.Extension), dtype=t.uint8, device=self.device)
            eh = t.zeros(rows * (new_cap + 1), dtype=t.int64, device=self.device)
            el = t.zeros(rows * (new_cap + 1), dtype=t.int64, device=self.device)
            out = t.empty(max(1, n_in) * ct.sizeof(_lib.Residual), dtype=t.uint8, device=self.device)
            out_count = t.zeros(1, dtype=t.int64, device=self.device)
            stats = t.zeros(_lib.NSTATS, dtype=t.int64, device=self.device)
            _lib.check(lib.ehss_extend_blocks(ptr(self.blocks_dev), n, ptr(row_dev), rows, ptr(queue), n_in, new_cap,
                                              ptr(ext), ptr(eh), ptr(el), ptr(out), max(1, n_in), ptr(out_count),
                                              ptr(stats), stream), 'cap extension')
            e = ext.cpu().numpy().view(np.uint64).reshape(rows, 4)
            ehh = eh.cpu().numpy().view(np.uint64).reshape(rows, new_cap + 1)
            ell = el.cpu().numpy().view(np.uint64).reshape(rows, new_cap + 1)
            st_dev = stats.cpu().numpy()
            if st_dev[_lib.STAT_ERRORS]:
                raise _lib.EHSSDeviceError(f'cap extension: {int(st_dev[_lib.STAT_ERRORS])} bounded device failures')
            secs = time.perf_counter() - tick
            for r, i in enumerate(need):
                st = state[i]
                cont = merge_extension(st, e[r], ehh[r], ell[r], new_cap)
                w = float(self._w[i])
                attempts[i].append(dict(cap=new_cap, ehss_angstrom2=w * (st['angle_fx'] * _lib.FX_SCALE),
                                        tail_bound_angstrom2=2 * w * st['unresolved'],
                                        unresolved_rays=st['unresolved'], continued_rays=cont, seconds=secs))
            queue, n_in = out, int(out_count.item())
        final = []
        for i, (r, st) in enumerate(zip(res, state)):
            d = dict(r)
            w = float(self._w[i])
            if self.jobs[i].ehss:
                d.update(ehss_angstrom2=w * (st['angle_fx'] * _lib.FX_SCALE), tail_bound_angstrom2=2 * w * st['unresolved'],
                         unresolved_rays=st['unresolved'], escaped_rays=st['escaped'], collision_histogram=st['hist'],
                         collision_contribution_angstrom2=[x * _lib.FX_SCALE * w for x in st['ledger']])
            d.update(cap=st['cap'], cap_attempts=attempts[i])
            final.append(d)
        return final


def merge_extension(st, ext, hist, ledger, new_cap):
    """Fold one block's cap extension into its integer totals.  ``st`` holds
    cap, angle_fx, escaped, unresolved and the hist/ledger lists (cap + 1
    entries); ``ext`` = (angle_fx, escaped, unresolved, continued) of the
    continued rays and hist/ledger their rows (new_cap + 1 entries).  The
    continued rays all stood at bounces == cap, so they leave that bin.
    Returns the number of continued rays."""
    angle, esc, unres, cont = (int(x) for x in ext)
    old = st['cap']
    st['hist'] += [0] * (new_cap - old)
    st['ledger'] += [0] * (new_cap - old)
    st['hist'][old] -= cont
    for k in range(old, new_cap + 1):
        st['hist'][k] += int(hist[k])
        st['ledger'][k] += int(ledger[k])
    st['angle_fx'] += angle
    st['escaped'] += esc
    st['unresolved'] += unres - cont
    st['cap'] = new_cap
    return cont


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
