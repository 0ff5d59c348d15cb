"""Batched cross sections: many structures, one build pass, one persistent launch.

``BatchCCS`` is the public entry for the batched form: it takes host arrays
of many structures of uneven size, stages them in pinned memory, builds every
LBVH in one pass of the builder kernels (ehss_scenes_build_ex; exterior
scenes by default, since every block ray starts outside the union), runs all
(structure, replicate) blocks in one persistent launch (optionally replayed
from a CUDA graph) and returns per-structure EHSS/PA summaries with the
reference CLI's replicate statistics (ccs_cli.summarize, ccs_cli.py:163-167).
"""
from __future__ import annotations

import ctypes as ct
import math
from collections.abc import Sequence

import numpy as np

from . import _lib
from .blocks import BlockJob, BlockPlan, seed_schedule
from .device import require_cuda, stream_handle, torch


def enclosing_radius(centers, radii):
    """Impact-disk radius exactly as the device computes it (ehss_state.py:46-47;
    ehss_enclosing_radius, host code)."""
    c = np.ascontiguousarray(centers, dtype=np.float64)
    r = np.ascontiguousarray(radii, dtype=np.float64)
    out = ct.c_double()
    _lib.check(_lib.load().ehss_enclosing_radius(len(r), c.ctypes.data, r.ctypes.data, ct.byref(out)), 'radius')
    return out.value


def summarize(values):
    a = np.asarray(values, dtype=float)
    sd = float(a.std(ddof=1)) if len(a) > 1 else None
    return dict(mean=float(a.mean()), sd=sd, sem=sd / math.sqrt(len(a)) if sd is not None else None,
                replicates=len(a))


class SceneRef:
    """A scene inside a batch buffer (what BlockPlan needs of a scene)."""

    def __init__(self, ptr, radius, n_atoms, device):
        self.ptr, self.radius, self.n_atoms, self.device = ptr, radius, n_atoms, device


class BatchScenes:
    """Many structures' scenes in one device allocation, built in one pass.

    ``exterior=True`` builds exterior scenes (EHSS_BUILD_EXTERIOR): atoms
    buried under their neighbours are left out of the trees, which the fused
    block trace may use because all its rays start outside the union.
    """

    def __init__(self, structures, leaf_size=_lib.DEFAULT_LEAF, device=None, exterior=False):
        lib = _lib.load()
        t = torch()
        self.device = require_cuda(device)
        S = len(structures)
        if S < 1:
            raise ValueError('at least one structure required')
        self.n_atoms = np.array([len(r) for _, r in structures], dtype=np.int64)
        if np.any(self.n_atoms < 1):
            raise ValueError('every structure needs at least one atom')
        N = int(self.n_atoms.sum())
        self.atom0 = np.concatenate([[0], np.cumsum(self.n_atoms)[:-1]])
        # pinned host staging, one contiguous copy per array
        self.h_xyz = t.empty(N * 3, dtype=t.float64, pin_memory=True)
        self.h_r = t.empty(N, dtype=t.float64, pin_memory=True)
        hx, hr = self.h_xyz.numpy(), self.h_r.numpy()
        radii = []
        for (c, r), a0, n in zip(structures, self.atom0, self.n_atoms):
            c = np.ascontiguousarray(c, dtype=np.float64); r = np.ascontiguousarray(r, dtype=np.float64)
            if c.shape != (n, 3) or not np.isfinite(c).all() or not np.isfinite(r).all() or np.any(r <= 0):
                raise ValueError('Finite centers (N,3) and positive finite radii required.')
            hx[3 * a0:3 * (a0 + n)] = c.ravel()
            hr[a0:a0 + n] = r
            radii.append(enclosing_radius(c, r))
        self.d_xyz = t.empty(N * 3, dtype=t.float64, device=self.device)
        self.d_r = t.empty(N, dtype=t.float64, device=self.device)
        sizes = []
        for n in self.n_atoms:
            sb, wb = ct.c_uint64(), ct.c_uint64()
            _lib.check(lib.ehss_scene_bytes(int(n), int(leaf_size), ct.byref(sb), ct.byref(wb)), 'scene size')
            sizes.append(sb.value)
        offs = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
        self.scene_buf = t.empty(int(sum(sizes)) + 256, dtype=t.uint8, device=self.device)
        base = (self.scene_buf.data_ptr() + 255) & ~255
        self.scene_ptrs = [base + int(o) for o in offs]
        wb = ct.c_uint64()
        _lib.check(lib.ehss_scenes_workspace_bytes(S, (ct.c_int64 * S)(*self.n_atoms), ct.byref(wb)), 'workspace')
        self.ws = t.empty(int(wb.value) + 256, dtype=t.uint8, device=self.device)
        self.ws_ptr = (self.ws.data_ptr() + 255) & ~255
        self.ws_bytes = int(wb.value)
        xp = self.d_xyz.data_ptr(); rp = self.d_r.data_ptr()
        self._xyz_ptrs = (ct.c_void_p * S)(*[xp + 24 * int(a) for a in self.atom0])
        self._r_ptrs = (ct.c_void_p * S)(*[rp + 8 * int(a) for a in self.atom0])
        self._n = (ct.c_int64 * S)(*self.n_atoms)
        self._scenes = (ct.c_void_p * S)(*self.scene_ptrs)
        self._sizes = (ct.c_uint64 * S)(*sizes)
        self.leaf_size = int(leaf_size)
        self.flags = _lib.BUILD_EXTERIOR if exterior else 0
        self.scenes = [SceneRef(p, R, int(n), self.device) for p, R, n in zip(self.scene_ptrs, radii, self.n_atoms)]
        self.h2d_bytes = (N * 3 + N) * 8

    def upload(self):
        self._require_build_buffers()
        self.d_xyz.copy_(self.h_xyz, non_blocking=True)
        self.d_r.copy_(self.h_r, non_blocking=True)

    def build(self, upload=True):
        self._require_build_buffers()
        if upload:
            self.upload()
        lib = _lib.load()
        _lib.check(lib.ehss_scenes_build_ex(len(self.scenes), self._xyz_ptrs, self._r_ptrs, self._n, self.leaf_size,
                                            self._scenes, self._sizes, self.ws_ptr, self.ws_bytes, self.flags,
                                            stream_handle(self.device)), 'batched scene build')

    def drop_build_buffers(self):
        """Free the builder's workspace and the device coordinates once the
        scenes are built (the served form keeps only the scene buffer).  The
        memory returns to torch's stream-ordered cache, so the build queued
        on this stream still finishes before anything reuses it.  Refit and
        rebuild are unavailable afterwards."""
        self.ws = self.d_xyz = self.d_r = self.h_xyz = self.h_r = None
        self.ws_ptr = 0
        self._xyz_ptrs = self._r_ptrs = None

    def _require_build_buffers(self):
        if self.ws is None:
            raise RuntimeError('the build buffers of this batch were freed (drop_build_buffers)')

    def stage(self, structures):
        """Write new coordinates (and radii) of the same structures into the
        pinned staging buffers; returns their enclosing radii."""
        if len(structures) != len(self.scenes):
            raise ValueError('Refit requires fixed primitive identities.')
        hx, hr = self.h_xyz.numpy(), self.h_r.numpy()
        radii = []
        for (c, r), a0, n in zip(structures, self.atom0, self.n_atoms):
            c = np.ascontiguousarray(c, dtype=np.float64); r = np.ascontiguousarray(r, dtype=np.float64)
            if c.shape != (n, 3) or r.shape != (n,):
                raise ValueError('Refit requires fixed primitive identities.')
            if not np.isfinite(c).all() or not np.isfinite(r).all() or np.any(r <= 0):
                raise ValueError('Finite centers (N,3) and positive finite radii required.')
            radii.append(enclosing_radius(c, r))
        # an earlier upload from the staging buffers may still be in flight
        torch().cuda.current_stream(self.device).synchronize()
        for (c, r), a0, n in zip(structures, self.atom0, self.n_atoms):
            hx[3 * a0:3 * (a0 + n)] = np.asarray(c, dtype=np.float64).ravel()
            hr[a0:a0 + n] = r
        return radii

    def refit(self, structures):
        """New coordinates of the same structures with every tree's topology
        kept (ehss_scenes_refit, one pass over the batch): the multi-frame
        form of SphereIndex.refit (pa_spatial.py:166-170).  Full scenes only;
        block plans made before a refit keep the old impact-disk radii, so
        make them after it."""
        if self.flags & _lib.BUILD_EXTERIOR:
            raise ValueError('exterior scenes cannot be refit: their trees hold the atoms exposed in the built coordinates')
        radii = self.stage(structures)
        self.upload()
        _lib.check(_lib.load().ehss_scenes_refit(len(self.scenes), self._xyz_ptrs, self._r_ptrs, self._n,
                                                 self._scenes, self.ws_ptr, self.ws_bytes,
                                                 stream_handle(self.device)), 'batched scene refit')
        for sc, R in zip(self.scenes, radii):
            sc.radius = R

    def info(self, i):
        """Header of scene i (synchronises the stream)."""
        info = _lib.SceneInfo()
        _lib.check(_lib.load().ehss_scene_info_get(self.scene_ptrs[i], ct.byref(info), stream_handle(self.device)),
                   'scene info')
        return info


class BatchCCS:
    def __init__(self, structures, log2_rays, seeds, repeats=3, cap=64, precision='fp32', ehss=True, pa=False,
                 leaf_size=_lib.DEFAULT_LEAF, launch=None, device=None, graph=True, exterior=True, cap_ladder=None,
                 tail_fraction=5e-4, boundary=None):
        S = len(structures)
        log2s = [int(log2_rays)] * S if np.isscalar(log2_rays) else [int(x) for x in log2_rays]
        seeds = [int(x) for x in (seeds if not np.isscalar(seeds) else [seeds] * S)]
        self.batch = BatchScenes(structures, leaf_size=leaf_size, device=device, exterior=exterior)
        self.device = self.batch.device
        self.scenes = self.batch.scenes
        self.n_atoms = self.batch.n_atoms
        prec = {'fp64': _lib.PREC_FP64, 'fp32': _lib.PREC_FP32}[precision] if isinstance(precision, str) else precision
        if boundary is not None and cap_ladder:
            raise ValueError('cap extension needs impact-disk blocks; choose boundary=None or no cap_ladder')
        fits = [None] * S
        if boundary is not None:
            # incidence on an enclosing boundary of each structure (CompactBoundary.fit, on the host)
            from types import SimpleNamespace
            from .compact import CompactBoundary
            fits = [CompactBoundary.fit(SimpleNamespace(centers=np.asarray(c, dtype=np.float64),
                                                        radii=np.asarray(r, dtype=np.float64)), boundary,
                                        device=self.device) for c, r in structures]
        jobs = []
        for s, (sc, lg, sd) in enumerate(zip(self.scenes, log2s, seeds)):
            for k, seed in enumerate(seed_schedule(sd, repeats)):
                jobs.append(BlockJob(sc, lg, seed, cap=cap, precision=prec, ehss=ehss, pa=pa, tag=(s, k),
                                     boundary=fits[s]))
        self.repeats = int(repeats)
        self.ehss, self.pa = bool(ehss), bool(pa)
        self.cap_ladder = tuple(int(c) for c in cap_ladder) if cap_ladder else ()
        self.tail_fraction = float(tail_fraction)
        rays = sum(1 << j.log2_rays for j in jobs)
        self.plan = BlockPlan(jobs, launch=launch, device=self.device,
                              residual_capacity=max(4096, rays // 256) if self.cap_ladder else 0)
        self.rays = self.plan.rays
        self.use_graph = graph
        self.h2d_bytes = self.batch.h2d_bytes
        self.d2h_bytes = self.plan.d2h_bytes

    # -- stages ---------------------------------------------------------------
    def upload(self):
        self.batch.upload()

    def build(self):
        self.batch.build(upload=False)

    def trace(self):
        if self.use_graph and self.plan.graph is None:
            self.plan.capture()
        self.plan.run()

    def download(self):
        """Per-structure summaries (one device-to-host copy).  Each structure's
        ``runs`` lists its blocks' full read-outs, built on first access."""
        S, R = len(self.scenes), self.repeats
        if self.cap_ladder:
            blocks = self.plan.extend_caps(self.cap_ladder, self.tail_fraction)
            ehss = np.array([b.get('ehss_angstrom2', 0.) for b in blocks])
            tail = np.array([b.get('tail_bound_angstrom2', 0.) for b in blocks])
            pa = np.array([b.get('pa_angstrom2', 0.) for b in blocks])
            unres = np.array([b.get('unresolved_rays', 0) for b in blocks])
            runs = [blocks[s * R:(s + 1) * R] for s in range(S)]
        else:
            packed = self.plan.fetch()
            t = self.plan.totals(packed)
            ehss, tail, pa, unres = t['ehss'], t['tail'], t['pa'], t['unresolved']
            lazy = _BlockReadout(self.plan, packed)
            runs = [_Runs(lazy, s * R, (s + 1) * R) for s in range(S)]
        out = [dict(structure=s, atoms=sc.n_atoms, runs=runs[s]) for s, sc in enumerate(self.scenes)]

        def summaries(values):
            a = np.asarray(values).reshape(S, R)
            mean = a.mean(axis=1).tolist()
            sd = a.std(axis=1, ddof=1).tolist() if R > 1 else [None] * S
            return [dict(mean=m, sd=d, sem=d / math.sqrt(R) if d is not None else None, replicates=R)
                    for m, d in zip(mean, sd)]
        if self.ehss:
            tails = np.asarray(tail).reshape(S, R).mean(axis=1).tolist()
            unr = np.asarray(unres).reshape(S, R).sum(axis=1).tolist()
            for o, e, tl, u in zip(out, summaries(ehss), tails, unr):
                o.update(ehss_angstrom2=e, ehss_tail_bound_mean_angstrom2=tl, ehss_unresolved_rays_total=int(u))
        if self.pa:
            for o, p in zip(out, summaries(pa)):
                o['pa_angstrom2'] = p
        return out

    def run(self):
        """Host arrays in, per-structure results out (upload, build, trace, download)."""
        self.upload()
        self.build()
        self.trace()
        return self.download()


class _BlockReadout:
    """Block dicts of one fetched result, built once when first needed."""

    def __init__(self, plan, packed):
        self.plan, self.packed, self.blocks = plan, packed, None

    def get(self):
        if self.blocks is None:
            self.blocks = self.plan.readout(self.packed)
        return self.blocks


class _Runs(Sequence):
    """One structure's blocks (a read-only list view, materialised lazily)."""

    def __init__(self, readout, begin, end):
        self._r, self._b, self._e = readout, begin, end

    def __len__(self):
        return self._e - self._b

    def __getitem__(self, i):
        return self._r.get()[self._b:self._e][i]

    def __eq__(self, other):
        return list(self) == list(other)

    def __repr__(self):
        return repr(list(self))
