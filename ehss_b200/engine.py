"""The reference's EHSS / PA plugin objects, backed by the CUDA library.

Drop-in counterparts of (paths relative to the reference project root):

* ``PreparedStaticGPUEHSS``  PreparedStaticCPUEHSS  src/support_exchange_transport/ehss_static.py:62-101
* ``GPUEHSSTransport.trace`` CPUEHSSTransport.trace ehss_cpu.py:118-142
* ``external_source``        ehss_state.external_source ehss_state.py:42-53
* ``SphereIndex.query``      pa_spatial.SphereIndex.query pa_spatial.py:157-164

Arguments, validation and error types follow the reference (ValueError for
bad caps, identities, groups).  Geometry lives on the device in a ``Scene``;
the host arrays of a source/result are numpy, as in the reference.
"""
from __future__ import annotations

import ctypes as ct
import time
from types import SimpleNamespace

import numpy as np

from . import _lib
from .device import empty, ptr, require_cuda, stream_handle, to_device, torch
from .state import EHSSResult, EHSSSource, Spheres

PRECISIONS = {'fp64': _lib.PREC_FP64, 'fp32': _lib.PREC_FP32}


def _precision(p):
    if isinstance(p, str):
        if p not in PRECISIONS:
            raise ValueError(f'precision must be one of {sorted(PRECISIONS)}')
        return PRECISIONS[p]
    if p not in (0, 1):
        raise ValueError('precision must be 0 (fp64) or 1 (fp32)')
    return int(p)


def _aligned_buffer(nbytes, device):
    """uint8 device buffer with a 256-byte aligned start; returns (tensor, address)."""
    buf = empty(int(nbytes) + 256, torch().uint8, device)
    addr = (buf.data_ptr() + 255) & ~255
    return buf, addr


class Scene:
    """One structure resident on the device: atoms plus the LBVH.

    Owns its coordinates (a device copy), so later changes to the caller's
    arrays cannot invalidate it, like the reference's prepared scene
    (ehss_static.py:68-69).
    """

    def __init__(self, centers, radii, leaf_size=_lib.DEFAULT_LEAF, device=None, exterior=False):
        lib = _lib.load()
        self.device = require_cuda(device)
        c = np.ascontiguousarray(centers, dtype=np.float64)
        r = np.ascontiguousarray(radii, dtype=np.float64)
        if c.ndim != 2 or c.shape[1] != 3 or r.shape != (len(c),) or len(c) == 0:
            raise ValueError('Expected nonempty centers (N,3) and radii (N,).')
        self.n_atoms = len(r)
        self._radii = r.copy()
        self.leaf_size = int(leaf_size)
        sb, wb = ct.c_uint64(), ct.c_uint64()
        _lib.check(lib.ehss_scene_bytes(self.n_atoms, self.leaf_size, ct.byref(sb), ct.byref(wb)), 'scene size')
        stream = stream_handle(self.device)
        self._buf, self.ptr = _aligned_buffer(sb.value, self.device)
        self.nbytes = sb.value
        xyz_d = to_device(c, np.float64, self.device)
        r_d = to_device(r, np.float64, self.device)
        ws, ws_addr = _aligned_buffer(wb.value, self.device)
        if exterior:
            # buried atoms left out of the tree: valid for the fused block trace only
            _lib.check(lib.ehss_scenes_build_ex(1, (ct.c_void_p * 1)(xyz_d.data_ptr()),
                                                (ct.c_void_p * 1)(r_d.data_ptr()), (ct.c_int64 * 1)(self.n_atoms),
                                                self.leaf_size, (ct.c_void_p * 1)(self.ptr), (ct.c_uint64 * 1)(sb.value),
                                                ws_addr, wb.value, _lib.BUILD_EXTERIOR, stream), 'scene build')
        else:
            _lib.check(lib.ehss_scene_build(self.n_atoms, xyz_d.data_ptr(), r_d.data_ptr(), self.leaf_size, self.ptr,
                                            sb.value, ws_addr, wb.value, stream), 'scene build')
        self._read_info('scene build')   # synchronises
        del ws, xyz_d, r_d

    def _read_info(self, what):
        info = _lib.SceneInfo()
        _lib.check(_lib.load().ehss_scene_info_get(self.ptr, ct.byref(info), stream_handle(self.device)), what)
        self.info = info
        self.exterior = bool(info.exterior)
        self.n_active = int(info.n_active)
        self.center = np.array(info.center[:])
        self.radius = float(info.radius)

    def refit(self, centers, radii=None):
        """New coordinates (and optionally radii) for the same atoms, tree
        topology kept (ehss_scenes_refit; SphereIndex.refit, pa_spatial.py:166-170).
        The header and atom records become those of a build of the new
        coordinates and every node box the union of its atoms' boxes, so
        traces return what a rebuilt scene returns.  Full scenes only."""
        if self.exterior:
            raise ValueError('an exterior scene cannot be refit: its tree holds the atoms exposed in the built coordinates')
        c = np.ascontiguousarray(centers, dtype=np.float64)
        r = self._radii if radii is None else np.ascontiguousarray(radii, dtype=np.float64)
        if c.shape != (self.n_atoms, 3) or r.shape != (self.n_atoms,):
            raise ValueError('Refit requires fixed primitive identities.')
        if not np.isfinite(c).all() or not np.isfinite(r).all() or np.any(r <= 0):
            raise ValueError('Finite centers (N,3) and positive finite radii required.')
        lib = _lib.load()
        sb, wb = ct.c_uint64(), ct.c_uint64()
        _lib.check(lib.ehss_scene_bytes(self.n_atoms, self.leaf_size, ct.byref(sb), ct.byref(wb)), 'scene size')
        xyz_d = to_device(c, np.float64, self.device)
        r_d = to_device(r, np.float64, self.device)
        ws, ws_addr = _aligned_buffer(wb.value, self.device)
        _lib.check(lib.ehss_scenes_refit(1, (ct.c_void_p * 1)(xyz_d.data_ptr()), (ct.c_void_p * 1)(r_d.data_ptr()),
                                         (ct.c_int64 * 1)(self.n_atoms), (ct.c_void_p * 1)(self.ptr), ws_addr,
                                         wb.value, stream_handle(self.device)), 'scene refit')
        self._read_info('scene refit')   # synchronises
        del ws, xyz_d, r_d
        self._radii = r.copy()
        return self

    @classmethod
    def from_spheres(cls, spheres, leaf_size=_lib.DEFAULT_LEAF, device=None):
        return cls(spheres.centers, spheres.radii, leaf_size, device)

    def source_rays(self, power, seed, first=0, n=None):
        """Device impact-disk rays (origins, directions) as torch tensors."""
        lib = _lib.load()
        total = 1 << int(power)
        n = total - first if n is None else int(n)
        o = empty((n, 3), torch().float64, self.device)
        d = empty((n, 3), torch().float64, self.device)
        _lib.check(lib.ehss_source_rays(self.ptr, int(power), int(seed), int(first), n, ptr(o), ptr(d),
                                        stream_handle(self.device)), 'source')
        return o, d


def _check_seed(seed):
    if isinstance(seed, (bool, np.bool_)) or not isinstance(seed, (int, np.integer)) or not 0 <= int(seed) < 2 ** 64:
        raise ValueError('seed must be an integer in 0..2**64-1')
    return int(seed)


def external_source(spheres, power, seed, scene=None):
    """Impact-disk source generated on the device from bit-exact Sobol points.

    Same contract as the reference's external_source: 2**power rays, weight
    pi R^2 / n each, no initial collider.  The ray arrays are numpy arrays
    over page-locked host memory, so handing them back to a trace copies them
    to the device by DMA.
    """
    power = int(power)
    if not 0 <= power <= 30:
        raise ValueError('power must be 0..30')
    seed = _check_seed(seed)
    scene = scene or Scene.from_spheres(spheres)
    o, d = scene.source_rays(power, seed)
    t = torch()
    # page-locked host arrays: the copy back and a later trace's copy in run as DMA
    host = t.empty((3, o.shape[0], 3), dtype=t.float64, pin_memory=True)
    host[0].copy_(o, non_blocking=True)
    host[1].copy_(d, non_blocking=True)
    host[2].copy_(d, non_blocking=True)
    t.cuda.current_stream(scene.device).synchronize()
    origins, directions, incoming = (a.numpy() for a in host)
    n = len(origins)
    R = scene.radius
    return EHSSSource(origins, directions, incoming, np.full(n, np.pi * R * R / n),
                      np.full(n, -1), np.zeros(n, dtype=np.int64), "external impact disk")


class GPUEHSSTransport:
    """EHSS tracer on one prepared scene (CPUEHSSTransport.trace contract).

    ``trace`` takes and returns host arrays, as the reference does.  The rays
    go through in up to four chunks on two streams, so one chunk's copy to
    the device overlaps the previous chunk's trace and copy back; results are
    copied into page-locked host buffers that become the returned arrays (no
    second copy).  Device buffers are kept and grown across calls.
    """

    PIPELINE_MIN_CHUNK = 1 << 15

    def __init__(self, scene, precision='fp32', threads=1):
        if getattr(scene, 'exterior', False):
            raise ValueError('an exterior scene holds only atoms reachable from outside; trace needs a full scene')
        self.scene = scene
        self.precision = _precision(precision)
        self.threads = threads
        self._dev = None
        self._dev_rays = 0
        self._streams = None

    def _buffers(self, n, cap, record_history):
        t = torch()
        dev = self.scene.device
        if self._dev is None or self._dev_rays < n:
            self._dev = dict(P=t.empty((n, 3), dtype=t.float64, device=dev), D=t.empty((n, 3), dtype=t.float64, device=dev),
                             last=t.empty(n, dtype=t.int64, device=dev), bounces=t.empty(n, dtype=t.int64, device=dev),
                             esc=t.empty(n, dtype=t.uint8, device=dev), unres=t.empty(n, dtype=t.uint8, device=dev))
            self._dev_rays = n
        if self._streams is None:
            self._streams = [t.cuda.Stream(dev), t.cuda.Stream(dev)]
        hist = t.empty((n, cap), dtype=t.int32, device=dev) if record_history else None
        return self._dev, hist

    def trace(self, source, cap=64, record_history=False):
        if type(cap) is not int or cap < 1 or cap > np.iinfo(np.int32).max or np.any(source.initial_bounces > 1):
            raise ValueError('Positive cap and zero/one initial collision required')
        n_atoms = self.scene.n_atoms
        if np.any(source.last_atom < -1) or np.any(source.last_atom >= n_atoms):
            raise ValueError('Invalid initial physical identity')
        lib = _lib.load()
        t = torch()
        start = time.perf_counter()
        n = len(source.weights)
        # host inputs as tensors over the caller's memory (no copy when already contiguous of the right type)
        host_in = dict(P=t.from_numpy(np.ascontiguousarray(source.origins, dtype=np.float64)),
                       D=t.from_numpy(np.ascontiguousarray(source.directions, dtype=np.float64)),
                       last=t.from_numpy(np.ascontiguousarray(source.last_atom, dtype=np.int64)),
                       bounces=t.from_numpy(np.ascontiguousarray(source.initial_bounces, dtype=np.int64)))
        d, hist = self._buffers(max(n, 1), cap, record_history)
        # results land in page-locked buffers that become the returned arrays
        pin = dict(pin_memory=True)
        out = dict(P=t.empty((n, 3), dtype=t.float64, **pin), D=t.empty((n, 3), dtype=t.float64, **pin),
                   bounces=t.empty(n, dtype=t.int64, **pin), esc=t.empty(n, dtype=t.uint8, **pin),
                   unres=t.empty(n, dtype=t.uint8, **pin))
        hist_out = t.empty((n, cap), dtype=t.int32, **pin) if record_history else None
        stats = t.zeros(_lib.NSTATS, dtype=t.int64, device=self.scene.device)
        main = t.cuda.current_stream(self.scene.device)
        parts = max(1, min(4, n // self.PIPELINE_MIN_CHUNK))
        bounds = [n * k // parts for k in range(parts + 1)]
        for s in self._streams:
            s.wait_stream(main)           # stats zeroed, buffers free
        for k in range(parts):
            a, b = bounds[k], bounds[k + 1]
            if a == b:
                continue
            s = self._streams[k % 2]
            with t.cuda.stream(s):
                for key in ('P', 'D', 'last', 'bounces'):
                    d[key][a:b].copy_(host_in[key][a:b], non_blocking=True)
                if hist is not None:
                    hist[a:b].fill_(-1)
                _lib.check(lib.ehss_trace(self.scene.ptr, b - a, cap, self.precision, ptr(d['P'][a:b]),
                                          ptr(d['D'][a:b]), ptr(d['last'][a:b]), ptr(d['bounces'][a:b]),
                                          ptr(d['esc'][a:b]), ptr(d['unres'][a:b]),
                                          None if hist is None else ptr(hist[a:b]), ptr(stats), s.cuda_stream),
                           'trace')
                for key in ('P', 'D', 'bounces', 'esc', 'unres'):
                    out[key][a:b].copy_(d[key][a:b], non_blocking=True)
                if hist is not None:
                    hist_out[a:b].copy_(hist[a:b], non_blocking=True)
        for s in self._streams:
            main.wait_stream(s)
        st = stats.cpu().numpy().astype(np.uint64)       # synchronises the main stream, hence both others
        if st[_lib.STAT_ERRORS]:
            raise _lib.EHSSDeviceError(f'{int(st[_lib.STAT_ERRORS])} rays reported a bounded device failure')
        history = hist_out.numpy() if record_history else np.full((n, 0), -1, dtype=np.int32)
        return EHSSResult(out['P'].numpy(), out['D'].numpy(), out['esc'].numpy().view(np.bool_),
                          out['unres'].numpy().view(np.bool_), out['bounces'].numpy(), history, source,
                          dict(query_s=time.perf_counter() - start, sphere_tests=int(st[_lib.STAT_SPHERE]),
                               box_tests=int(st[_lib.STAT_BOX]), queries=int(st[_lib.STAT_QUERIES]),
                               grazing_queries=int(st[_lib.STAT_GRAZING]),
                               fp64_fallback_queries=int(st[_lib.STAT_FALLBACK]),
                               fp64_sphere_tests=int(st[_lib.STAT_FP64]), backend='B200 CUDA',
                               precision='fp64' if self.precision == _lib.PREC_FP64 else 'fp32',
                               threads=self.threads, history_recorded=bool(record_history),
                               response_reuse=False))


def _check_groups(groups, n):
    g = np.asarray(groups)
    if g.shape != (n,) or not np.issubdtype(g.dtype, np.integer):
        raise ValueError('One integer group per atom required')
    unique = np.unique(g)
    if not np.array_equal(unique, np.arange(len(unique))):
        raise ValueError('Contiguous nonempty groups required')


class PreparedStaticGPUEHSS:
    """Owned geometry for repeated sampling of one unchanged structure.

    ``groups`` and ``threads`` are accepted and validated as in the
    reference; neither affects results (the device LBVH replaces the
    reference's median-split groups, and the GPU replaces worker threads).
    """

    def __init__(self, spheres, groups=None, leaf_size=None, threads=1, boundary='sphere', simplify=False,
                 coverage_depth=4, precision='fp32', device=None):
        # leaf_size bounds the device LBVH leaves (capped at 16); left out, the fast default is used
        if type(threads) is not int or threads < 1:
            raise ValueError('Threads must be a positive integer')
        leaf_size = _lib.DEFAULT_LEAF if leaf_size is None else leaf_size
        if type(leaf_size) is not int or leaf_size < 1:
            raise ValueError('Positive integer leaf size required')
        start = time.perf_counter()
        s = Spheres(spheres.centers, spheres.radii, deduplicate=False)
        if groups is not None:
            _check_groups(groups, len(s.radii))
        scene = Scene.from_spheres(s, leaf_size=min(leaf_size, 16), device=device)
        self.model = SimpleNamespace(spheres=s, scene=scene)
        self.scene = scene
        tick = time.perf_counter()
        from .compact import CompactBoundary
        # incidence boundary, as the reference's prepared engine carries it (ehss_static.py:94)
        self.boundary = CompactBoundary.fit(s, boundary, device=scene.device)
        boundary_s = time.perf_counter() - tick
        self.engine = GPUEHSSTransport(scene, precision=precision, threads=threads)
        self.setup = dict(total_s=time.perf_counter() - start, preparation='static device LBVH',
                          nodes=int(scene.info.n_nodes), depth=int(scene.info.depth), threads=threads,
                          boundary_s=boundary_s)


class SphereIndex:
    """Any-hit PA index (SphereIndex(spheres, kind, leaf_size).query)."""

    def __init__(self, spheres, kind='bvh', leaf_size=None, device=None):
        leaf_size = _lib.DEFAULT_LEAF if leaf_size is None else leaf_size
        if kind not in ('bvh', 'octree') or leaf_size < 1:
            raise ValueError('Valid kind, positive leaf size and nonempty primitives required.')
        self.spheres = spheres
        self.scene = Scene.from_spheres(spheres, leaf_size=min(int(leaf_size), 16), device=device)

    def refit(self, spheres):
        """Same atoms at new positions (SphereIndex.refit, pa_spatial.py:166-170):
        the device tree is refit in place (ehss_scenes_refit)."""
        if len(spheres.radii) != len(self.spheres.radii):
            raise ValueError('Refit requires fixed primitive identities.')
        self.scene.refit(spheres.centers, spheres.radii)
        self.spheres = spheres

    def query(self, source):
        owners = getattr(source, 'owners', None)
        if owners is None:
            owners = source.last_atom
        lib = _lib.load()
        t = torch()
        dev = self.scene.device
        n = len(source.origins)
        P = to_device(source.origins, np.float64, dev)
        D = to_device(source.directions, np.float64, dev)
        own = to_device(owners, np.int64, dev)
        blocked = t.zeros(n, dtype=t.uint8, device=dev)
        stats = t.zeros(_lib.NSTATS, dtype=t.int64, device=dev)
        _lib.check(lib.ehss_pa_anyhit(self.scene.ptr, n, ptr(P), ptr(D), ptr(own), ptr(blocked), ptr(stats),
                                      stream_handle(dev)), 'PA query')
        st = stats.cpu().numpy()
        if st[_lib.STAT_ERRORS]:
            raise _lib.EHSSDeviceError('PA query reported a bounded device failure')
        return blocked.cpu().numpy().astype(bool), int(st[_lib.STAT_BOX]), int(st[_lib.STAT_SPHERE])
