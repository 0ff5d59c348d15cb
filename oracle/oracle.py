"""TEST INFRASTRUCTURE — CPU oracle for the PA + EHSS cross-section path.

This module is the checker, not the product.  Only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` import
it.  It restates the SCIMMS/EHSS reference's FP64 CPU algorithm:

* scrambled Sobol points exactly as scipy's ``qmc.Sobol(d, scramble=True,
  seed=s).random_base2(m)`` produces them (the reference calls it at
  ``src/support_exchange_transport/ehss_state.py:44``): numpy's
  ``default_rng(seed)`` draws the random-shift bits and then the lower
  triangular LMS matrices, as scipy's ``Sobol._scramble`` does; the LMS
  matrix (unit diagonal) multiplies each direction number's MSB-first
  30-digit vector over GF(2); point n is ``shift ^ XOR_{k in gray(n)} v_k``
  scaled by 2**-30.  Direction numbers are the published Joe--Kuo
  (new-joe-kuo-6.21201) values;
* the impact-disk source (``ehss_state.external_source``, ehss_state.py:42-53;
  ``unit_sphere``/``tangent_frames``, inside_out_pa.py:45-58) and the
  compact-boundary sources (``CompactBoundary.source``,
  ehss_compact_source.py:47-87) in numpy, which is the same arithmetic the
  reference performs;
* the static BVH, nearest-entry trace and any-hit PA in ``ehss_oracle.c``
  (see that file for per-function citations), loaded through ctypes;
* the readout (``EHSSResult``, ehss_state.py:84-108; ``ccs_cli.solve_frame``
  readout, ccs_cli.py:209-219) and replicate statistics (``summarize``,
  ccs_cli.py:163-167).

Parity of every piece is pinned against fixtures generated from the reference
itself (``tests/golden/make_golden.py``).
"""
from __future__ import annotations

import ctypes as ct
import math
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
BITS = 30
SCALE = 2.0 ** -BITS

# Joe--Kuo direction-number parameters (degree s, coefficient a, initial m_i)
# for Sobol dimensions 2..8; dimension 1 is the van der Corput sequence.
JOE_KUO = [(1, 0, (1,)), (2, 1, (1, 3)), (3, 1, (1, 3, 1)), (3, 2, (1, 1, 1)),
           (4, 1, (1, 1, 3, 3)), (4, 4, (1, 3, 5, 13)), (5, 2, (1, 1, 5, 5, 17))]
MAXDIM = len(JOE_KUO) + 1


# --------------------------------------------------------------------------
# Sobol
# --------------------------------------------------------------------------
def direction_numbers(d):
    """Unscrambled direction numbers v[j, k] (30-bit, MSB-aligned)."""
    if not 1 <= d <= MAXDIM:
        raise ValueError(f"oracle Sobol supports 1..{MAXDIM} dimensions")
    v = np.zeros((d, BITS), dtype=np.uint64)
    for k in range(BITS):
        v[0, k] = 1 << (BITS - 1 - k)
    for j in range(1, d):
        s, a, m = JOE_KUO[j - 1]
        for k in range(BITS):
            if k < s:
                v[j, k] = m[k] << (BITS - 1 - k)
            else:
                x = int(v[j, k - s]) ^ (int(v[j, k - s]) >> s)
                for t in range(1, s):
                    if (a >> (s - 1 - t)) & 1:
                        x ^= int(v[j, k - t])
                v[j, k] = x
    return v.astype(np.uint32)


def sobol_scramble(d, seed):
    """(sv, shift): LMS-scrambled direction numbers and the random shift."""
    rng = np.random.default_rng(seed)
    bits = rng.integers(2, size=(d, BITS), dtype=np.uint32).astype(np.uint64)
    shift = (bits * (np.uint64(1) << np.arange(BITS, dtype=np.uint64))).sum(axis=1).astype(np.uint32)
    ltm = np.tril(rng.integers(2, size=(d, BITS, BITS), dtype=np.uint32)).astype(np.uint8)
    idx = np.arange(BITS)
    ltm[:, idx, idx] = 1
    v = direction_numbers(d)
    # MSB-first digit vectors: digits[j, k, i] = bit (29 - i) of v[j, k]
    digits = ((v[:, :, None] >> (BITS - 1 - idx)[None, None, :]) & 1).astype(np.uint8)
    # new digit i = XOR_{jj <= i} L[i, jj] * digit jj
    new = np.einsum('jil,jkl->jki', ltm.astype(np.int64), digits.astype(np.int64)) & 1
    weights = (np.uint64(1) << (BITS - 1 - idx).astype(np.uint64))
    sv = (new.astype(np.uint64) * weights[None, None, :]).sum(axis=2).astype(np.uint32)
    return sv, shift


def sobol_integers(d, m, seed, scramble=True):
    """uint32 Sobol integers q[n, d] for n = 2**m points (point 0 included)."""
    if scramble:
        sv, shift = sobol_scramble(d, seed)
    else:
        sv, shift = direction_numbers(d), np.zeros(d, dtype=np.uint32)
    n = 1 << m
    index = np.arange(n, dtype=np.uint64)
    gray = index ^ (index >> np.uint64(1))
    q = np.tile(shift.astype(np.uint64), (n, 1))
    for k in range(m):
        sel = ((gray >> np.uint64(k)) & np.uint64(1)).astype(bool)
        q[sel] ^= sv[:, k].astype(np.uint64)
    return q.astype(np.uint32)


def sobol_points(d, m, seed):
    return sobol_integers(d, m, seed).astype(np.float64) * SCALE


# --------------------------------------------------------------------------
# Impact-disk source
# --------------------------------------------------------------------------
def unit_sphere(uv):
    z = 1 - 2 * uv[:, 0]
    phi = 2 * np.pi * uv[:, 1]
    rho = np.sqrt(np.maximum(0, 1 - z * z))
    return np.column_stack((rho * np.cos(phi), rho * np.sin(phi), z))


def tangent_frames(normals):
    axes = np.zeros_like(normals)
    axes[:, 2] = 1
    axes[np.abs(normals[:, 2]) > .9] = [1, 0, 0]
    t = np.cross(axes, normals)
    t /= np.linalg.norm(t, axis=1)[:, None]
    return t, np.cross(normals, t)


def enclosing(centers, radii):
    center = centers.mean(axis=0)
    radius = float(np.max(np.linalg.norm(centers - center, axis=1) + radii)) * (1. + 1e-9)
    return center, radius


def map_impact_disk(u, centers, radii):
    """Rays from Sobol points u[n, 4] (ehss_state.py:45-52)."""
    directions = unit_sphere(u[:, :2])
    t, b = tangent_frames(directions)
    center, radius = enclosing(centers, radii)
    rho = radius * np.sqrt(u[:, 2])
    phi = 2 * np.pi * u[:, 3]
    origins = center - radius * directions + rho[:, None] * (np.cos(phi)[:, None] * t + np.sin(phi)[:, None] * b)
    n = len(u)
    return dict(origins=origins, directions=directions, incoming=directions.copy(),
                weights=np.full(n, np.pi * radius * radius / n),
                last_atom=np.full(n, -1, dtype=np.int64), initial_bounces=np.zeros(n, dtype=np.int64),
                center=center, radius=radius)


def external_source(centers, radii, power, seed):
    return map_impact_disk(sobol_points(4, power, seed), np.asarray(centers, float), np.asarray(radii, float))


def compact_source(kind, center, rotation, axes, u):
    """Rays of an enclosing boundary from Sobol points u[n, 4 or 5]
    (CompactBoundary.source, ehss_compact_source.py:47-87): directions
    uniform on S2, origins uniform over the boundary's projection, upstream
    of it, weight = projected area / n."""
    center, rotation, axes = (np.asarray(x, dtype=np.float64) for x in (center, rotation, axes))
    d = unit_sphere(u[:, :2])
    n = len(d)
    if kind == 'sphere':
        t, b = tangent_frames(d)
        radius = axes[0]
        rho, phi = radius * np.sqrt(u[:, 2]), 2 * np.pi * u[:, 3]
        origins = center - radius * d + rho[:, None] * (np.cos(phi)[:, None] * t + np.sin(phi)[:, None] * b)
        area = np.full(n, np.pi * radius * radius)
    elif kind == 'box':
        local_d = d @ rotation
        face_areas = 4 * np.prod(axes) / axes
        projected = np.abs(local_d) * face_areas
        area = projected.sum(axis=1)
        # face k with probability projected[k] / area (u[:, 2] against the running sums)
        face = (u[:, 2, None] * area[:, None] >= np.cumsum(projected, axis=1)).sum(axis=1)
        p = np.empty((n, 3))
        for axis in range(3):
            sel = face == axis
            p[sel, axis] = -np.sign(local_d[sel, axis]) * axes[axis]
            other = [k for k in range(3) if k != axis]
            p[np.ix_(sel, other)] = (2 * u[sel, 3:5] - 1) * axes[other]
        origins = center + p @ rotation.T - 1e-10 * max(1., axes.max()) * d
    elif kind == 'ellipsoid':
        t, b = tangent_frames(d)
        lt, lb = (t @ rotation) * axes, (b @ rotation) * axes
        g00, g01, g11 = np.sum(lt * lt, axis=1), np.sum(lt * lb, axis=1), np.sum(lb * lb, axis=1)
        l00 = np.sqrt(g00)
        l10 = g01 / l00
        l11 = np.sqrt(np.maximum(0., g11 - l10 * l10))
        rho, phi = np.sqrt(u[:, 2]), 2 * np.pi * u[:, 3]
        x, y = rho * np.cos(phi), rho * np.sin(phi)
        offset = (l00 * x)[:, None] * t + (l10 * x + l11 * y)[:, None] * b
        extent = np.linalg.norm((d @ rotation) * axes, axis=1)
        origins = center + offset - (extent * (1 + 1e-10))[:, None] * d
        area = np.pi * l00 * l11
    else:
        raise ValueError('Boundary must be sphere, ellipsoid, or box')
    return dict(origins=origins, directions=d, incoming=d.copy(), weights=area / n,
                last_atom=np.full(n, -1, dtype=np.int64), initial_bounces=np.zeros(n, dtype=np.int64))


# --------------------------------------------------------------------------
# Native oracle (ehss_oracle.c)
# --------------------------------------------------------------------------
_LIB = None
_REF = None
P = ct.c_void_p
I64 = ct.c_int64


def build(reference=None):
    """Compile liboracle.so and, when ``reference`` (or the EHSS_REFERENCE
    environment variable) names a reference checkout, the reference's own
    C++ kernel into _ref/."""
    cmd = ['make', '-s', '-C', str(HERE)]
    reference = reference or os.environ.get('EHSS_REFERENCE')
    if reference:
        cmd.append(f'REF={reference}')
    subprocess.run(cmd, check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = HERE / 'liboracle.so'
        if not path.exists():
            build()
        L = ct.CDLL(str(path))
        L.oracle_median_groups.restype = I64
        L.oracle_median_groups.argtypes = [I64, P, I64, P]
        L.oracle_box_centres.restype = None
        L.oracle_box_centres.argtypes = [I64, P, P, P]
        L.oracle_static_tree.restype = None
        L.oracle_static_tree.argtypes = [I64, P, P, P, I64] + [P] * 6
        L.oracle_trace.restype = None
        L.oracle_trace.argtypes = [I64, I64, I64, ct.c_int, ct.c_int] + [P] * 18
        L.oracle_trace_flat.restype = None
        L.oracle_trace_flat.argtypes = [I64, I64, I64] + [P] * 9
        L.oracle_entry.restype = ct.c_double
        L.oracle_entry.argtypes = [P, P, P, ct.c_double]
        L.oracle_sphere_hit.restype = ct.c_int
        L.oracle_sphere_hit.argtypes = [P, P, P, ct.c_double]
        L.oracle_pa_tree.restype = I64
        L.oracle_pa_tree.argtypes = [I64, P, P, I64] + [P] * 6
        L.oracle_union_count.restype = I64
        L.oracle_union_count.argtypes = [I64, P, P, ct.c_double, ct.c_double, ct.c_double, I64, P]
        L.oracle_pa_blocked.restype = None
        L.oracle_pa_blocked.argtypes = [I64, P, P, P, P, P, I64] + [P] * 6 + [P, P, ct.c_int]
        _LIB = L
    return _LIB


def _p(a):
    return ct.c_void_p(a.ctypes.data) if a is not None else None


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


class StaticTree:
    """PreparedStaticCPUEHSS tree arrays (ehss_static.py:62-91)."""

    def __init__(self, centers, radii, leaf_size=4):
        if type(leaf_size) is not int or leaf_size < 1:
            raise ValueError('Positive integer leaf size required')
        self.centers = _c(centers, np.float64).copy()
        self.radii = _c(radii, np.float64).copy()
        n = len(self.radii)
        L = lib()
        box_c = np.empty((n, 3))
        L.oracle_box_centres(n, _p(self.centers), _p(self.radii), _p(box_c))
        self.groups = np.empty(n, dtype=np.int64)
        ng = L.oracle_median_groups(n, _p(box_c), leaf_size, _p(self.groups))
        nodes = 2 * ng - 1
        self.lo = np.empty((nodes, 3)); self.hi = np.empty((nodes, 3))
        self.end = np.empty(nodes, dtype=np.int64); self.leaf_group = np.empty(nodes, dtype=np.int64)
        self.offsets = np.empty(ng + 1, dtype=np.int64); self.ids = np.empty(n, dtype=np.int64)
        L.oracle_static_tree(n, _p(self.centers), _p(self.radii), _p(self.groups), ng, _p(self.lo), _p(self.hi),
                             _p(self.end), _p(self.leaf_group), _p(self.offsets), _p(self.ids))

    def trace(self, origins, directions, last_atom=None, initial_bounces=None, cap=64, record=False,
              threads=1, per_ray_counts=False):
        """CPUEHSSTransport.trace semantics (ehss_cpu.py:118-142)."""
        if type(cap) is not int or cap < 1:
            raise ValueError('Positive cap required')
        n = len(origins)
        p = _c(origins, np.float64).copy(); d = _c(directions, np.float64).copy()
        lasts = _c(np.full(n, -1) if last_atom is None else last_atom, np.int64)
        counts = _c(np.zeros(n) if initial_bounces is None else initial_bounces, np.int64).copy()
        if np.any(counts > 1) or np.any(lasts < -1) or np.any(lasts >= len(self.radii)):
            raise ValueError('Invalid initial state')
        escaped = np.zeros(n, dtype=np.uint8); unresolved = np.zeros(n, dtype=np.uint8)
        history = np.full((n, cap if record else 0), -1, dtype=np.int32)
        counters = np.zeros(2, dtype=np.int64)
        nb = np.zeros(n, dtype=np.int64) if per_ray_counts else None
        ns = np.zeros(n, dtype=np.int64) if per_ray_counts else None
        lib().oracle_trace(n, len(self.end), cap, int(bool(record)), int(threads), _p(p), _p(d), _p(lasts),
                           _p(counts), _p(escaped), _p(unresolved), _p(history) if record else None,
                           _p(self.lo), _p(self.hi), _p(self.end), _p(self.leaf_group), _p(self.offsets),
                           _p(self.ids), _p(self.centers), _p(self.radii), _p(counters), _p(nb), _p(ns))
        out = dict(positions=p, outgoing=d, escaped=escaped.astype(bool), unresolved=unresolved.astype(bool),
                   bounces=counts, collider_ids=history, box_tests=int(counters[0]), sphere_tests=int(counters[1]))
        if per_ray_counts:
            out['ray_box_tests'] = nb; out['ray_sphere_tests'] = ns
        return out


def trace_flat(centers, radii, origins, directions, last_atom=None, initial_bounces=None, cap=64):
    """Independent all-atom search (ehss_reference.trace_all, ehss_reference.py:40-64)."""
    centers = _c(centers, np.float64); radii = _c(radii, np.float64)
    n = len(origins)
    p = _c(origins, np.float64).copy(); d = _c(directions, np.float64).copy()
    lasts = _c(np.full(n, -1) if last_atom is None else last_atom, np.int64)
    counts = _c(np.zeros(n) if initial_bounces is None else initial_bounces, np.int64).copy()
    escaped = np.zeros(n, dtype=np.uint8); unresolved = np.zeros(n, dtype=np.uint8)
    ledger = np.full((n, cap), -1, dtype=np.int32)
    lib().oracle_trace_flat(n, len(radii), cap, _p(p), _p(d), _p(lasts), _p(counts), _p(escaped),
                            _p(unresolved), _p(ledger), _p(centers), _p(radii))
    return dict(positions=p, outgoing=d, escaped=escaped.astype(bool), unresolved=unresolved.astype(bool),
                bounces=counts, collider_ids=ledger)


def entry_distance(o, d, c, r):
    o, d, c = (_c(x, np.float64) for x in (o, d, c))   # keep the buffers alive across the call
    return lib().oracle_entry(_p(o), _p(d), _p(c), float(r))


def sphere_hit(o, d, c, r):
    o, d, c = (_c(x, np.float64) for x in (o, d, c))
    return bool(lib().oracle_sphere_hit(_p(o), _p(d), _p(c), float(r)))


class PATree:
    """SphereIndex BVH (pa_spatial.py:38-75, 157-164)."""

    def __init__(self, centers, radii, leaf_size=4):
        self.centers = _c(centers, np.float64).copy(); self.radii = _c(radii, np.float64).copy()
        n = len(self.radii)
        plo = self.centers - self.radii[:, None]; phi = self.centers + self.radii[:, None]
        cap_nodes = 2 * n
        lo = np.empty((cap_nodes, 3)); hi = np.empty((cap_nodes, 3))
        end = np.empty(cap_nodes, dtype=np.int64); first = np.empty(cap_nodes, dtype=np.int64)
        count = np.empty(cap_nodes, dtype=np.int64); ids = np.empty(n, dtype=np.int64)
        nodes = lib().oracle_pa_tree(n, _p(plo), _p(phi), leaf_size, _p(lo), _p(hi), _p(end), _p(first),
                                     _p(count), _p(ids))
        self.lo, self.hi, self.end = lo[:nodes].copy(), hi[:nodes].copy(), end[:nodes].copy()
        self.first, self.count, self.ids = first[:nodes].copy(), count[:nodes].copy(), ids

    def query(self, origins, directions, owners=None, threads=1):
        n = len(origins)
        o = _c(origins, np.float64); d = _c(directions, np.float64)
        own = _c(np.full(n, -1) if owners is None else owners, np.int64)
        blocked = np.zeros(n, dtype=np.uint8); counters = np.zeros(2, dtype=np.int64)
        lib().oracle_pa_blocked(n, _p(o), _p(d), _p(own), _p(self.centers), _p(self.radii), len(self.end),
                                _p(self.lo), _p(self.hi), _p(self.end), _p(self.first), _p(self.count),
                                _p(self.ids), _p(blocked), _p(counters), int(threads))
        return blocked.astype(bool), int(counters[0]), int(counters[1])


# --------------------------------------------------------------------------
# The reference's own C++ kernel (oracle/_ref), driven with oracle tree arrays
# --------------------------------------------------------------------------
def ref_available():
    return (HERE / '_ref' / 'libehss_ref.so').exists()


def ref_lib():
    global _REF
    if _REF is None:
        L = ct.CDLL(str(HERE / '_ref' / 'libehss_ref.so'))
        L.ehss_trace.restype = None
        L.ehss_trace.argtypes = [I64, I64, ct.c_int, ct.c_int, ct.c_int] + [P] * 17
        _REF = L
    return _REF


def ref_trace(tree, origins, directions, cap=64, threads=1, record=False):
    """Drive src/native/ehss_cpu.cpp:42-82 as ehss_cpu_cpp.py:18-38 does."""
    n = len(origins)
    p = _c(origins, np.float64).copy(); d = _c(directions, np.float64).copy()
    lasts = np.full(n, -1, dtype=np.int64); counts = np.zeros(n, dtype=np.int64)
    escaped = np.zeros(n, dtype=np.uint8); unresolved = np.zeros(n, dtype=np.uint8)
    history = np.full((n, cap if record else 0), -1, dtype=np.int32)
    counters = np.zeros(2, dtype=np.int64); observed = np.zeros(1, dtype=np.int32)
    arrays = [p, d, lasts, counts, escaped, unresolved, history, tree.lo, tree.hi, tree.end, tree.leaf_group,
              tree.offsets, tree.ids, tree.centers, tree.radii, counters, observed]
    ref_lib().ehss_trace(n, len(tree.end), cap, int(threads), int(bool(record)), *(_p(a) for a in arrays))
    return dict(positions=p, outgoing=d, escaped=escaped.astype(bool), unresolved=unresolved.astype(bool),
                bounces=counts, collider_ids=history, box_tests=int(counters[0]), sphere_tests=int(counters[1]),
                observed_threads=int(observed[0]))


# --------------------------------------------------------------------------
# Readout and statistics
# --------------------------------------------------------------------------
def contributions(incoming, outgoing, weights, escaped):
    angle = np.clip(1 - np.sum(incoming * outgoing, axis=1), 0., 2.)
    return weights * angle * escaped


def readout(source, result, cap):
    """The per-replicate EHSS readout of ccs_cli.solve_frame (ccs_cli.py:209-219)."""
    c = contributions(source['incoming'], result['outgoing'], source['weights'], result['escaped'])
    w = source['weights']
    omega = float(c.sum())
    tail = 2 * float(w[result['unresolved']].sum())
    pa = float(w[(result['bounces'] > 0) | result['unresolved']].sum())
    counts = np.bincount(result['bounces'], minlength=cap + 1)
    ledger = np.bincount(result['bounces'], weights=c, minlength=cap + 1)
    return dict(ehss_angstrom2=omega, pa_from_same_rays_angstrom2=pa, tail_bound_angstrom2=tail,
                unresolved_rays=int(result['unresolved'].sum()), collision_histogram=counts.tolist(),
                collision_contribution_angstrom2=ledger.tolist())


def summarize(values):
    a = np.asarray(values, dtype=float)
    sd = float(a.std(ddof=1)) if len(a) > 1 else None
    return dict(mean=float(a.mean()), sd=sd, sem=sd / math.sqrt(len(a)) if sd is not None else None,
                replicates=len(a))


def host_cores():
    return len(os.sched_getaffinity(0)) if hasattr(os, 'sched_getaffinity') else (os.cpu_count() or 1)


# --------------------------------------------------------------------------
# Adaptive finite-grid PA (ccs_cli.adaptive_pa, ccs_cli.py:142-160;
# project_grid, pa_walsh_geometry.py:171-180)
# --------------------------------------------------------------------------
def pa_directions(n_dirs, seed):
    return unit_sphere(sobol_points(2, int(n_dirs).bit_length() - 1, seed))


def project_grid(centers, radii, direction, n):
    direction = np.asarray(direction, float)
    direction = direction / np.linalg.norm(direction)
    axis = np.array([0., 0., 1.]) if abs(direction[2]) < .9 else np.array([1., 0., 0.])
    u = np.cross(axis, direction); u /= np.linalg.norm(u); v = np.cross(direction, u)
    centered = centers - centers.mean(axis=0)
    xy = np.column_stack((centered @ u, centered @ v))
    extent = float(np.max(np.abs(xy) + radii[:, None])) * (1. + 1e-10)
    lower = np.array([-extent, -extent]); spacing = 2 * extent / n
    return xy, lower, spacing


def union_count(xy, radii, lower, spacing, n):
    xy = _c(xy, np.float64); radii = _c(radii, np.float64)
    bits = np.zeros(int(n) * ((int(n) + 63) // 64), dtype=np.uint64)
    return int(lib().oracle_union_count(len(radii), _p(xy), _p(radii), float(lower[0]), float(lower[1]),
                                        float(spacing), int(n), _p(bits)))


def adaptive_pa(centers, radii, n_dirs, grid, seed):
    centers = _c(centers, np.float64); radii = _c(radii, np.float64)
    counts, spacings, values = [], [], []
    for d in pa_directions(n_dirs, seed):
        xy, lower, spacing = project_grid(centers, radii, d, grid)
        c = union_count(xy, radii, lower, spacing, grid)
        counts.append(c); spacings.append(spacing)
        values.append(float(c) * spacing ** 2)
    return dict(pa_angstrom2=float(np.mean(values)), counts=counts, spacings=spacings, values=values)
