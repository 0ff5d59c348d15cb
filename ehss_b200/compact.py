"""Isotropic incidence on compact enclosing boundaries (sphere, ellipsoid, box).

Drop-in counterpart of ``CompactBoundary`` (src/support_exchange_transport/
ehss_compact_source.py:16-87), which the reference's prepared engines carry
as ``.boundary`` (ehss_static.py:94).  Directions are uniform on S2; for each
direction the origin is uniform over the boundary's projection onto the plane
perpendicular to it, upstream of the boundary, and the ray's weight is that
projected area divided by the ray count.  The sphere boundary is the impact
disk of ``external_source``; the box boundary (5-D Sobol) and the ellipsoid
give smaller projected areas, hence less variance per ray.

``fit`` runs once per structure on the host in FP64 with the reference's
operations (numpy for the centroid, covariance and eigen-decomposition; the
enclosing scale of the ellipsoid by the same bisection as the reference's
``ball_metric_bounds``, pa_ellipsoidal.py:15-66).  ``source`` generates the
rays on the device (ehss_compact_source_rays) from bit-exact scrambled Sobol
points.
"""
from __future__ import annotations

import ctypes as ct
import time
from dataclasses import dataclass

import numpy as np

from . import _lib
from .device import empty, ptr, require_cuda, stream_handle, torch
from .state import EHSSSource

KINDS = {'sphere': 0, 'ellipsoid': 1, 'box': 2}


def _dot3(a, b):
    return (a[..., 0] * b[..., 0] + a[..., 1] * b[..., 1]) + a[..., 2] * b[..., 2]


def ball_metric_high(points, radii, axes):
    """Upper bound of sqrt(sum((p + u)^2 / a^2)) over ||u|| <= r for every ball
    (the ``high`` output of ball_metric_bounds, pa_ellipsoidal.py:25-49),
    vectorised over balls with the same per-ball FP64 operations: the dual
    bound base + lam r^2 + sum(b^2 / (lam - D)) with lam found by 64 rounds
    of bisection that stop early exactly where the reference's loop stops."""
    points = np.asarray(points, dtype=np.float64)
    radii = np.asarray(radii, dtype=np.float64)
    dd = 1. / (axes * axes)
    dmax = np.max(dd)
    b = dd * points
    base = _dot3(points, b)
    bnorm = np.sqrt(_dot3(b, b))
    high = np.empty(len(points))
    zero = bnorm == 0.
    high[zero] = radii[zero] * np.sqrt(dmax) * (1. + 1e-12)
    idx = np.flatnonzero(~zero)
    if len(idx):
        bb, r, bs = b[idx], radii[idx], base[idx]
        left = np.full(len(idx), dmax)
        with np.errstate(divide='ignore', invalid='ignore'):
            right = np.nextafter(dmax + bnorm[idx] / r, np.inf)
            live = np.ones(len(idx), dtype=bool)
            r2 = r * r
            for _ in range(64):
                mid = left + (right - left) / 2.
                live &= ~((mid <= dmax) | (mid == left) | (mid == right))
                if not live.any():
                    break
                length2 = np.zeros(len(idx))
                for k in range(3):
                    length2 = length2 + (bb[:, k] / (mid - dd[k])) ** 2
                go_left = live & (length2 > r2)
                go_right = live & ~(length2 > r2)
                left = np.where(go_left, mid, left)
                right = np.where(go_right, mid, right)
        lam = np.maximum(right, np.nextafter(dmax, np.inf))
        upper = bs + lam * r * r
        for k in range(3):
            upper = upper + bb[:, k] * bb[:, k] / (lam - dd[k])
        high[idx] = np.sqrt(np.maximum(0., upper + 1e-12 * np.maximum(1., upper)))
    return high


@dataclass
class CompactBoundary:
    kind: str
    center: np.ndarray
    rotation: np.ndarray
    axes: np.ndarray
    prepare_s: float = 0.
    device: object = None

    @classmethod
    def fit(cls, spheres, kind='ellipsoid', device=None):
        """Boundary of ``kind`` around the spheres (CompactBoundary.fit, ehss_compact_source.py:24-45)."""
        start = time.perf_counter()
        centers = np.asarray(spheres.centers, dtype=np.float64)
        radii = np.asarray(spheres.radii, dtype=np.float64)
        center = centers.mean(axis=0)
        rotation = np.eye(3)
        if kind == 'sphere':
            radius = np.max(np.linalg.norm(centers - center, axis=1) + radii) * (1 + 1e-9)
            axes = np.full(3, radius)
        elif kind == 'ellipsoid':
            # centroid PCA with an isotropic radius floor, scaled to enclose every ball
            centered = centers - center
            covariance = centered.T @ centered / len(centered) + np.eye(3) * np.mean(radii ** 2) / 5.
            eigenvalues, rotation = np.linalg.eigh(covariance)
            axes = np.sqrt(eigenvalues)
            points = np.ascontiguousarray(centered @ rotation)
            axes = axes * (np.max(ball_metric_high(points, radii, axes)) * (1. + 1e-10))
        elif kind == 'box':
            low = np.min(centers - radii[:, None], axis=0)
            high = np.max(centers + radii[:, None], axis=0)
            center = (low + high) / 2
            axes = (high - low) / 2 * (1 + 1e-9)
        else:
            raise ValueError('Boundary must be sphere, ellipsoid, or box')
        return cls(kind, center, rotation, axes, time.perf_counter() - start, device)

    def device_rays(self, power, seed, first=0, n=None):
        """Device origins, directions [n,3] and weights [n] (float64 torch tensors)."""
        if not isinstance(power, (int, np.integer)) or power < 0:
            raise ValueError('Nonnegative integer Sobol power required')
        if power > 30:
            raise ValueError('Sobol power must be <= 30')
        if isinstance(seed, (bool, np.bool_)) or not isinstance(seed, (int, np.integer)) or not 0 <= seed < 2 ** 64:
            raise ValueError('seed must be an integer in 0..2**64-1')
        dev = require_cuda(self.device)
        lib = _lib.load()
        t = torch()
        total = 1 << int(power)
        n = total - first if n is None else int(n)
        o = empty((n, 3), t.float64, dev)
        d = empty((n, 3), t.float64, dev)
        w = empty((n,), t.float64, dev)
        b = _lib.Boundary(KINDS[self.kind], 0, (ct.c_double * 3)(*self.center),
                          (ct.c_double * 9)(*np.asarray(self.rotation, dtype=np.float64).ravel()),
                          (ct.c_double * 3)(*self.axes))
        _lib.check(lib.ehss_compact_source_rays(ct.byref(b), int(power), int(seed), int(first), n, ptr(o), ptr(d),
                                                ptr(w), stream_handle(dev)), 'compact source')
        return o, d, w

    def max_projected_area(self):
        """Largest projected area over all directions, widened by 1e-9 so that
        every ray's weight times ray count stays below it (the reference weight
        of fused boundary blocks): pi r^2 for the sphere, pi a b for the
        ellipsoid's two largest semi-axes, |(A_x, A_y, A_z)| for a box with face
        areas A_k (the maximum of sum_k |d_k| A_k over unit d)."""
        ax = np.sort(np.asarray(self.axes, dtype=np.float64))[::-1]
        if self.kind == 'sphere':
            area = np.pi * ax[0] * ax[0]
        elif self.kind == 'ellipsoid':
            area = np.pi * ax[0] * ax[1]
        else:
            faces = 4 * np.prod(self.axes) / np.asarray(self.axes, dtype=np.float64)
            area = float(np.sqrt(np.sum(faces * faces)))
        return float(area) * (1 + 1e-9)

    def fill_ray_buffer(self, power, seed, buf):
        """Write the 2**power rays into one float64 device tensor laid out as
        origins [3n], directions [3n], weights [n] (the ray buffer of a fused
        boundary block)."""
        n = 1 << int(power)
        if buf.numel() < 7 * n:
            raise ValueError('ray buffer holds fewer than 7 * 2**power values')
        lib = _lib.load()
        b = _lib.Boundary(KINDS[self.kind], 0, (ct.c_double * 3)(*self.center),
                          (ct.c_double * 9)(*np.asarray(self.rotation, dtype=np.float64).ravel()),
                          (ct.c_double * 3)(*self.axes))
        p = buf.data_ptr()
        _lib.check(lib.ehss_compact_source_rays(ct.byref(b), int(power), int(seed), 0, n, p, p + 24 * n, p + 48 * n,
                                                stream_handle(buf.device)), 'compact source')

    def source(self, power, seed):
        """EHSSSource of 2**power rays (CompactBoundary.source, ehss_compact_source.py:47-87)."""
        o, d, w = self.device_rays(power, seed)
        origins, directions = o.cpu().numpy(), d.cpu().numpy()
        n = len(origins)
        return EHSSSource(origins, directions, directions.copy(), w.cpu().numpy(), np.full(n, -1),
                          np.zeros(n, dtype=np.int64), f'isotropic projected {self.kind}')
