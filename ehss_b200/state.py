"""Sphere sets, incidence sources and results: the reference's data types.

These mirror, field for field and rule for rule, the reference classes a
caller of the EHSS path already holds, so the CUDA engine is a drop-in:

* ``Spheres``      inside_out_pa.Spheres (src/support_exchange_transport/inside_out_pa.py:17-42)
* ``EHSSSource``   ehss_state.EHSSSource (ehss_state.py:8-39)
* ``EHSSResult``   ehss_state.EHSSResult (ehss_state.py:72-108)
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass(frozen=True)
class Spheres:
    centers: np.ndarray
    radii: np.ndarray
    deduplicate: bool = True

    def __post_init__(self):
        c = np.ascontiguousarray(self.centers, dtype=np.float64)
        r = np.ascontiguousarray(self.radii, dtype=np.float64)
        if c.ndim != 2 or c.shape[1] != 3 or r.shape != (len(c),) or len(c) == 0:
            raise ValueError("Expected nonempty centers (N,3) and radii (N,).")
        if not np.isfinite(c).all() or not np.isfinite(r).all() or np.any(r <= 0):
            raise ValueError("Finite centers and positive finite radii required.")
        if self.deduplicate:
            # exact duplicates need one surface owner: keep the first occurrence
            _, keep = np.unique(np.column_stack((c, r)), axis=0, return_index=True)
            keep.sort()
        else:
            keep = np.arange(len(c))
        object.__setattr__(self, "centers", c[keep].copy())
        object.__setattr__(self, "radii", r[keep].copy())

    @property
    def area(self):
        return float(4 * np.pi * np.dot(self.radii, self.radii))


@dataclass
class EHSSSource:
    origins: np.ndarray
    directions: np.ndarray
    incoming: np.ndarray
    weights: np.ndarray
    last_atom: np.ndarray
    initial_bounces: np.ndarray
    convention: str

    def __post_init__(self):
        n = len(self.weights)
        for name in ("origins", "directions", "incoming"):
            value = np.ascontiguousarray(getattr(self, name), dtype=float)
            if value.shape != (n, 3) or not np.isfinite(value).all():
                raise ValueError("Finite (N,3) positions and directions required")
            setattr(self, name, value)
        for name in ("directions", "incoming"):
            if not np.allclose(np.linalg.norm(getattr(self, name), axis=1), 1., atol=1e-12, rtol=1e-12):
                raise ValueError("Unit physical directions required")
        self.weights = np.ascontiguousarray(self.weights, dtype=float)
        if self.weights.shape != (n,) or not np.isfinite(self.weights).all() or np.any(self.weights < 0):
            raise ValueError("Nonnegative finite source weights required")
        for name in ("last_atom", "initial_bounces"):
            value = np.ascontiguousarray(getattr(self, name), dtype=np.int64)
            if value.shape != (n,):
                raise ValueError("One initial identity and bounce count per state required")
            setattr(self, name, value)
        if np.any(self.initial_bounces < 0):
            raise ValueError("Nonnegative initial bounce count required")
        if np.any((self.initial_bounces == 1) & (self.last_atom < 0)):
            raise ValueError("First-reflected source states require their collider identity")


@dataclass
class EHSSResult:
    positions: np.ndarray
    outgoing: np.ndarray
    escaped: np.ndarray
    unresolved: np.ndarray
    bounces: np.ndarray
    collider_ids: np.ndarray
    source: EHSSSource
    metrics: dict = field(default_factory=dict)

    @property
    def contributions(self):
        # clamp only at the analytic [0, 2] bounds of 1 - cos(chi)
        angle = np.clip(1 - np.sum(self.source.incoming * self.outgoing, axis=1), 0., 2.)
        return self.source.weights * angle * self.escaped

    @property
    def omega(self):
        return float(self.contributions.sum())

    @property
    def residual_mass(self):
        return float(self.source.weights[self.unresolved].sum())

    @property
    def tail_bound(self):
        return 2 * self.residual_mass

    @property
    def pa(self):
        return float(self.source.weights[(self.bounces > 0) | self.unresolved].sum())

    def order_ledger(self):
        c = self.contributions
        top = int(self.bounces.max(initial=0))
        return [dict(order=k, count=int(np.count_nonzero(self.escaped & (self.bounces == k))),
                     mass=float(self.source.weights[self.escaped & (self.bounces == k)].sum()),
                     omega=float(c[self.bounces == k].sum())) for k in range(top + 1)]
