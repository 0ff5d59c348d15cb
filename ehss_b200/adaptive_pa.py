"""Adaptive finite-grid PA on the device (ccs_cli.adaptive_pa, ccs_cli.py:142-160).

For each of ``directions`` Sobol(2, seed) directions the atom disks are
projected on a ``grid_size`` x ``grid_size`` midpoint grid and the covered
pixels are counted exactly (libehss_b200: ehss_pa_grid); the PA is the mean of
count * spacing^2 over the directions, as in the reference.
"""
from __future__ import annotations

import ctypes as ct
import time

import numpy as np

from . import _lib
from .device import empty, ptr, stream_handle, torch


def grid_counts(scene, directions, grid_size, seed, with_xy=False):
    """Per-direction covered-pixel counts, pixel spacings (and projections)."""
    lib = _lib.load()
    t = torch()
    n_dirs, n = int(directions), int(grid_size)
    wb = ct.c_uint64()
    _lib.check(lib.ehss_pa_grid_workspace_bytes(scene.n_atoms, n_dirs, n, ct.byref(wb)), 'adaptive PA')
    ws = empty(int(wb.value) + 256, t.uint8, scene.device)
    counts = t.zeros(n_dirs, dtype=t.int64, device=scene.device)
    spacing = t.zeros(n_dirs, dtype=t.float64, device=scene.device)
    xy = empty((n_dirs, scene.n_atoms, 2), t.float64, scene.device) if with_xy else None
    _lib.check(lib.ehss_pa_grid(scene.ptr, scene.n_atoms, n_dirs, int(seed), n, ptr(counts), ptr(spacing), ptr(xy),
                                (ws.data_ptr() + 255) & ~255, int(wb.value), stream_handle(scene.device)),
               'adaptive PA')
    out = (counts.cpu().numpy(), spacing.cpu().numpy())
    return out + ((xy.cpu().numpy(),) if with_xy else ())


def adaptive_pa(spheres, directions, grid_size, seed, scene=None):
    from .engine import Scene
    tick = time.perf_counter()
    scene = scene or Scene(spheres.centers, spheres.radii)
    setup_s = time.perf_counter() - tick
    tick = time.perf_counter()
    counts, spacing = grid_counts(scene, directions, grid_size, seed)
    query_s = time.perf_counter() - tick
    tick = time.perf_counter()
    values = [float(c) * float(sp) ** 2 for c, sp in zip(counts, spacing)]
    value = float(np.mean(values))
    return dict(pa_angstrom2=value, source_s=0., projection_s=setup_s, query_s=query_s,
                readout_s=time.perf_counter() - tick)
