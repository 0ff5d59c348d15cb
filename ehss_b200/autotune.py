"""Launch-shape autotuner for the fused blocks kernel.

Tunes, on the caller's own workload, the persistent kernel's block shape
(threads per CTA and resident warps per SM), rays per work item (chunk_rays,
i.e. chunk_rays / 32 rays per lane), how many finished queries a warp batches
before its FP64 resolve phase, and how many traversal-stack entries per lane
live in shared memory (the rest spill to local memory).  Coordinate descent
from the defaults, each candidate timed with CUDA events (best of a few runs
after a warm-up).  Results are cached per GPU and workload signature in
$XDG_CACHE_HOME/ehss_b200/autotune.json (default ~/.cache).
"""
from __future__ import annotations

import dataclasses
import json
import os
from pathlib import Path

import numpy as np

from .blocks import DEFAULT_LAUNCH, BlockJob, BlockPlan
from .device import torch

SPACE = dict(block_threads=(64, 128), warps_per_sm=(16, 24, 32), chunk_rays=(128, 256, 512),
             resolve_batch=(24, 30, 32), smem_stack=(4, 5, 8))


def cache_path():
    root = Path(os.environ.get('XDG_CACHE_HOME', Path.home() / '.cache'))
    return root / 'ehss_b200' / 'autotune.json'


def signature(jobs):
    t = torch()
    name = t.cuda.get_device_name()
    rays = sum(1 << j.log2_rays for j in jobs)
    atoms = np.mean([j.scene.n_atoms for j in jobs])
    return f'{name}|blocks~{2 ** int(np.log2(len(jobs)))}|rays~2^{int(np.log2(rays))}|atoms~{int(2 ** round(np.log2(atoms)))}'


def to_launch(cfg):
    L = dict(DEFAULT_LAUNCH)
    L.update({k: v for k, v in cfg.items() if k in L})
    L['ctas_per_sm'] = max(1, cfg['warps_per_sm'] // (cfg['block_threads'] // 32))
    return L


def time_config(jobs, cfg, repeats=2):
    t = torch()
    plan = BlockPlan([dataclasses.replace(j) for j in jobs],
                     launch=to_launch(cfg))
    plan.enqueue()
    best = float('inf')
    for _ in range(repeats):
        a = t.cuda.Event(enable_timing=True); b = t.cuda.Event(enable_timing=True)
        a.record(); plan.enqueue(); b.record(); b.synchronize()
        best = min(best, a.elapsed_time(b))
    return best


def tune(jobs, passes=2, use_cache=True, space=None, log=None):
    """Best launch configuration (dict for BlockPlan(launch=...)) and its time in ms."""
    space = space or SPACE
    sig = signature(jobs)
    path = cache_path()
    cache = {}
    if use_cache and path.exists():
        try:
            cache = json.loads(path.read_text())
        except ValueError:
            cache = {}
        if sig in cache:
            return to_launch(cache[sig]['config']), cache[sig]['ms']
    cfg = dict(block_threads=DEFAULT_LAUNCH['block_threads'],
               warps_per_sm=DEFAULT_LAUNCH['ctas_per_sm'] * DEFAULT_LAUNCH['block_threads'] // 32,
               chunk_rays=DEFAULT_LAUNCH['chunk_rays'], resolve_batch=DEFAULT_LAUNCH['resolve_batch'],
               smem_stack=DEFAULT_LAUNCH['smem_stack'])
    best = time_config(jobs, cfg)
    for _ in range(passes):
        improved = False
        for key, values in space.items():
            for v in values:
                if v == cfg[key]:
                    continue
                trial = dict(cfg, **{key: v})
                ms = time_config(jobs, trial)
                if log:
                    log(f'autotune {trial} -> {ms:.3f} ms')
                if ms < best * 0.99:
                    best, cfg, improved = ms, trial, True
        if not improved:
            break
    if use_cache:
        cache[sig] = dict(config=cfg, ms=best)
        path.parent.mkdir(parents=True, exist_ok=True)
        path.write_text(json.dumps(cache, indent=1))
    return to_launch(cfg), best
