"""Benchmark of the batched EHSS cross-section path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload batched|plain]

Workload (default, "batched"): 256 synthetic RSA globules (0.1 atoms/A^3,
1.0 A minimum pair distance, H/C/N/O/S 0.49/0.32/0.09/0.09/0.01) with atom
counts log-uniform in 20..5000 and ray budgets 2^14..2^18 (log-uniform,
rounded to powers of two), 3 scrambled-Sobol replicate blocks each, collision
cap 64, FP32 traversal with FP64 re-test (outcomes identical to FP64).  One
step = batched LBVH build of all 256 structures + all 768 blocks traced and
reduced in one persistent launch (CUDA-graph replay).  Inputs (atoms) are
resident in HBM for `value`; `e2e` runs the public BatchCCS API from pinned
host arrays to host results.  L2 (126 MB) is flushed by a 256 MB write
between timed steps.  Metric: EHSS rays/s (whole job); structures/s, the
plain one-structure-per-launch path, p50/p99 per-structure latency of the
plain path and the CCS error against the FP64 oracle are reported beside it.

Under torchrun (N > 1) every rank runs its own batch (rank-seeded): weak
scaling with no data-path collective; the max time over ranks is used.
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "EHSS rays/s and structures/s at <=1e-5 rel CCS err; batched vs plain; p50/p99 latency"
UNIT = "rays/s"
N_STRUCT = 256
REPEATS = 3
CAP = 64
MASTER_SEED = 2026
# per-ray FP32 op counts of the reference's sphere and box tests
# (entry_scalar, ehss_cpu.py:12-24: 35 ops; box_interval, ehss_support_tree.py:20-31: 27 ops)
C_SPHERE, C_BOX = 35, 27
CLOCK_FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=20)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', choices=['ours', 'reference'], default='ours')
    ap.add_argument('--workload', choices=['batched'], default='batched')
    ap.add_argument('--structures', type=int, default=N_STRUCT)
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--no-plain', action='store_true')
    ap.add_argument('--no-serve', action='store_true')
    ap.add_argument('--no-autotune', action='store_true')
    return ap.parse_args()


def dist_env():
    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    return world, rank, local


def make_structures(count, seed):
    from ehss_b200 import workloads as W
    spec = W.mixed_batch(count, seed=seed)
    structures, log2s, seeds = [], [], []
    for n, lg, s in spec:
        c, r, _ = W.globule(n, s)
        structures.append((c, r))
        log2s.append(lg)
        seeds.append(s % (2 ** 32))
    return structures, log2s, seeds


def config(args, world):
    return {"workload": f"batched mixed-size globules: {args.structures} structures/GPU, atoms log-uniform 20..5000, "
                        f"rays 2^14..2^18 per replicate, {REPEATS} replicates, cap {CAP}",
            "structures_per_gpu": args.structures, "replicates": REPEATS, "cap": CAP,
            "precision": "fp32 traversal + fp64 re-test", "master_seed": MASTER_SEED,
            "scenes": "exterior (buried atoms left out of the trees; outcomes unchanged)",
            "l2": "flushed (256 MB write) between timed steps", "host": "gc.freeze() after set-up",
            "parallelism": "1 GPU" if world == 1 else
            f"one job of {args.structures * world} structures over {world} GPUs: LPT structure shards, "
            "NCCL all-reduce of the block integers in every step (weak: structures per GPU fixed)"}


# ----------------------------------------------------------------------------
# clocks
# ----------------------------------------------------------------------------
class ClockSampler:
    def __init__(self, index):
        self.proc = None
        try:
            self.proc = subprocess.Popen(['nvidia-smi', f'--query-gpu={CLOCK_FIELDS}', '--format=csv,noheader,nounits',
                                          '-lms', '200', '-i', str(index)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, mx, reasons = [], [], set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(',')]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1])); mx.append(float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith('active'):
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# ----------------------------------------------------------------------------
# oracle-side measurements (CPU): reference op counts, CPU baseline, CCS error
# ----------------------------------------------------------------------------
def oracle_check_blocks(plan, structures, struct_of, budget_s=120.0, stride=16):
    """The FP64 oracle on the device's own rays of every block of ``plan``
    (its structure, seed and 2^k rays): per-block relative CCS error of the
    device result, and the reference BVH's sphere and box tests on exactly
    those rays (the roofline's algorithmic work).  Blocks are visited
    every ``stride``-th first, so a run cut short by ``budget_s`` still holds
    a spread sample; the return value says how many blocks were checked."""
    import torch
    from oracle import oracle as O
    from ehss_b200 import _lib
    lib = _lib.load()
    got = plan.collect()
    n = len(plan.jobs)
    order = sorted(range(n), key=lambda i: (i % stride, i))
    trees = {}
    cores = O.host_cores()
    err = np.full(n, np.nan)
    dev = np.array([g['ehss_angstrom2'] for g in got])
    ora = np.full(n, np.nan)
    sphere = np.full(n, np.nan)
    box = np.full(n, np.nan)
    t0 = time.perf_counter()
    stream = torch.cuda.current_stream().cuda_stream
    for i in order:
        if time.perf_counter() - t0 > budget_s:
            break
        j = plan.jobs[i]
        nr = 1 << j.log2_rays
        o = torch.empty((nr, 3), dtype=torch.float64, device='cuda')
        d = torch.empty((nr, 3), dtype=torch.float64, device='cuda')
        _lib.check(lib.ehss_source_rays(j.scene.ptr, j.log2_rays, j.seed, 0, nr, o.data_ptr(), d.data_ptr(), stream))
        o, d = o.cpu().numpy(), d.cpu().numpy()
        s = struct_of(i)
        if s not in trees:
            trees[s] = O.StaticTree(*structures[s], 4)
        res = trees[s].trace(o, d, cap=j.cap, threads=cores)
        ro = O.readout(dict(incoming=d, weights=np.full(nr, np.pi * j.scene.radius ** 2 / nr)), res, j.cap)
        ora[i] = ro['ehss_angstrom2']
        err[i] = abs(dev[i] - ora[i]) / ora[i]
        sphere[i], box[i] = res['sphere_tests'], res['box_tests']
    checked = np.isfinite(err)
    return dict(checked=int(checked.sum()), blocks=n, seconds=time.perf_counter() - t0, rel_err=err,
                device=dev, oracle=ora, sphere_tests=sphere, box_tests=box, cores=cores)


def ops_from_check(check, rays_per_block):
    """Algorithmic FP32 ops of the blocks (35 per reference sphere test, 27
    per reference box test) and the reference test counts per ray; blocks the
    check did not reach are counted at the checked blocks' mean per ray."""
    ok = np.isfinite(check['sphere_tests'])
    rays = np.asarray(rays_per_block, dtype=np.float64)
    s_ray = check['sphere_tests'][ok].sum() / rays[ok].sum()
    b_ray = check['box_tests'][ok].sum() / rays[ok].sum()
    ops = np.where(ok, C_SPHERE * np.nan_to_num(check['sphere_tests']) + C_BOX * np.nan_to_num(check['box_tests']),
                   rays * (C_SPHERE * s_ray + C_BOX * b_ray))
    return float(ops.sum()), float(s_ray), float(b_ray)


def cpu_reference_rate(structures, log2, seed, budget_s=12.0, threads=None):
    """Rays/s of the reference's own C++ kernel (oracle/_ref) on a bounded sample."""
    from oracle import oracle as O
    threads = threads or O.host_cores()
    kind = 'reference' if O.ref_available() else 'port'
    prepared = []
    for c, r in structures:
        src = O.external_source(c, r, log2, seed)
        prepared.append((O.StaticTree(c, r, 4), src['origins'], src['directions']))
    rays, elapsed, passes = 0, 0.0, 0
    while elapsed < budget_s or passes == 0:
        t0 = time.perf_counter()
        for tree, o, d in prepared:
            if kind == 'reference':
                O.ref_trace(tree, o, d, cap=CAP, threads=threads)
            else:
                tree.trace(o, d, cap=CAP, threads=threads)
            rays += len(o)
        elapsed += time.perf_counter() - t0
        passes += 1
    return rays / elapsed, kind, threads, rays, elapsed


def numba_reference_rates(structures, log2, seed, budget_s=5.0):
    """The reference's production kernel, ``PreparedStaticCPUEHSS(spheres,
    threads=T).engine.trace(source, cap)`` (Numba; ehss_cpu.py:118-142), run
    from the reference package installed into baseline/_ref, on the same
    sample as the C++ baseline: T = 1 and T = every host thread.  Sources
    (the reference's external_source) and JIT compilation stay outside the
    timing, as the reference CLI times them apart."""
    ref = ROOT / 'baseline' / '_ref'
    if not (ref / 'support_exchange_transport').is_dir():
        return {"unavailable": "the reference package is not installed in baseline/_ref"}
    sys.path.insert(0, str(ref))
    try:
        import numba
        from support_exchange_transport.ehss_state import external_source
        from support_exchange_transport.ehss_static import PreparedStaticCPUEHSS
        from support_exchange_transport.inside_out_pa import Spheres
    except Exception as exc:          # noqa: BLE001 - report why the arm is missing
        return {"unavailable": f"{type(exc).__name__}: {exc}"}
    cores = int(numba.config.NUMBA_NUM_THREADS)
    work = []
    for c, r in structures:
        s = Spheres(np.asarray(c, dtype=np.float64), np.asarray(r, dtype=np.float64), deduplicate=False)
        work.append((s, external_source(s, log2, seed)))
    out = {"kind": "reference (Numba CPUEHSSTransport.trace)", "unit": UNIT,
           "sample": f"{len(structures)} structures, 2^{log2} rays each, cap {CAP}, trace only"}
    for threads in sorted({1, cores}):
        engines = [(PreparedStaticCPUEHSS(s, threads=threads).engine, src) for s, src in work]
        engines[0][0].trace(engines[0][1], CAP)            # JIT compilation
        rays, elapsed = 0, 0.0
        while elapsed < budget_s or rays == 0:
            for eng, src in engines:
                t0 = time.perf_counter()
                eng.trace(src, CAP)
                elapsed += time.perf_counter() - t0
                rays += len(src.weights)
        out[f"threads_{threads}"] = {"value": rays / elapsed, "cores": threads, "rays": rays, "seconds": elapsed}
    return out


def configuration_lines(eb, flush, peak_of, reps=10):
    """The single-structure configurations, each as one persistent launch of
    its seed blocks (exterior scene, cap 64), timed with CUDA events after an
    L2 flush, and checked against the FP64 oracle on the device's own rays:
      C1  bent triatomic (O-H 0.9572 A, 104.52 deg), 4096 rays x seeds 0-2,
          geometry rotated per seed by a seeded uniform SO(3) rotation, FP64;
      C2  650-atom globule, 65,536 rays x 20 seeds, FP64, with BVH PA;
      C3  2000-atom globule, 262,144 rays x 20 seeds, FP32 filter + FP64 re-test.
    Each line: rays/s, roofline fraction, CCS error per seed (max), grazing
    and fallback queries, bounce histogram."""
    import torch
    from oracle import oracle as O
    from ehss_b200 import _lib, workloads as W
    from ehss_b200.blocks import BlockJob, BlockPlan
    cores = O.host_cores()
    out = {}
    c0, r0, _ = W.triatomic()
    cases = {
        'C1_triatomic': [(c0 @ W.random_rotation(seed).T, r0, 12, seed, _lib.PREC_FP64, False) for seed in (0, 1, 2)],
        'C2_globule650': [(None, None, 16, seed, _lib.PREC_FP64, True) for seed in range(20)],
        'C3_globule2000': [(None, None, 18, seed, _lib.PREC_FP32, False) for seed in range(20)],
    }
    shared = {'C2_globule650': W.globule(650, 650)[:2], 'C3_globule2000': W.globule(2000, 2000)[:2]}
    stream = torch.cuda.current_stream()
    for name, blocks in cases.items():
        jobs, geo = [], []
        scenes = {}
        for k, (c, r, lg, seed, prec, pa) in enumerate(blocks):
            if c is None:
                c, r = shared[name]
            key = id(c)
            if key not in scenes:
                scenes[key] = eb.Scene(c, r, exterior=True)
            jobs.append(BlockJob(scenes[key], lg, seed, cap=CAP, precision=prec, pa=pa, tag=k))
            geo.append((c, r))
        plan = BlockPlan(jobs)
        for _ in range(3):
            plan.enqueue()
        ms = []
        for _ in range(reps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            plan.enqueue()
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        got = plan.collect()
        rays = plan.rays
        worst, sph, box, pa_equal = 0.0, 0, 0, True
        hist = np.zeros(CAP + 1, dtype=np.int64)
        trees = {}
        for j, g, (c, r) in zip(jobs, got, geo):
            o, d = (x.cpu().numpy() for x in j.scene.source_rays(j.log2_rays, j.seed))
            if id(c) not in trees:
                trees[id(c)] = (O.StaticTree(c, r, 4), O.PATree(c, r, 4) if j.pa else None)
            tree, patree = trees[id(c)]
            res = tree.trace(o, d, cap=CAP, threads=cores)
            nr = len(o)
            ro = O.readout(dict(incoming=d, weights=np.full(nr, np.pi * j.scene.radius ** 2 / nr)), res, CAP)
            worst = max(worst, abs(g['ehss_angstrom2'] - ro['ehss_angstrom2']) / ro['ehss_angstrom2'])
            sph += res['sphere_tests']; box += res['box_tests']
            hist += np.asarray(g['collision_histogram'], dtype=np.int64)
            if patree is not None:
                pa_equal &= int(patree.query(o, d, threads=cores)[0].sum()) == g['pa_blocked_rays']
        mean_ms = float(np.mean(ms))
        ops = C_SPHERE * sph + C_BOX * box
        achieved = ops / (mean_ms * 1e-3) / 1e12
        last = int(np.max(np.nonzero(hist)[0])) if hist.any() else 0
        line = {"rays": rays, "seeds": len(jobs), "atoms": int(len(geo[0][1])), "ms_per_launch": mean_ms,
                "rays_per_s": rays / (mean_ms * 1e-3),
                "precision": "fp64" if jobs[0].precision == _lib.PREC_FP64 else "fp32 filter + fp64 re-test",
                "ops_per_ray": ops / rays, "achieved_tflops": achieved, "roofline_frac": achieved / peak_of(),
                "ccs_rel_err_max_vs_fp64_oracle": worst,
                "queries": int(sum(g['queries'] for g in got)),
                "grazing_queries": int(sum(g['grazing_queries'] for g in got)),
                "fp64_fallback_queries": int(sum(g['fp64_fallback_queries'] for g in got)),
                "bounce_histogram": hist[:last + 1].tolist()}
        if any(j.pa for j in jobs):
            line["pa_blocked_rays_equal_oracle"] = bool(pa_equal)
        out[name] = line
    return out


def explicit_trace_e2e(eb, reps=5):
    """The reference-shaped drop-in call on C3's rays: host arrays in,
    ``PreparedStaticGPUEHSS(...).engine.trace(source, 64)`` with host arrays
    out (positions, directions, flags, bounce counts), FP32 filter."""
    import torch
    from ehss_b200 import workloads as W
    c, r, _ = W.globule(2000, 2000)
    s = eb.Spheres(c, r, deduplicate=False)
    prep = eb.PreparedStaticGPUEHSS(s, precision='fp32')
    src = eb.external_source(s, 18, 0, scene=prep.scene)
    for _ in range(2):
        prep.engine.trace(src, CAP)
    torch.cuda.synchronize()
    ms = []
    for _ in range(reps):
        t0 = time.perf_counter()
        res = prep.engine.trace(src, CAP)
        ms.append((time.perf_counter() - t0) * 1e3)
    n = len(src.weights)
    return {"workload": "C3 rays (2000-atom globule, 2^18 rays, seed 0) through engine.trace with host arrays "
                        "(the source as external_source returns it: numpy arrays over page-locked memory)",
            "ms_per_call": float(np.median(ms)), "rays_per_s": n / (float(np.median(ms)) * 1e-3),
            "h2d_bytes_per_call": n * (24 + 24 + 8 + 8), "d2h_bytes_per_call": n * (24 + 24 + 1 + 1 + 8),
            "timer": "host clock around the synchronous call (median of %d)" % reps,
            "escaped_rays": int(res.escaped.sum())}


def peaks():
    p = ROOT / 'MEASURED_PEAKS.json'
    try:
        return json.loads(p.read_text())
    except (OSError, ValueError):
        return {}


def measured_fp32_tflops(n=8192, reps=3):
    """FP32 CUDA-core throughput measured on this GPU: cuBLAS SGEMM with TF32
    off (2 n^3 flops), best of ``reps`` after one warm-up, CUDA events.  The
    analogue, for FP32 FMA work, of the measured-peaks file's bf16 GEMM figure."""
    import torch
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        a = torch.randn(n, n, device='cuda', dtype=torch.float32)
        b = torch.randn(n, n, device='cuda', dtype=torch.float32)
        c = a @ b
        best = float('inf')
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            torch.matmul(a, b, out=c)
            e1.record()
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1))
        del a, b, c
        return 2.0 * n ** 3 / (best * 1e-3) / 1e12
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev


def traffic_per_launch():
    p = ROOT / 'profiles' / 'k_blocks_traffic.json'
    try:
        return json.loads(p.read_text())
    except (OSError, ValueError):
        return None


# ----------------------------------------------------------------------------
# served form: Poisson arrivals, repeat blocks until rel. RMSE <= 1 %
# ----------------------------------------------------------------------------
def serving_measurement(duration_s=2.0, rate=200.0, seed=7):
    from ehss_b200 import workloads as W
    from ehss_b200.serve import CCSRequest, CCSServer, DeviceExecutor
    reqs = W.request_stream(int(duration_s * rate), rate=rate, seed=seed)
    base, base_r, _ = W.globule(1500, 4242)
    ex = DeviceExecutor()
    ex.warmup()         # every builder path's kernels loaded before traffic
    # warm-up (context, module, allocator) outside the measurement
    warm = CCSServer(ex, block_log2=15, target=0.01)
    warm.submit(CCSRequest('w', base, base_r, seed=1))
    warm.run()
    server = CCSServer(ex, block_log2=15, target=0.01)
    for i, (t, kind, v, s) in enumerate(reqs):
        if kind == 'globule':
            c, r, _ = W.globule(v, s)
        else:
            c, r = W.ensemble_frame(base, v, sigma=0.3, seed=4242), base_r
        server.submit(CCSRequest(i, c, r, seed=s % (2 ** 32), arrival=t))
    server.t0 = server.clock()
    done = server.run()
    wall = server.now()
    lat = server.latency_percentiles()
    return {"requests": len(done), "arrival_rate_per_s": rate, "p50_latency_ms": lat['p50_ms'],
            "p99_latency_ms": lat['p99_ms'], "structures_per_s": len(done) / wall, "rays_per_s": server.rays / wall,
            "rounds": server.rounds, "converged": int(sum(d['converged'] for d in done.values())),
            "block_rays": 1 << 15, "target_rel_rmse": 0.01}


# ----------------------------------------------------------------------------
# reference arm
# ----------------------------------------------------------------------------
def run_reference(args, world, rank):
    """The reference's own C++ trace kernel (oracle/_ref; the oracle port where
    it was not compiled) with every host thread, on the timed workload's own
    blocks for every 8th structure: each step builds the reference's static
    tree of each sampled structure and traces its replicate blocks at their
    2^k rays and replicate seeds (impact-disk rays made once, outside the
    timed steps, as the reference times source generation apart)."""
    if rank != 0:
        return
    from oracle import oracle as O
    from ehss_b200.blocks import seed_schedule
    structures, log2s, seeds = make_structures(args.structures, MASTER_SEED)
    pick = list(range(0, len(structures), 8))
    threads = O.host_cores()
    kind = 'reference' if O.ref_available() else 'port'
    work = []
    for s in pick:
        c, r = structures[s]
        rays = [O.external_source(c, r, log2s[s], sd) for sd in seed_schedule(seeds[s], REPEATS)]
        work.append((c, r, [(x['origins'], x['directions']) for x in rays]))
    rays_step = sum(len(o) for _, _, blocks in work for o, _ in blocks)

    def step():
        for c, r, blocks in work:
            tree = O.StaticTree(c, r, 4)
            for o, d in blocks:
                if kind == 'reference':
                    O.ref_trace(tree, o, d, cap=CAP, threads=threads)
                else:
                    tree.trace(o, d, cap=CAP, threads=threads)
    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = time.perf_counter() - t0
    value = rays_step * args.steps / dt
    sample_txt = (f"{len(pick)} of {len(structures)} structures (every 8th) with their own timed blocks: "
                  f"{REPEATS} replicates at 2^14..2^18 rays, replicate seeds, cap {CAP}; {rays_step} rays per step; "
                  f"static tree build and trace inside the step, impact-disk rays made before timing")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": dict(config(args, world), precision="fp64 (the reference's own C++ kernel)",
                           scenes="full (the reference's static tree over every atom)", sample=sample_txt),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind, "sample": sample_txt},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------
# our arm
# ----------------------------------------------------------------------------
def main():
    args = parse()
    world, rank, local = dist_env()
    if args.impl == 'reference':
        run_reference(args, world, rank)
        return
    import torch
    import torch.distributed as dist
    if not torch.cuda.is_available():
        raise SystemExit('bench.py needs a CUDA device')
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group('nccl', timeout=timedelta(seconds=600), device_id=torch.device('cuda', local))
    import ehss_b200 as eb
    from ehss_b200 import _lib
    from ehss_b200.batch import BatchCCS
    from ehss_b200.blocks import BlockPlan
    _lib.load()

    def barrier():
        if world > 1:
            dist.barrier()

    # one job: args.structures structures per GPU, made by one generator; with N GPUs the
    # N * args.structures structures are shared out by LPT and one all-reduce of the block
    # integers closes every step (at N = 1 there is nothing to exchange)
    from ehss_b200.distributed import ShardedBatch
    mine = None
    if world > 1:
        # every rank makes only its own structures (the LPT shares follow from the sizes alone)
        from ehss_b200 import distributed as D, workloads as W
        spec = W.mixed_batch(args.structures * world, seed=MASTER_SEED)
        owner = D.shard([D.estimated_cost(n, 1 << lg) for n, lg, _ in spec], world)
        mine = [i for i, o in enumerate(owner) if o == rank]
        all_structures = [W.globule(n, sd)[:2] if o == rank else (np.zeros((n, 3)), np.ones(n))
                          for (n, _, sd), o in zip(spec, owner)]
        all_log2s = [lg for _, lg, _ in spec]
        all_seeds = [sd % (2 ** 32) for _, _, sd in spec]
        structures = [all_structures[i] for i in mine]
        log2s = [all_log2s[i] for i in mine]
        seeds = [all_seeds[i] for i in mine]
    else:
        structures, log2s, seeds = make_structures(args.structures, MASTER_SEED)
    launch = None
    if not args.no_autotune:
        from ehss_b200 import autotune
        probe = BatchCCS(structures, log2s, seeds, repeats=REPEATS, cap=CAP, precision='fp32', graph=False)
        probe.upload(); probe.build()
        launch, _ = autotune.tune(probe.plan.jobs, passes=1)
        del probe
    job = None
    if world > 1:
        job = ShardedBatch(all_structures, all_log2s, all_seeds, rank, world, repeats=REPEATS, cap=CAP,
                           precision='fp32', launch=launch)
        assert job.mine == mine
        bc = job.batch
    else:
        bc = BatchCCS(structures, log2s, seeds, repeats=REPEATS, cap=CAP, precision='fp32', launch=launch)

    def exchange():
        if job is not None:
            job.exchange()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device='cuda')
    stream = torch.cuda.current_stream()

    bc.upload()
    for _ in range(max(args.warmup, 3)):
        bc.build()
        bc.trace()
        exchange()
    bc.run()
    torch.cuda.synchronize()
    # a long-running service moves its start-up objects out of the collector's
    # way; otherwise a full collection of the interpreter heap (~0.2 M objects
    # with torch loaded) lands inside whichever step allocates next
    gc.collect()
    gc.freeze()

    # -- device-resident steps ---------------------------------------------------
    step_ms, trace_ms = [], []
    barrier(); torch.cuda.synchronize()
    sampler = ClockSampler(local)
    for _ in range(args.steps):
        flush.zero_()
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record(stream)
        bc.build()
        e1.record(stream)
        bc.trace()
        e2.record(stream)
        exchange()
        e3 = torch.cuda.Event(enable_timing=True)
        e3.record(stream)
        e3.synchronize()
        step_ms.append(e0.elapsed_time(e3)); trace_ms.append(e1.elapsed_time(e2))
    torch.cuda.synchronize(); barrier()
    clocks = sampler.stop()
    total_ms = float(sum(step_ms))
    if world > 1:
        t = torch.tensor([total_ms], device='cuda', dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    rays_step = bc.rays
    job_rays = job.rays if job is not None else rays_step
    value = job_rays * args.steps / (total_ms * 1e-3)
    structs_per_s = args.structures * world * args.steps / (total_ms * 1e-3)
    mean_trace_ms = float(np.mean(trace_ms))
    stats = np.sum([r['stats'] for r in bc.plan.collect()], axis=0)
    # one instrumented launch (outside the timed region): our own box/sphere tests per query
    bc.plan.launch.options |= _lib.LAUNCH_COUNT_TESTS
    bc.plan.enqueue()
    cstats = np.sum([r['stats'] for r in bc.plan.collect()], axis=0)
    bc.plan.launch.options &= ~_lib.LAUNCH_COUNT_TESTS
    bc.plan.enqueue()            # the block results of the timed work again (the checks below read them)
    own = {"box_tests_per_query": float(cstats[_lib.STAT_BOX]) / max(1, cstats[_lib.STAT_QUERIES]),
           "sphere_tests_per_query": float(cstats[_lib.STAT_SPHERE]) / max(1, cstats[_lib.STAT_QUERIES]),
           "queries_per_ray": float(cstats[_lib.STAT_QUERIES]) / rays_step}

    # -- end to end through the public API (pinned host in, host results out) -----
    e2e_ms = []
    for _ in range(max(3, args.steps // 2)):
        flush.zero_()
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True); b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        results = bc.run()
        if job is not None:
            job.exchange().cpu()     # the whole job's block integers on every rank's host
        b.record(stream)
        b.synchronize()
        e2e_ms.append(a.elapsed_time(b))
    e2e_total = float(np.mean(e2e_ms))
    if world > 1:
        t = torch.tensor([e2e_total], device='cuda', dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_total = float(t.item())
    e2e_value = job_rays / (e2e_total * 1e-3)

    # -- plain path: one structure per build + launch, no graph --------------------
    plain = None
    if not args.no_plain and world == 1:
        from ehss_b200.blocks import BlockJob
        lib = _lib.load()
        import ctypes as ct
        plans = []
        for s, sc in enumerate(bc.scenes):
            jobs = [j for j in bc.plan.jobs if j.tag[0] == s]
            plans.append(BlockPlan([BlockJob(j.scene, j.log2_rays, j.seed, cap=j.cap, precision=j.precision,
                                             tag=j.tag) for j in jobs]))
        bs = bc.batch
        ws = torch.empty(bs.ws_bytes + 256, dtype=torch.uint8, device='cuda')
        ws_ptr = (ws.data_ptr() + 255) & ~255
        sh = torch.cuda.current_stream().cuda_stream

        def plain_structure(s):
            # same scene kind as the batch (exterior), one structure per build
            _lib.check(lib.ehss_scenes_build_ex(1, (ct.c_void_p * 1)(bs._xyz_ptrs[s]), (ct.c_void_p * 1)(bs._r_ptrs[s]),
                                                (ct.c_int64 * 1)(int(bs.n_atoms[s])), bs.leaf_size,
                                                (ct.c_void_p * 1)(bs.scene_ptrs[s]), (ct.c_uint64 * 1)(bs._sizes[s]),
                                                ws_ptr, bs.ws_bytes, bs.flags, sh))
            plans[s].enqueue()
        for s in range(len(plans)):          # warm-up
            plain_structure(s)
        torch.cuda.synchronize()
        lat = []
        t0 = torch.cuda.Event(enable_timing=True); t1 = torch.cuda.Event(enable_timing=True)
        flush.zero_()
        t0.record(stream)
        for s in range(len(plans)):
            a = torch.cuda.Event(enable_timing=True); b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            plain_structure(s)
            b.record(stream)
            lat.append((a, b))
        t1.record(stream)
        t1.synchronize()
        plain_ms = t0.elapsed_time(t1)
        lats = np.array([a.elapsed_time(b) for a, b in lat])
        plain = {"rays_per_s": rays_step / (plain_ms * 1e-3), "structures_per_s": args.structures / (plain_ms * 1e-3),
                 "ms_per_pass": plain_ms, "latency_ms_p50": float(np.percentile(lats, 50)),
                 "latency_ms_p99": float(np.percentile(lats, 99))}

    # -- roofline, CPU baseline and CCS error (rank 0, N = 1 only for the baseline) ---
    n_sm = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    clock_mhz = float(clocks['sm_mhz']) if clocks else 1965.0

    def peak_tflops():
        # FP32 CUDA-core peak at the clock sampled under load: SMs x 128 lanes x 2 (FMA) x clock
        return n_sm * 128 * 2 * clock_mhz * 1e6 / 1e12
    roof = None
    cpu = None
    ccs = None
    configs = None
    explicit = None
    if rank == 0:
        check = oracle_check_blocks(bc.plan, structures, lambda i: bc.plan.jobs[i].tag[0])
        rays_per_block = [1 << j.log2_rays for j in bc.plan.jobs]
        ops_step, s_ray, b_ray = ops_from_check(check, rays_per_block)
        achieved = ops_step / (mean_trace_ms * 1e-3) / 1e12
        traffic = traffic_per_launch()
        peak = peak_tflops()
        sgemm_tflops = measured_fp32_tflops()
        roof = {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "traffic": traffic.get('bytes_per_launch') if traffic else None,
                "kernel": "ehss::k_blocks", "kernel_ms": mean_trace_ms,
                "ops_per_ray": ops_step / rays_step, "ref_sphere_tests_per_ray": s_ray, "ref_box_tests_per_ray": b_ray,
                "ops_source": f"reference BVH sphere/box tests counted by the oracle on the timed rays of "
                              f"{check['checked']} of {check['blocks']} blocks (35 and 27 FP32 ops each)",
                "peak_note": f"FP32 peak: {n_sm} SMs x 128 lanes x 2 x {clock_mhz:.0f} MHz (median SM clock sampled "
                             f"during the timed steps; the measured-peaks file holds no FP32 figure)",
                "sgemm_fp32_tflops_side_note": sgemm_tflops}
        sphere_rate = s_ray * rays_step / (mean_trace_ms * 1e-3)
        roof["ray_sphere_tests"] = {"achieved_per_s": sphere_rate, "peak_per_s": peak * 1e12 / C_SPHERE,
                                    "frac": sphere_rate / (peak * 1e12 / C_SPHERE),
                                    "own_tests_per_s": own["sphere_tests_per_query"] * own["queries_per_ray"] *
                                    rays_step / (mean_trace_ms * 1e-3)}
        # per-structure CCS (mean of the replicate blocks) against the oracle's on the same rays
        ok = np.isfinite(check['rel_err'])
        dev_s = check['device'].reshape(-1, REPEATS)
        ora_s = check['oracle'].reshape(-1, REPEATS)
        full = ok.reshape(-1, REPEATS).all(axis=1)
        per_struct = np.abs(dev_s.mean(axis=1) - ora_s.mean(axis=1)) / ora_s.mean(axis=1)
        ccs = {"blocks_checked": check['checked'], "blocks": check['blocks'],
               "block_rel_err_max": float(np.nanmax(check['rel_err'])),
               "block_rel_err_median": float(np.nanmedian(check['rel_err'])),
               "structures_checked": int(full.sum()),
               "structure_rel_err_max": float(per_struct[full].max()) if full.any() else None,
               "oracle_seconds": check['seconds'], "oracle_threads": check['cores'],
               "rays": "the timed blocks' own device rays (same structures, seeds and 2^k counts)"}
        if world == 1:
            configs = configuration_lines(eb, flush, peak_tflops)
            explicit = explicit_trace_e2e(eb)
        if world == 1 and not args.no_cpu_baseline:
            rate, kind, cores, rays_done, secs = cpu_reference_rate(structures[::16], 12, 190003)
            cpu = {"value": rate, "unit": UNIT, "cores": cores, "kind": kind,
                   "sample": f"{len(structures[::16])} of {len(structures)} structures (every 16th), 2^12 rays each, "
                             f"cap {CAP}; {rays_done} rays in {secs:.1f} s",
                   "numba": numba_reference_rates(structures[::16], 12, 190003)}
    serve = None
    if rank == 0 and world == 1 and not args.no_serve:
        serve = serving_measurement()
    if rank == 0:
        # builder: scene index + stats, 5 tree kernels per pass (keys sorted per structure in one
        # kernel: every structure here holds at most 8192 atoms), two passes around exposure + its
        # fix-up; then 1 persistent trace kernel
        launches_per_step = 2 + 5 * 2 + 2 + 1
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
                "config": config(args, world),
                "structures_per_s": structs_per_s,
                "rays_per_step": job_rays,
                "trace_ms_per_step": mean_trace_ms, "build_ms_per_step": float(np.mean(step_ms) - mean_trace_ms),
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": bc.h2d_bytes,
                        "d2h_bytes_per_step": bc.d2h_bytes + (job.packed.numel() * 8 if job is not None else 0),
                        "ms_per_step": e2e_total,
                        "structures_per_s": args.structures * world / (e2e_total * 1e-3)},
                "plain": plain,
                "batched_over_plain": (value / world / plain['rays_per_s']) if plain else None,
                "ccs_rel_err_max_vs_fp64_oracle": ccs["block_rel_err_max"] if ccs else None,
                "ccs_vs_fp64_oracle": ccs, "configs": configs, "e2e_explicit": explicit,
                "grazing_queries": int(stats[_lib.STAT_GRAZING]), "fp64_fallback_queries": int(stats[_lib.STAT_FALLBACK]),
                "queries": int(stats[_lib.STAT_QUERIES]), "own_traversal": own,
                "served": serve, "launch": {k: int(v) for k, v in (launch or {}).items()} or None,
                "roofline": roof, "cpu_baseline": cpu, "clocks": clocks,
                "gpu_launches": launches_per_step * args.steps}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == '__main__':
    main()
