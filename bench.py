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
            "l2": "flushed (256 MB write) between timed steps", "host": "gc.freeze() after set-up", "parallelism": f"replicas x{world} (weak)"}


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
def reference_ops_per_ray(structures, sample_log2=10, seed=12345):
    """Mean reference sphere/box tests per ray for each structure (oracle counters)."""
    from oracle import oracle as O
    ops, s_mean, b_mean = [], [], []
    for c, r in structures:
        src = O.external_source(c, r, sample_log2, seed)
        t = O.StaticTree(c, r, 4)
        res = t.trace(src['origins'], src['directions'], cap=CAP, threads=O.host_cores())
        n = len(src['origins'])
        s, b = res['sphere_tests'] / n, res['box_tests'] / n
        s_mean.append(s); b_mean.append(b)
        ops.append(C_SPHERE * s + C_BOX * b)
    return np.array(ops), np.array(s_mean), np.array(b_mean)


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


def ccs_error_vs_oracle(eb, structures, log2=12, seed=777):
    """Max relative CCS error of the FP32 device path vs the FP64 oracle on the same rays."""
    from oracle import oracle as O
    from ehss_b200.blocks import BlockJob, BlockPlan
    worst = 0.0
    for c, r in structures:
        scene = eb.Scene(c, r, exterior=True)
        plan = BlockPlan([BlockJob(scene, log2, seed, cap=CAP)])
        plan.run()
        got = plan.collect()[0]['ehss_angstrom2']
        o, d = scene.source_rays(log2, seed)
        o, d = o.cpu().numpy(), d.cpu().numpy()
        res = O.StaticTree(c, r, 4).trace(o, d, cap=CAP, threads=O.host_cores())
        n = len(o)
        ro = O.readout(dict(incoming=d, weights=np.full(n, np.pi * scene.radius ** 2 / n)), res, CAP)
        worst = max(worst, abs(got - ro['ehss_angstrom2']) / ro['ehss_angstrom2'])
    return worst


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
    if rank != 0:
        return
    from oracle import oracle as O
    structures, log2s, seeds = make_structures(args.structures, MASTER_SEED)
    sample = structures[::8]
    threads = O.host_cores()
    kind = 'reference' if O.ref_available() else 'port'
    prepared = []
    for c, r in sample:
        src = O.external_source(c, r, 12, 190003)
        prepared.append((O.StaticTree(c, r, 4), src['origins'], src['directions']))
    rays_step = sum(len(o) for _, o, _ in prepared)

    def step():
        for tree, o, d in prepared:
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
    sample_txt = f"{len(sample)} of {len(structures)} structures (every 8th), 2^12 rays each, cap {CAP}, per step"
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": dict(config(args, world), precision="fp64 (the reference's own C++ kernel)",
                           scenes="full (the reference's static tree over every atom)"),
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

    structures, log2s, seeds = make_structures(args.structures, MASTER_SEED + rank)
    launch = None
    if not args.no_autotune:
        from ehss_b200 import autotune
        probe = BatchCCS(structures, log2s, seeds, repeats=REPEATS, cap=CAP, precision='fp32', graph=False)
        probe.upload(); probe.build()
        launch, _ = autotune.tune(probe.plan.jobs, passes=1)
        del probe
    bc = BatchCCS(structures, log2s, seeds, repeats=REPEATS, cap=CAP, precision='fp32', launch=launch)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device='cuda')
    stream = torch.cuda.current_stream()

    bc.upload()
    for _ in range(max(args.warmup, 3)):
        bc.build()
        bc.trace()
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
        e2.synchronize()
        step_ms.append(e0.elapsed_time(e2)); trace_ms.append(e1.elapsed_time(e2))
    torch.cuda.synchronize(); barrier()
    clocks = sampler.stop()
    total_ms = float(sum(step_ms))
    if world > 1:
        t = torch.tensor([total_ms], device='cuda', dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    rays_step = bc.rays
    value = rays_step * world * args.steps / (total_ms * 1e-3)
    structs_per_s = args.structures * world * args.steps / (total_ms * 1e-3)
    mean_trace_ms = float(np.mean(trace_ms))
    stats = np.sum([r['stats'] for r in bc.plan.collect()], axis=0)
    # one instrumented launch (outside the timed region): our own box/sphere tests per query
    bc.plan.launch.options |= _lib.LAUNCH_COUNT_TESTS
    bc.plan.enqueue()
    cstats = np.sum([r['stats'] for r in bc.plan.collect()], axis=0)
    bc.plan.launch.options &= ~_lib.LAUNCH_COUNT_TESTS
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
        b.record(stream)
        b.synchronize()
        e2e_ms.append(a.elapsed_time(b))
    e2e_total = float(np.mean(e2e_ms))
    if world > 1:
        t = torch.tensor([e2e_total], device='cuda', dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_total = float(t.item())
    e2e_value = rays_step * world / (e2e_total * 1e-3)

    # -- plain path: one structure per build + launch, no graph --------------------
    plain = None
    if not args.no_plain:
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
    pk = peaks()
    sm_max = float(pk.get('sm_max_mhz', 1965.0))
    n_sm = torch.cuda.get_device_properties(0).multi_processor_count
    nominal_tflops = n_sm * 128 * 2 * sm_max * 1e6 / 1e12
    sgemm_tflops = measured_fp32_tflops() if rank == 0 else None
    roof = None
    cpu = None
    ccs_err = None
    if rank == 0:
        ops, s_ref, b_ref = reference_ops_per_ray(structures)
        ray_counts = np.array([(1 << lg) * REPEATS for lg in log2s], dtype=np.float64)
        ops_step = float(np.sum(ray_counts * ops))
        achieved = ops_step / (mean_trace_ms * 1e-3) / 1e12
        traffic = traffic_per_launch()
        peak_tflops = sgemm_tflops
        roof = {"bound": "fp32", "achieved": achieved, "peak": peak_tflops, "unit": "TFLOP/s",
                "frac": achieved / peak_tflops, "peak_nominal": nominal_tflops,
                "frac_of_nominal": achieved / nominal_tflops,
                "traffic": traffic.get('bytes_per_launch') if traffic else None,
                "kernel": "ehss::k_blocks", "kernel_ms": mean_trace_ms,
                "ops_per_ray": ops_step / rays_step,
                "ref_sphere_tests_per_ray": float(np.sum(ray_counts * s_ref) / ray_counts.sum()),
                "ref_box_tests_per_ray": float(np.sum(ray_counts * b_ref) / ray_counts.sum()),
                "peak_note": "measured: cuBLAS FP32 SGEMM 8192^3, TF32 off, best of 3 (the measured-peaks file has "
                             f"no FP32 figure); nominal: {n_sm} SMs x 128 lanes x 2 x {sm_max:.0f} MHz"}
        # the ray-sphere-test roofline: reference sphere tests per second against peak / 35 ops
        sphere_rate = float(np.sum(ray_counts * s_ref)) / (mean_trace_ms * 1e-3)
        roof["ray_sphere_tests"] = {"achieved_per_s": sphere_rate, "peak_per_s": peak_tflops * 1e12 / C_SPHERE,
                                    "frac": sphere_rate / (peak_tflops * 1e12 / C_SPHERE),
                                    "own_tests_per_s": own["sphere_tests_per_query"] * own["queries_per_ray"] *
                                    rays_step / (mean_trace_ms * 1e-3)}
        ccs_err = ccs_error_vs_oracle(eb, structures[::32])
        if world == 1 and not args.no_cpu_baseline:
            rate, kind, cores, rays_done, secs = cpu_reference_rate(structures[::16], 12, 190003)
            cpu = {"value": rate, "unit": UNIT, "cores": cores, "kind": kind,
                   "sample": f"{len(structures[::16])} of {len(structures)} structures (every 16th), 2^12 rays each, "
                             f"cap {CAP}; {rays_done} rays in {secs:.1f} s"}
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
                "rays_per_step": rays_step * world,
                "trace_ms_per_step": mean_trace_ms, "build_ms_per_step": float(np.mean(step_ms) - mean_trace_ms),
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": bc.h2d_bytes,
                        "d2h_bytes_per_step": bc.d2h_bytes, "ms_per_step": e2e_total,
                        "structures_per_s": args.structures * world / (e2e_total * 1e-3)},
                "plain": plain,
                "batched_over_plain": (value / world / plain['rays_per_s']) if plain else None,
                "ccs_rel_err_max_vs_fp64_oracle": ccs_err,
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
