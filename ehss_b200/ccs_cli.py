"""The ccs.py calculation surface on the B200 path.

Same command line, validation, input handling, error codes and output files
as the reference CLI (src/support_exchange_transport/ccs_cli.py): XYZ frames
in, ``summary.csv`` and ``results.json`` out.  What changes is solve_frame:
every replicate of a frame runs on the device in one fused launch (Sobol ->
impact disk -> EHSS trace and/or BVH PA -> reduction), with the scene's LBVH
built once and kept resident across replicates.  ``--threads`` is accepted
and recorded (the GPU replaces worker threads); ``--leaf-size`` bounds the
device LBVH leaves (1..16).
"""
from __future__ import annotations

import argparse
import csv
import glob
import hashlib
import json
import math
import platform
import re
import sys
import time
from collections import Counter
from dataclasses import dataclass
from datetime import datetime, timezone
from pathlib import Path

import numpy as np

VERSION = "0.1.0"
# van der Waals radii (Mantina et al. 2009, Table 12; H = 1.10), Angstrom,
# the reference CLI's table (ccs_cli.py:29-31)
VDW_RADII = {"H": 1.10, "He": 1.40, "C": 1.70, "N": 1.55, "O": 1.52, "F": 1.47, "Si": 2.10, "P": 1.80,
             "S": 1.80, "Cl": 1.75, "Se": 1.90, "Br": 1.83, "I": 1.98}
RADII_SOURCE = 'Mantina et al. 2009 Table 12, subset; DOI 10.1021/jp8111556; user overrides recorded in table'


@dataclass
class XYZFrame:
    number: int
    comment: str
    elements: tuple
    coordinates: np.ndarray


def element_symbol(value):
    if not isinstance(value, str) or not re.fullmatch(r"[A-Za-z]{1,2}", value):
        raise ValueError(f"Expected an element symbol, got {value!r}")
    return value[0].upper() + value[1:].lower()


def read_xyz(path):
    """Strict standard XYZ, every frame read (ccs_cli.read_xyz, ccs_cli.py:48-83)."""
    lines = Path(path).read_text(encoding="utf-8-sig").splitlines()
    frames = []
    i = 0
    while i < len(lines):
        if not lines[i].strip():
            i += 1
            continue
        head = lines[i].strip()
        if not re.fullmatch(r"[1-9][0-9]*", head):
            raise ValueError(f"{path}:{i + 1}: expected a positive atom count")
        count = int(head)
        if i + count + 1 >= len(lines):
            raise ValueError(f"{path}:{i + 1}: incomplete XYZ frame (comment and {count} atom rows required)")
        comment = lines[i + 1]
        if "Lattice=" in comment or "Properties=" in comment:
            raise ValueError(f"{path}:{i + 2}: extended/periodic XYZ is not supported; export a standard isolated molecule")
        elements, coords = [], []
        for j in range(i + 2, i + 2 + count):
            fields = lines[j].split()
            if len(fields) != 4:
                raise ValueError(f"{path}:{j + 1}: expected exactly 'Element x y z'")
            try:
                symbol = element_symbol(fields[0])
                xyz = [float(x.replace('D', 'E').replace('d', 'e')) for x in fields[1:]]
            except ValueError as exc:
                raise ValueError(f"{path}:{j + 1}: invalid element or coordinates") from exc
            if not np.isfinite(xyz).all():
                raise ValueError(f"{path}:{j + 1}: coordinates must be finite")
            elements.append(symbol)
            coords.append(xyz)
        frames.append(XYZFrame(len(frames) + 1, comment, tuple(elements), np.array(coords)))
        i += count + 2
    if not frames:
        raise ValueError(f"{path}: no XYZ frames")
    return frames


def radius_table(path=None):
    table = dict(VDW_RADII)
    if path:
        raw = json.loads(Path(path).read_text(encoding="utf-8-sig"))
        if not isinstance(raw, dict) or not raw:
            raise ValueError("Radii JSON must be a nonempty object: {\"C\": 1.70, ...}")
        seen = set()
        for name, value in raw.items():
            symbol = element_symbol(name)
            if symbol in seen:
                raise ValueError(f"Duplicate normalized radius key: {symbol}")
            seen.add(symbol)
            if isinstance(value, bool) or not isinstance(value, (int, float)) or not math.isfinite(value) or value <= 0:
                raise ValueError(f"Radius for {symbol} must be a positive finite number in angstrom")
            table[symbol] = float(value)
    return table


def prepare_frame(frame, radii, probe_radius, units="angstrom", exclude_hydrogen=False):
    """Selected atoms, recentred, effective radius = vdW + probe (ccs_cli.py:104-126)."""
    from .state import Spheres
    keep = [i for i, e in enumerate(frame.elements) if not (exclude_hydrogen and e == "H")]
    if not keep:
        raise ValueError(f"Frame {frame.number}: atom selection is empty")
    elements = [frame.elements[i] for i in keep]
    unknown = sorted(set(elements) - radii.keys())
    if unknown:
        raise ValueError(f"Frame {frame.number}: no radius for {', '.join(unknown)}; supply --radii-json")
    xyz = frame.coordinates[keep] * (10. if units == "nm" else 1.)
    if not np.isfinite(xyz).all():
        raise ValueError("Coordinates overflow after unit conversion")
    if len(np.unique(xyz, axis=0)) != len(xyz):
        raise ValueError(f"Frame {frame.number}: coincident selected atom centers; check duplicate atoms")
    offset = xyz[0] + np.mean(xyz - xyz[0], axis=0)
    effective = np.array([radii[e] + probe_radius for e in elements])
    spheres = Spheres(xyz - offset, effective, deduplicate=False)
    info = dict(frame=frame.number, comment=frame.comment, input_atoms=len(frame.elements),
                selected_atoms=len(keep), selected_atom_rows_1based=[i + 1 for i in keep],
                element_counts=dict(Counter(elements)), recenter_offset_angstrom=offset.tolist(),
                effective_radii_angstrom={e: radii[e] + probe_radius for e in sorted(set(elements))})
    return spheres, info


def summarize(values):
    a = np.asarray(values, dtype=float)
    sd = float(a.std(ddof=1)) if len(a) > 1 else None
    return dict(mean=float(a.mean()), sd=sd, sem=sd / math.sqrt(len(a)) if sd is not None else None,
                replicates=len(a))


def solve_frame(spheres, args, progress=True):
    """All replicates of one frame on the device (ccs_cli.solve_frame, ccs_cli.py:170-232)."""
    import torch
    from . import _lib
    from .blocks import BlockJob, BlockPlan, seed_schedule
    from .engine import Scene
    ehss = args.method in ("ehss", "both")
    pa = args.method in ("pa", "both")
    start = time.perf_counter()
    tick = time.perf_counter()
    # block rays all start on the impact disk, so buried atoms can leave the tree (exterior scene)
    scene = Scene(spheres.centers, spheres.radii, leaf_size=min(int(args.leaf_size), 16), exterior=True)
    setup_s = time.perf_counter() - tick
    seeds = seed_schedule(args.seed, args.repeats)
    rows = [dict(repeat=k + 1, seed=s) for k, s in enumerate(seeds)]
    adaptive = pa and args.pa_method == "adaptive"
    bvh_pa = pa and args.pa_method == "bvh"
    if adaptive:
        from .adaptive_pa import adaptive_pa
        for row in rows:
            if progress:
                print(f"  replicate {row['repeat']}/{args.repeats} (seed {row['seed']})", file=sys.stderr, flush=True)
            row['pa'] = adaptive_pa(spheres, args.directions, args.grid_size, row['seed'], scene=scene)
    if ehss or bvh_pa:
        log2 = args.rays.bit_length() - 1
        jobs = [BlockJob(scene, log2, s, cap=args.max_collisions, precision=_lib.PREC_FP32, ehss=ehss, pa=bvh_pa,
                         tag=k) for k, s in enumerate(seeds)]
        plan = BlockPlan(jobs)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        plan.enqueue()
        e1.record()
        tick = time.perf_counter()
        results = plan.collect()
        readout_s = (time.perf_counter() - tick) / len(rows)
        query_s = e0.elapsed_time(e1) * 1e-3 / len(rows)
        for row, res in zip(rows, results):
            _frame_row(row, res, ehss, bvh_pa, query_s, readout_s)
            if ehss:
                tail = res['tail_bound_angstrom2']
                if progress:
                    print(f"  replicate {row['repeat']}/{args.repeats} (seed {row['seed']})", file=sys.stderr,
                          flush=True)
                    if res['unresolved_rays']:
                        print(f"  WARNING: {res['unresolved_rays']} unresolved rays; omitted contribution <= {tail:.6g} "
                              "A^2. Increase --max-collisions.", file=sys.stderr)
    total = time.perf_counter() - start
    summary = _summary(rows, ehss, pa)
    return dict(summary=summary, runs=rows,
                timings=dict(ehss_setup_s=setup_s if ehss else 0., pa_setup_s=setup_s if bvh_pa else 0.,
                             all_replicates_with_setup_s=total))


def _frame_row(row, res, ehss, bvh_pa, query_s, readout_s):
    row['impact_source_s'] = 0.0            # generated inside the fused kernel
    if bvh_pa:
        row['pa'] = dict(pa_angstrom2=res['pa_angstrom2'], query_s=query_s, readout_s=readout_s,
                         box_tests=None, sphere_tests=None)
    if ehss:
        omega, tail = res['ehss_angstrom2'], res['tail_bound_angstrom2']
        row['ehss'] = dict(ehss_angstrom2=omega, pa_from_same_rays_angstrom2=res['pa_from_same_rays_angstrom2'],
                           tail_bound_angstrom2=tail, sampled_interval_angstrom2=[omega, omega + tail],
                           unresolved_rays=res['unresolved_rays'], query_s=query_s,
                           collision_histogram=res['collision_histogram'],
                           collision_contribution_angstrom2=res['collision_contribution_angstrom2'],
                           box_tests=None, sphere_tests=None, readout_s=readout_s,
                           grazing_queries=res['grazing_queries'], fp64_fallback_queries=res['fp64_fallback_queries'])


def _summary(rows, ehss, pa):
    summary = {}
    if pa:
        summary['pa_angstrom2'] = summarize([r['pa']['pa_angstrom2'] for r in rows])
    if ehss:
        summary['ehss_angstrom2'] = summarize([r['ehss']['ehss_angstrom2'] for r in rows])
        summary['ehss_tail_bound_mean_angstrom2'] = float(np.mean([r['ehss']['tail_bound_angstrom2'] for r in rows]))
        summary['ehss_unresolved_rays_total'] = sum(r['ehss']['unresolved_rays'] for r in rows)
    return summary


# frames traced together in one batched build and one persistent launch
FRAME_BATCH_ATOMS = 2_000_000
FRAME_BATCH_FRAMES = 1024


def solve_frames(frames, args, progress=True):
    """Many frames (``--all-frames``, several files) at once: one batched
    scene build and one persistent launch for all replicates of a group of
    frames, instead of one of each per frame.  Each frame's results are the
    same integers as solve_frame's (block sums do not depend on what shares
    the launch); timings are the group's, divided evenly over its frames."""
    import torch
    from .batch import BatchCCS
    from .blocks import seed_schedule
    ehss = args.method in ("ehss", "both")
    pa = args.method in ("pa", "both")
    bvh_pa = pa and args.pa_method == "bvh"
    if not (ehss or bvh_pa):
        return [solve_frame(s, args, progress) for s in frames]
    out = []
    i = 0
    while i < len(frames):
        group, atoms = [], 0
        while i < len(frames) and len(group) < FRAME_BATCH_FRAMES and \
                (not group or atoms + len(frames[i].radii) <= FRAME_BATCH_ATOMS):
            group.append(frames[i]); atoms += len(frames[i].radii); i += 1
        start = time.perf_counter()
        seeds = seed_schedule(args.seed, args.repeats)
        log2 = args.rays.bit_length() - 1
        bc = BatchCCS([(s.centers, s.radii) for s in group], log2, [args.seed] * len(group), repeats=args.repeats,
                      cap=args.max_collisions, precision='fp32', ehss=ehss, pa=bvh_pa,
                      leaf_size=min(int(args.leaf_size), 16), graph=False)
        bc.upload()
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record()
        bc.build()
        e1.record()
        bc.trace()
        e2.record()
        tick = time.perf_counter()
        per = bc.download()
        readout_s = (time.perf_counter() - tick) / (len(group) * args.repeats)
        setup_s = e0.elapsed_time(e1) * 1e-3 / len(group)
        query_s = e1.elapsed_time(e2) * 1e-3 / (len(group) * args.repeats)
        total = (time.perf_counter() - start) / len(group)
        for spheres, p in zip(group, per):
            rows = [dict(repeat=k + 1, seed=sd) for k, sd in enumerate(seeds)]
            if pa and args.pa_method == "adaptive":
                from .adaptive_pa import adaptive_pa
                for row in rows:
                    row['pa'] = adaptive_pa(spheres, args.directions, args.grid_size, row['seed'])
            for row, res in zip(rows, p['runs']):
                _frame_row(row, res, ehss, bvh_pa, query_s, readout_s)
            out.append(dict(summary=_summary(rows, ehss, pa), runs=rows,
                            timings=dict(ehss_setup_s=setup_s if ehss else 0., pa_setup_s=setup_s if bvh_pa else 0.,
                                         all_replicates_with_setup_s=total, batched_frames=len(group))))
        if progress:
            print(f"  traced {len(group)} frame(s) in one batch", file=sys.stderr, flush=True)
    return out


def parser():
    p = argparse.ArgumentParser(description="PA/EHSS for isolated molecules in standard XYZ files (results in A^2).")
    p.add_argument('xyz', nargs='+', help='XYZ paths; quoted wildcard patterns also work on Windows')
    p.add_argument('--version', action='version', version='ccs-xyz ' + VERSION)
    p.add_argument('--method', choices=['pa', 'ehss', 'both'], default='both')
    p.add_argument('--pa-method', choices=['adaptive', 'bvh'], default='adaptive')
    p.add_argument('--rays', type=int, default=16384, help='EHSS/BVH PA rays per replicate, power of two (default: 16384)')
    p.add_argument('--directions', type=int, default=64, help='Adaptive PA directions per replicate, power of two (default: 64)')
    p.add_argument('--grid-size', type=int, default=512, help='Adaptive PA square midpoint grid, power of two (default: 512)')
    p.add_argument('--repeats', type=int, default=3, help='Independent scrambled Sobol replicates (default: 3)')
    p.add_argument('--seed', type=int, default=190003)
    p.add_argument('--threads', type=int, default=1, help='Accepted for compatibility; the GPU replaces CPU threads')
    p.add_argument('--leaf-size', type=int, default=14, help='Maximum atoms per device LBVH leaf (1..16, default: 14)')
    p.add_argument('--max-collisions', type=int, default=64)
    p.add_argument('--probe-radius', type=float, default=1.4, help='Added probe radius in angstrom (default: 1.4, He scenario)')
    p.add_argument('--radii-json', type=Path, help='Overrides/additions to atomic VDW radii in angstrom, never effective radii')
    p.add_argument('--units', choices=['angstrom', 'nm'], default='angstrom', help='Input coordinate units only')
    p.add_argument('--exclude-hydrogen', action='store_true', help='Explicitly omit H; default includes every supplied atom')
    f = p.add_mutually_exclusive_group()
    f.add_argument('--frame', type=int, default=1, help='1-based frame selection (default: first frame)')
    f.add_argument('--all-frames', action='store_true', help='Calculate every frame independently, no MD cache reuse')
    p.add_argument('--output', type=Path, default=Path('ccs_results'), help='New result directory; existing directory is preserved')
    return p


def validate_args(args):
    for name, low, high in [('rays', 8, 2 ** 22), ('directions', 1, 2 ** 16), ('grid_size', 8, 8192)]:
        value = getattr(args, name)
        if not low <= value <= high or value & (value - 1):
            raise ValueError(f"--{name.replace('_', '-')} must be a power of two in {low}..{high}")
    for name in ['repeats', 'threads', 'leaf_size', 'max_collisions', 'frame']:
        if getattr(args, name) < 1:
            raise ValueError(f"--{name.replace('_', '-')} must be positive")
    if args.max_collisions > 100000:
        raise ValueError('--max-collisions must be <= 100000')
    if not 0 <= args.seed < 2 ** 32:
        raise ValueError('--seed must be in 0..4294967295')
    if not math.isfinite(args.probe_radius) or args.probe_radius < 0:
        raise ValueError('--probe-radius must be finite and nonnegative')
    if args.output.exists():
        raise ValueError(f"Output already exists: {args.output}; choose a new --output directory")


def environment():
    import torch
    env = dict(python=platform.python_version(), platform=platform.platform(), numpy=np.__version__,
               torch=torch.__version__, cuda=torch.version.cuda)
    if torch.cuda.is_available():
        env['gpu'] = torch.cuda.get_device_name()
    return env


def execute(args):
    validate_args(args)
    from .device import require_cuda
    from .state import Spheres
    require_cuda()
    started = time.perf_counter()
    table = radius_table(args.radii_json)
    jobs, seen = [], set()
    for pattern in args.xyz:
        matches = [pattern] if Path(pattern).is_file() else sorted(glob.glob(pattern))
        if not matches:
            raise ValueError(f"No XYZ files match: {pattern}")
        for match in matches:
            path = Path(match).resolve()
            if path in seen:
                continue
            seen.add(path)
            frames = read_xyz(path)
            if not args.all_frames and args.frame > len(frames):
                raise ValueError(f"{path.name}: --frame {args.frame} exceeds {len(frames)} frames")
            selected = frames if args.all_frames else [frames[args.frame - 1]]
            if len(frames) > 1 and not args.all_frames:
                print(f"{path.name}: using frame {args.frame}/{len(frames)}; use --all-frames for all.", file=sys.stderr)
            digest = hashlib.sha256(path.read_bytes()).hexdigest()
            for frame in selected:
                spheres, info = prepare_frame(frame, table, args.probe_radius, args.units, args.exclude_hydrogen)
                jobs.append((spheres, dict(input_file=str(path), input_sha256=digest, total_frames=len(frames), **info)))
    print(f"Validated {len(jobs)} frame(s). Preparing the device kernels...", file=sys.stderr, flush=True)
    # first launch (context, module load) outside the per-frame timing
    warm = argparse.Namespace(**vars(args))
    warm.rays, warm.directions, warm.grid_size, warm.repeats = 8, 1, 8, 1
    tick = time.perf_counter()
    solve_frame(Spheres(np.array([[0., 0., 0.], [2., 0., 0.]]), np.array([1., 1.])), warm, progress=False)
    warmup_s = time.perf_counter() - tick
    records = []
    solved = solve_frames([s for s, _ in jobs], args) if len(jobs) > 1 else [None]
    for (spheres, info), result in zip(jobs, solved):
        print(f"{Path(info['input_file']).name}, frame {info['frame']}, {info['selected_atoms']} atoms", file=sys.stderr,
              flush=True)
        record = dict(**info, **(result if result is not None else solve_frame(spheres, args)))
        records.append(record)
        for name in ['pa_angstrom2', 'ehss_angstrom2']:
            if name in record['summary']:
                v = record['summary'][name]
                sd = 'n/a' if v['sd'] is None else f"{v['sd']:.6f}"
                print(f"  {name.split('_')[0].upper()}: {v['mean']:.6f} A^2 (replicate SD {sd})")
        print(f"  Compute: {record['timings']['all_replicates_with_setup_s']:.4f} s (setup + all replicates; warmup excluded)")
    config = {k: str(v) if isinstance(v, Path) else v for k, v in vars(args).items()}
    payload = dict(schema_version=1, tool='ccs-xyz', version=VERSION, backend='ehss_b200 (B200, sm_100a)',
                   created_utc=datetime.now(timezone.utc).isoformat(), settings=config, atomic_radii_angstrom=table,
                   radii_source=RADII_SOURCE, environment=environment(), warmup_s=warmup_s,
                   elapsed_before_output_s=time.perf_counter() - started,
                   notes=['Static elastic hard-sphere model; atomic VDW radius + probe radius. Not TM or fitted IMoS/EHSSrot parameters.',
                          'XYZ atoms, device LBVH; no support response reuse.',
                          'Independent Sobol scrambles across replicates. SD/SEM measure replicate variation, not total error or a guaranteed confidence interval.',
                          'Adaptive PA has finite-grid and directional error; replicate SD does not estimate grid bias.',
                          'EHSS sampled interval covers omitted cap survivors only, not sampling error or physical model error.',
                          'Warmup/import/IO excluded from per-frame compute timing; setup is once per frame, shared across replicates.',
                          'For both + BVH PA, the impact rays are shared with EHSS.',
                          'EHSS paths use FP32 traversal with FP64 re-test of every candidate; per-ray outcomes equal the FP64 path.'],
                   records=records)
    args.output.mkdir(parents=True, exist_ok=False)
    (args.output / 'results.json').write_text(json.dumps(payload, ensure_ascii=False, indent=2, allow_nan=False) + '\n',
                                              encoding='utf-8')
    columns = ['input_file', 'frame', 'atoms', 'pa_mean_A2', 'pa_sd_A2', 'ehss_mean_A2', 'ehss_sd_A2',
               'ehss_tail_bound_mean_A2', 'unresolved_rays_total', 'compute_all_replicates_s']
    with (args.output / 'summary.csv').open('w', newline='', encoding='utf-8-sig') as f:
        writer = csv.DictWriter(f, fieldnames=columns)
        writer.writeheader()
        for r in records:
            s = r['summary']
            pa_s, eh = s.get('pa_angstrom2', {}), s.get('ehss_angstrom2', {})
            writer.writerow(dict(input_file=r['input_file'], frame=r['frame'], atoms=r['selected_atoms'],
                                 pa_mean_A2=pa_s.get('mean'), pa_sd_A2=pa_s.get('sd'), ehss_mean_A2=eh.get('mean'),
                                 ehss_sd_A2=eh.get('sd'), ehss_tail_bound_mean_A2=s.get('ehss_tail_bound_mean_angstrom2'),
                                 unresolved_rays_total=s.get('ehss_unresolved_rays_total'),
                                 compute_all_replicates_s=r['timings']['all_replicates_with_setup_s']))
    print(f"Saved {args.output.resolve() / 'summary.csv'}")
    print(f"Saved {args.output.resolve() / 'results.json'}")
    return payload


def main(argv=None):
    p = parser()
    args = p.parse_args(argv)
    try:
        execute(args)
    except (ValueError, OSError) as exc:
        p.exit(2, f"Error: {exc}\n")
    except KeyboardInterrupt:
        p.exit(130, 'Interrupted.\n')
    return 0


if __name__ == '__main__':
    raise SystemExit(main())
