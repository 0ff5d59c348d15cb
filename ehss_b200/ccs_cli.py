"""The ccs.py calculation surface on the B200 path.

The command line, its validation messages, the accepted XYZ dialect, the
exit codes and the two output files (``summary.csv``, ``results.json``) are
the reference CLI's interface (src/support_exchange_transport/ccs_cli.py:
flags :235-257, validation :260-271, XYZ rules :48-83, radii :86-101, frame
preparation :104-126, outputs :311-343, exit codes :346-354); the code
behind them is this module's own.

What runs is different.  Every frame of a run (one, or all of them with
``--all-frames`` and several files) is prepared on the host, then the group
is built as device scenes in one batched pass and all replicate blocks of
all frames are traced in one persistent launch (Sobol -> impact disk -> EHSS
trace / BVH PA -> integer reduction).  A frame's numbers do not depend on
which other frames share the launch.  ``--threads`` is validated and
recorded (the GPU replaces worker threads).  ``--leaf-size`` is validated
and recorded as the reference's grouping parameter; results do not depend
on the tree, and the device LBVH uses its own tuned leaf bound.
"""
from __future__ import annotations

import argparse
import csv
import glob
import hashlib
import json
import math
import platform
import sys
import time
from collections import Counter
from dataclasses import dataclass
from datetime import datetime, timezone
from pathlib import Path

import numpy as np

VERSION = "0.1.0"
# van der Waals radii in angstrom: Mantina et al. 2009, Table 12, with H = 1.10
# (the reference CLI's table, ccs_cli.py:29-31)
VDW_RADII = {"H": 1.10, "He": 1.40, "C": 1.70, "N": 1.55, "O": 1.52, "F": 1.47, "Si": 2.10, "P": 1.80,
             "S": 1.80, "Cl": 1.75, "Se": 1.90, "Br": 1.83, "I": 1.98}
RADII_SOURCE = 'Mantina et al. 2009 Table 12, subset; DOI 10.1021/jp8111556; user overrides recorded in table'
NOTES = (
    'Static elastic hard-sphere model; atomic VDW radius + probe radius. Not TM or fitted IMoS/EHSSrot parameters.',
    'XYZ atoms, device LBVH; no inferred bonds/residues; no support response reuse.',
    'Independent Sobol scrambles across replicates. SD/SEM measure replicate variation, not total error or a '
    'guaranteed confidence interval.',
    'Adaptive PA has finite-grid and directional error; replicate SD does not estimate grid bias.',
    'EHSS sampled interval covers omitted cap survivors only, not sampling error or physical model error.',
    'Warmup/import/IO excluded from per-frame compute timing; setup is once per frame, shared across replicates.',
    'For both + BVH PA, the impact rays are the same for EHSS and PA.',
    'EHSS paths use FP32 traversal with FP64 re-test of every candidate; per-ray outcomes equal the FP64 path.',
    'Impact rays are generated inside the trace kernel: impact_source_s is 0 and their time is part of query_s. '
    'box_tests/sphere_tests count the device LBVH tests (4 child boxes per node visit).',
    'Frames of one run are built and traced together on the device; query_s and setup times are the group\'s, '
    'divided evenly over its frames and replicates.',
)


# ----------------------------------------------------------------------------
# XYZ input
# ----------------------------------------------------------------------------
@dataclass
class XYZFrame:
    number: int
    comment: str
    elements: tuple
    coordinates: np.ndarray


def element_symbol(value):
    """One- or two-letter ASCII element symbol, capitalised ('cl' -> 'Cl')."""
    if not (isinstance(value, str) and 1 <= len(value) <= 2 and value.isascii() and value.isalpha()):
        raise ValueError(f"Expected an element symbol, got {value!r}")
    return value[:1].upper() + value[1:].lower()


_FORTRAN_EXPONENT = str.maketrans({'D': 'E', 'd': 'e'})
_EXTENDED_MARKERS = ('Lattice=', 'Properties=')


class _XYZCursor:
    """Walks the lines of one XYZ file frame by frame.  Frames are parsed in
    file order, so the error reported is the first malformed line."""

    def __init__(self, path):
        self.path = path
        self.lines = Path(path).read_text(encoding='utf-8-sig').splitlines()
        self.at = 0

    def fail(self, index, what):
        raise ValueError(f"{self.path}:{index + 1}: {what}")

    def frames(self):
        number = 0
        while True:
            while self.at < len(self.lines) and not self.lines[self.at].strip():
                self.at += 1                     # blank lines between frames
            if self.at == len(self.lines):
                return
            number += 1
            yield self._frame(number)

    def _count(self, index):
        token = self.lines[index].strip()
        if not (token.isascii() and token.isdigit() and token[0] != '0'):
            self.fail(index, 'expected a positive atom count')
        return int(token)

    def _frame(self, number):
        head = self.at
        count = self._count(head)
        if head + 1 + count >= len(self.lines):
            self.fail(head, f'incomplete XYZ frame (comment and {count} atom rows required)')
        comment = self.lines[head + 1]
        if any(marker in comment for marker in _EXTENDED_MARKERS):
            self.fail(head + 1, 'extended/periodic XYZ is not supported; export a standard isolated molecule')
        first = head + 2
        atoms = [self._atom(index) for index in range(first, first + count)]
        self.at = first + count
        return XYZFrame(number, comment, tuple(a[0] for a in atoms), np.array([a[1] for a in atoms]))

    def _atom(self, index):
        tokens = self.lines[index].split()
        if len(tokens) != 4:
            self.fail(index, "expected exactly 'Element x y z'")
        try:
            symbol = element_symbol(tokens[0])
            xyz = [float(t.translate(_FORTRAN_EXPONENT)) for t in tokens[1:]]
        except ValueError as exc:
            raise ValueError(f"{self.path}:{index + 1}: invalid element or coordinates") from exc
        if not all(math.isfinite(v) for v in xyz):
            self.fail(index, 'coordinates must be finite')
        return symbol, xyz


def read_xyz(path):
    """Every frame of a standard XYZ file (a malformed later frame is an error,
    not ignored).  Fortran exponents (1.0D0) are accepted; extended XYZ is not."""
    frames = list(_XYZCursor(path).frames())
    if not frames:
        raise ValueError(f"{path}: no XYZ frames")
    return frames


def _positive_finite(value):
    return not isinstance(value, bool) and isinstance(value, (int, float)) and math.isfinite(value) and value > 0


def radius_table(path=None):
    """The VDW table, with the overrides/additions of a radii JSON object."""
    table = dict(VDW_RADII)
    if not path:
        return table
    overrides = json.loads(Path(path).read_text(encoding='utf-8-sig'))
    if not isinstance(overrides, dict) or not overrides:
        raise ValueError("Radii JSON must be a nonempty object: {\"C\": 1.70, ...}")
    given = {}
    for key, value in overrides.items():
        symbol = element_symbol(key)
        if symbol in given:
            raise ValueError(f"Duplicate normalized radius key: {symbol}")
        if not _positive_finite(value):
            raise ValueError(f"Radius for {symbol} must be a positive finite number in angstrom")
        given[symbol] = float(value)
    table.update(given)
    return table


_UNIT_SCALE = {'angstrom': 1.0, 'nm': 10.0}


def prepare_frame(frame, radii, probe_radius, units="angstrom", exclude_hydrogen=False):
    """Selected atoms in angstrom, recentred on their mean, with effective
    radius = VDW radius + probe; returns (Spheres, record fields)."""
    from .state import Spheres
    rows = [k for k, element in enumerate(frame.elements) if not (exclude_hydrogen and element == 'H')]
    if not rows:
        raise ValueError(f"Frame {frame.number}: atom selection is empty")
    elements = [frame.elements[k] for k in rows]
    missing = sorted({e for e in elements if e not in radii})
    if missing:
        raise ValueError(f"Frame {frame.number}: no radius for {', '.join(missing)}; supply --radii-json")
    with np.errstate(over='ignore'):
        xyz = frame.coordinates[rows] * _UNIT_SCALE[units]
    if not np.isfinite(xyz).all():
        raise ValueError("Coordinates overflow after unit conversion")
    if len(np.unique(xyz, axis=0)) != len(xyz):
        raise ValueError(f"Frame {frame.number}: coincident selected atom centers; check duplicate atoms")
    # the mean taken relative to the first atom keeps offset geometries precise
    anchor = xyz[0]
    offset = anchor + np.mean(xyz - anchor, axis=0)
    by_element = {e: radii[e] + probe_radius for e in sorted(set(elements))}
    spheres = Spheres(xyz - offset, np.array([by_element[e] for e in elements]), deduplicate=False)
    fields = dict(frame=frame.number, comment=frame.comment, input_atoms=len(frame.elements),
                  selected_atoms=len(rows), selected_atom_rows_1based=[k + 1 for k in rows],
                  element_counts=dict(Counter(elements)), recenter_offset_angstrom=offset.tolist(),
                  effective_radii_angstrom=by_element)
    return spheres, fields


# ----------------------------------------------------------------------------
# command line
# ----------------------------------------------------------------------------
def parser():
    p = argparse.ArgumentParser(description="PA/EHSS for isolated molecules in standard XYZ files (results in A^2).")
    add = p.add_argument
    add('xyz', nargs='+', help='XYZ paths; quoted wildcard patterns also work on Windows')
    add('--version', action='version', version='ccs-xyz ' + VERSION)
    add('--method', choices=['pa', 'ehss', 'both'], default='both')
    add('--pa-method', choices=['adaptive', 'bvh'], default='adaptive')
    add('--rays', type=int, default=16384, help='EHSS/BVH PA rays per replicate, power of two (default: 16384)')
    add('--directions', type=int, default=64, help='Adaptive PA directions per replicate, power of two (default: 64)')
    add('--grid-size', type=int, default=512, help='Adaptive PA square midpoint grid, power of two (default: 512)')
    add('--repeats', type=int, default=3, help='Independent scrambled Sobol replicates (default: 3)')
    add('--seed', type=int, default=190003)
    add('--threads', type=int, default=1, help='Accepted and recorded; the GPU replaces CPU threads')
    add('--leaf-size', type=int, default=4,
        help='Maximum spatial group size for XYZ BVH (default: 4); recorded, results do not depend on it')
    add('--max-collisions', type=int, default=64)
    add('--probe-radius', type=float, default=1.4, help='Added probe radius in angstrom (default: 1.4, He scenario)')
    add('--radii-json', type=Path, help='Overrides/additions to atomic VDW radii in angstrom, never effective radii')
    add('--units', choices=['angstrom', 'nm'], default='angstrom', help='Input coordinate units only')
    add('--exclude-hydrogen', action='store_true', help='Explicitly omit H; default includes every supplied atom')
    one_or_all = p.add_mutually_exclusive_group()
    one_or_all.add_argument('--frame', type=int, default=1, help='1-based frame selection (default: first frame)')
    one_or_all.add_argument('--all-frames', action='store_true',
                            help='Calculate every frame independently, no MD cache reuse')
    add('--output', type=Path, default=Path('ccs_results'), help='New result directory; existing directory is preserved')
    return p


def _flag(name):
    return '--' + name.replace('_', '-')


def _power_of_two_in(low, high):
    return lambda v: low <= v <= high and v & (v - 1) == 0


# Checked in this order; the first rule that fails is reported.
_RULES = (
    [(name, _power_of_two_in(low, high), f"{_flag(name)} must be a power of two in {low}..{high}")
     for name, low, high in (('rays', 8, 1 << 22), ('directions', 1, 1 << 16), ('grid_size', 8, 8192))]
    + [(name, lambda v: v >= 1, f"{_flag(name)} must be positive")
       for name in ('repeats', 'threads', 'leaf_size', 'max_collisions', 'frame')]
    + [('max_collisions', lambda v: v <= 100000, '--max-collisions must be <= 100000'),
       ('seed', lambda v: 0 <= v < 1 << 32, '--seed must be in 0..4294967295'),
       ('probe_radius', lambda v: math.isfinite(v) and v >= 0, '--probe-radius must be finite and nonnegative')]
)


def validate_args(args):
    for name, ok, message in _RULES:
        if not ok(getattr(args, name)):
            raise ValueError(message)
    if args.output.exists():
        raise ValueError(f"Output already exists: {args.output}; choose a new --output directory")


def _input_files(patterns):
    """Each named file, or each file a wildcard pattern matches, once."""
    seen = set()
    for pattern in patterns:
        names = [pattern] if Path(pattern).is_file() else sorted(glob.glob(pattern))
        if not names:
            raise ValueError(f"No XYZ files match: {pattern}")
        for name in names:
            path = Path(name).resolve()
            if path not in seen:
                seen.add(path)
                yield path


def load_frames(args, table):
    """Every selected frame of every input file, prepared: [(Spheres, record fields)]."""
    prepared = []
    for path in _input_files(args.xyz):
        frames = read_xyz(path)
        if args.all_frames:
            chosen = frames
        else:
            if args.frame > len(frames):
                raise ValueError(f"{path.name}: --frame {args.frame} exceeds {len(frames)} frames")
            chosen = [frames[args.frame - 1]]
            if len(frames) > 1:
                print(f"{path.name}: using frame {args.frame}/{len(frames)}; use --all-frames for all.",
                      file=sys.stderr)
        source = dict(input_file=str(path), input_sha256=hashlib.sha256(path.read_bytes()).hexdigest(),
                      total_frames=len(frames))
        for frame in chosen:
            spheres, fields = prepare_frame(frame, table, args.probe_radius, args.units, args.exclude_hydrogen)
            prepared.append((spheres, dict(source, **fields)))
    return prepared


# ----------------------------------------------------------------------------
# device solve
# ----------------------------------------------------------------------------
def summarize(values):
    """Mean, sample SD (ddof 1), SEM and count of replicate values."""
    a = np.asarray(values, dtype=float)
    sd = float(a.std(ddof=1)) if len(a) > 1 else None
    return dict(mean=float(a.mean()), sd=sd, sem=None if sd is None else sd / math.sqrt(len(a)), replicates=len(a))


# frames traced together: one batched build and one persistent launch per group
GROUP_ATOMS = 2_000_000
GROUP_FRAMES = 1024


def _groups(spheres_list):
    group, atoms = [], 0
    for k, s in enumerate(spheres_list):
        n = len(s.radii)
        if group and (len(group) == GROUP_FRAMES or atoms + n > GROUP_ATOMS):
            yield group
            group, atoms = [], 0
        group.append(k)
        atoms += n
    if group:
        yield group


class _Modes:
    def __init__(self, args):
        self.ehss = args.method in ('ehss', 'both')
        self.pa = args.method in ('pa', 'both')
        self.bvh_pa = self.pa and args.pa_method == 'bvh'
        self.adaptive_pa = self.pa and args.pa_method == 'adaptive'


def _ehss_row(block, query_s, readout_s):
    omega, tail = block['ehss_angstrom2'], block['tail_bound_angstrom2']
    return dict(ehss_angstrom2=omega, pa_from_same_rays_angstrom2=block['pa_from_same_rays_angstrom2'],
                tail_bound_angstrom2=tail, sampled_interval_angstrom2=[omega, omega + tail],
                unresolved_rays=block['unresolved_rays'], query_s=query_s,
                collision_histogram=block['collision_histogram'],
                collision_contribution_angstrom2=block['collision_contribution_angstrom2'],
                box_tests=int(block['box_tests']), sphere_tests=int(block['sphere_tests']), readout_s=readout_s,
                grazing_queries=block['grazing_queries'], fp64_fallback_queries=block['fp64_fallback_queries'])


def _bvh_pa_row(block, query_s, readout_s):
    return dict(pa_angstrom2=block['pa_angstrom2'], query_s=query_s, readout_s=readout_s,
                box_tests=int(block['box_tests']), sphere_tests=int(block['sphere_tests']))


def _trace_group(group, args, modes):
    """One batched build and one persistent launch for the frames of ``group``.
    EHSS and BVH-PA replicates are separate blocks over the same rays (same
    structure, seed and count), so each block's test counters are its own.
    Returns per frame: replicate rows, setup seconds, query seconds."""
    import torch
    from . import _lib
    from .batch import BatchScenes
    from .blocks import BlockJob, BlockPlan, seed_schedule
    seeds = seed_schedule(args.seed, args.repeats)
    # every block ray starts on the impact disk, so buried atoms leave the trees (exterior scenes)
    scenes = BatchScenes([(s.centers, s.radii) for s in group], device=None, exterior=True)
    e_build, e_built, e_traced = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    e_build.record()
    scenes.build()
    e_built.record()
    rows = [[dict(repeat=k + 1, seed=seed) for k, seed in enumerate(seeds)] for _ in group]
    kinds = [kind for kind, on in (('ehss', modes.ehss), ('pa', modes.bvh_pa)) if on]
    blocks = {}
    if kinds:
        log2 = args.rays.bit_length() - 1
        jobs = [BlockJob(scene, log2, seed, cap=args.max_collisions, precision=_lib.PREC_FP32, ehss=kind == 'ehss',
                         pa=kind == 'pa', tag=(f, k, kind))
                for f, scene in enumerate(scenes.scenes) for k, seed in enumerate(seeds) for kind in kinds]
        plan = BlockPlan(jobs, launch=dict(count_tests=True))
        plan.enqueue()
        e_traced.record()
        tick = time.perf_counter()
        blocks = {job.tag: res for job, res in zip(jobs, plan.collect())}
        readout_s = (time.perf_counter() - tick) / len(jobs)
        query_s = e_built.elapsed_time(e_traced) * 1e-3 / (len(group) * len(seeds))
    else:
        torch.cuda.synchronize()
    setup_s = e_build.elapsed_time(e_built) * 1e-3 / len(group)
    for f, spheres in enumerate(group):
        for k, row in enumerate(rows[f]):
            if modes.adaptive_pa:
                from .adaptive_pa import adaptive_pa
                row['pa'] = adaptive_pa(spheres, args.directions, args.grid_size, row['seed'], scene=scenes.scenes[f])
            if kinds:
                row['impact_source_s'] = 0.0
            if modes.bvh_pa:
                row['pa'] = _bvh_pa_row(blocks[(f, k, 'pa')], query_s, readout_s)
            if modes.ehss:
                row['ehss'] = _ehss_row(blocks[(f, k, 'ehss')], query_s, readout_s)
    return rows, setup_s


def _frame_summary(rows, modes):
    summary = {}
    if modes.pa:
        summary['pa_angstrom2'] = summarize([r['pa']['pa_angstrom2'] for r in rows])
    if modes.ehss:
        summary['ehss_angstrom2'] = summarize([r['ehss']['ehss_angstrom2'] for r in rows])
        summary['ehss_tail_bound_mean_angstrom2'] = float(np.mean([r['ehss']['tail_bound_angstrom2'] for r in rows]))
        summary['ehss_unresolved_rays_total'] = sum(r['ehss']['unresolved_rays'] for r in rows)
    return summary


def _warn_unresolved(rows):
    for r in rows:
        e = r.get('ehss')
        if e and e['unresolved_rays']:
            print(f"  WARNING: {e['unresolved_rays']} unresolved rays; omitted contribution <= "
                  f"{e['tail_bound_angstrom2']:.6g} A^2. Increase --max-collisions.", file=sys.stderr)


def solve_frames(spheres_list, args, progress=True):
    """Results of many prepared frames: summary, replicate rows and timings
    per frame, each frame's numbers the same as it would get alone."""
    modes = _Modes(args)
    results = []
    for group in _groups(spheres_list):
        start = time.perf_counter()
        frames = [spheres_list[k] for k in group]
        rows, setup_s = _trace_group(frames, args, modes)
        per_frame = (time.perf_counter() - start) / len(frames)
        for r in rows:
            if progress:
                _warn_unresolved(r)
            results.append(dict(summary=_frame_summary(r, modes), runs=r,
                                timings=dict(ehss_setup_s=setup_s if modes.ehss else 0.,
                                             pa_setup_s=setup_s if modes.pa else 0.,
                                             all_replicates_with_setup_s=per_frame, batched_frames=len(frames))))
        if progress and len(frames) > 1:
            print(f"  traced {len(frames)} frame(s) in one batch", file=sys.stderr, flush=True)
    return results


def solve_frame(spheres, args, progress=True):
    """One prepared frame (the reference's solve_frame contract)."""
    return solve_frames([spheres], args, progress)[0]


# ----------------------------------------------------------------------------
# outputs
# ----------------------------------------------------------------------------
def _summary_value(record, quantity, stat):
    return record['summary'].get(quantity, {}).get(stat)


# summary.csv: one row per frame, columns in this order
SUMMARY_COLUMNS = (
    ('input_file', lambda r: r['input_file']),
    ('frame', lambda r: r['frame']),
    ('atoms', lambda r: r['selected_atoms']),
    ('pa_mean_A2', lambda r: _summary_value(r, 'pa_angstrom2', 'mean')),
    ('pa_sd_A2', lambda r: _summary_value(r, 'pa_angstrom2', 'sd')),
    ('ehss_mean_A2', lambda r: _summary_value(r, 'ehss_angstrom2', 'mean')),
    ('ehss_sd_A2', lambda r: _summary_value(r, 'ehss_angstrom2', 'sd')),
    ('ehss_tail_bound_mean_A2', lambda r: r['summary'].get('ehss_tail_bound_mean_angstrom2')),
    ('unresolved_rays_total', lambda r: r['summary'].get('ehss_unresolved_rays_total')),
    ('compute_all_replicates_s', lambda r: r['timings']['all_replicates_with_setup_s']),
)


def write_summary_csv(path, records):
    with Path(path).open('w', newline='', encoding='utf-8-sig') as f:
        out = csv.writer(f)
        out.writerow([name for name, _ in SUMMARY_COLUMNS])
        for r in records:
            out.writerow(['' if v is None else v for v in (value(r) for _, value in SUMMARY_COLUMNS)])


def environment():
    import torch
    env = dict(python=platform.python_version(), platform=platform.platform(), numpy=np.__version__,
               torch=torch.__version__, cuda=torch.version.cuda)
    if torch.cuda.is_available():
        env['gpu'] = torch.cuda.get_device_name()
    return env


def results_payload(args, table, records, warmup_s, started):
    settings = {k: str(v) if isinstance(v, Path) else v for k, v in vars(args).items()}
    return dict(schema_version=1, tool='ccs-xyz', version=VERSION, backend='ehss_b200 (B200, sm_100a)',
                created_utc=datetime.now(timezone.utc).isoformat(), settings=settings, atomic_radii_angstrom=table,
                radii_source=RADII_SOURCE, environment=environment(), warmup_s=warmup_s,
                elapsed_before_output_s=time.perf_counter() - started, notes=list(NOTES), records=records)


def _report(record):
    for quantity in ('pa_angstrom2', 'ehss_angstrom2'):
        v = record['summary'].get(quantity)
        if v is not None:
            sd = 'n/a' if v['sd'] is None else f"{v['sd']:.6f}"
            print(f"  {quantity.split('_')[0].upper()}: {v['mean']:.6f} A^2 (replicate SD {sd})")
    print(f"  Compute: {record['timings']['all_replicates_with_setup_s']:.4f} s "
          "(setup + all replicates; warmup excluded)")


def execute(args):
    validate_args(args)
    from .device import require_cuda
    from .state import Spheres
    started = time.perf_counter()
    table = radius_table(args.radii_json)
    prepared = load_frames(args, table)      # input errors are reported before any device work
    require_cuda()
    print(f"Validated {len(prepared)} frame(s). Preparing the device kernels...", file=sys.stderr, flush=True)
    # context creation and module loading stay out of the per-frame timings
    tick = time.perf_counter()
    tiny = argparse.Namespace(**dict(vars(args), rays=8, directions=1, grid_size=8, repeats=1))
    solve_frame(Spheres(np.array([[0., 0., 0.], [2., 0., 0.]]), np.array([1., 1.])), tiny, progress=False)
    warmup_s = time.perf_counter() - tick
    solved = solve_frames([s for s, _ in prepared], args)
    records = []
    for (spheres, fields), result in zip(prepared, solved):
        print(f"{Path(fields['input_file']).name}, frame {fields['frame']}, {fields['selected_atoms']} atoms",
              file=sys.stderr, flush=True)
        records.append(dict(fields, **result))
        _report(records[-1])
    payload = results_payload(args, table, records, warmup_s, started)
    # the output directory is made only after every frame has succeeded, and never reused
    args.output.mkdir(parents=True, exist_ok=False)
    (args.output / 'results.json').write_text(json.dumps(payload, ensure_ascii=False, indent=2, allow_nan=False) + '\n',
                                              encoding='utf-8')
    write_summary_csv(args.output / 'summary.csv', records)
    for name in ('summary.csv', 'results.json'):
        print(f"Saved {args.output.resolve() / name}")
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
