"""Generate the golden fixtures that pin the oracle and the CUDA path.

Run once, in a container that holds the SCIMMS/EHSS reference tree:

    python tests/golden/make_golden.py --reference <reference checkout>

It imports the reference's own Python package (its Numba kernels, scipy's
Sobol generator and its CLI helpers) and records their outputs on small,
seeded inputs as compressed ``.npz``/``.json`` files beside this script.
Nothing at test time reads the reference tree; the tests read these files.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent

SOBOL_CASES = [(4, 12, 0), (4, 10, 190003), (2, 6, 5), (5, 8, 77), (4, 8, 4294967295), (1, 4, 3),
               (4, 6, 104729), (4, 14, 170100001)]


def cloud(seed, n, scale, lo, hi):
    rng = np.random.default_rng(seed)
    return rng.normal(size=(n, 3)) * scale, rng.uniform(lo, hi, n)


def triatomic():
    angle = np.deg2rad(104.52)
    xyz = np.array([[0., 0., 0.], [0.9572, 0., 0.], [0.9572 * np.cos(angle), 0.9572 * np.sin(angle), 0.]])
    return xyz, np.array([1.52 + 1.4, 1.10 + 1.4, 1.10 + 1.4])


def trim_history(h, bounces):
    width = int(max(1, bounces.max(initial=0)))
    return np.ascontiguousarray(h[:, :width])


def compact_fixtures(Spheres):
    """Enclosing-boundary fits and their incidence sources (ehss_compact_source.py)."""
    from support_exchange_transport.ehss_compact_source import CompactBoundary
    comp = {}
    structures = [('cloud37', Spheres(*cloud(317, 37, 3, .7, 1.5))), ('cloud300', Spheres(*cloud(4242, 300, 6, 2.5, 3.2))),
                  ('tri', Spheres(*triatomic(), deduplicate=False)),
                  ('line', Spheres(np.array([[0., 0., 0.], [1.5, 0., 0.], [3., 0., 0.]]), np.array([1.7, 1.2, 1.7]))),
                  ('single', Spheres(np.zeros((1, 3)), np.array([3.1])))]
    for name, s in structures:
        comp[name + '_centers'] = s.centers
        comp[name + '_radii'] = s.radii
        for kind in ('sphere', 'ellipsoid', 'box'):
            b = CompactBoundary.fit(s, kind)
            comp[f'{name}_{kind}_center'] = b.center
            comp[f'{name}_{kind}_rotation'] = b.rotation
            comp[f'{name}_{kind}_axes'] = b.axes
            for m, seed in [(6, 11), (9, 190003)]:
                e = b.source(m, seed)
                key = f'{name}_{kind}_{m}_{seed}'
                comp[key + '_origins'] = e.origins
                comp[key + '_directions'] = e.directions
                comp[key + '_weights'] = e.weights
    np.savez_compressed(HERE / 'compact.npz', **comp)


# Error cases of the reference CLI: (kind, input, ...) -> the message it raises.
BAD_ARGS = [
    ['--rays', '1000'], ['--rays', '4'], ['--rays', str(2 ** 23)], ['--directions', '3'], ['--directions', '0'],
    ['--grid-size', '4'], ['--grid-size', '16384'], ['--repeats', '0'], ['--threads', '0'], ['--leaf-size', '0'],
    ['--max-collisions', '0'], ['--frame', '0'], ['--max-collisions', '100001'], ['--seed', '-1'],
    ['--seed', str(2 ** 32)], ['--probe-radius', '-0.5'], ['--probe-radius', 'nan'], ['--probe-radius', 'inf'],
    ['--rays', '1000', '--repeats', '0'], ['--repeats', '0', '--seed', '-1'],
]
BAD_XYZ = {
    'empty': '\n\n',
    'count': 'x\ncomment\nC 0 0 0\n',
    'zero': '0\ncomment\n',
    'short': '2\ncomment\nC 0 0 0\n',
    'extended': '1\nLattice="1 0 0 0 1 0 0 0 1" Properties=species:S:1\nC 0 0 0\n',
    'fields': '1\ncomment\nC 0 0\n',
    'fields5': '1\ncomment\nC 0 0 0 7\n',
    'symbol': '1\ncomment\nC1 0 0 0\n',
    'number': '1\ncomment\nC 0 zero 0\n',
    'finite': '1\ncomment\nC 0 inf 0\n',
    'second_frame': '1\na\nC 0 0 0\n2\nb\nC 0 0 0\n',
    'second_frame_row': '1\na\nC 0 0 0\n\n1\nb\nO 1 2\n',
}
GOOD_XYZ = {
    'fortran_exponent': '2\nfortran\nc 1.0D0 0 0\nO 0 2.5d-1 0\n',
    'frames_and_blanks': '\n1\na\nC 0 0 0\n\n\n2\nb b\nC 0 0 0\nN 1 0 0\n',
    'bom': '\ufeff1\nbom\nS 0 0 0\n',
}
BAD_RADII = {'list': [1, 2], 'empty': {}, 'symbol': {'C12': 1.0}, 'duplicate': {'C': 1.7, 'c': 1.6},
             'negative': {'C': -1.0}, 'bool': {'C': True}, 'string': {'C': '1.7'}, 'zero': {'N': 0}}


def cli_interface_fixtures(ccs_cli):
    """The reference CLI's messages and output layout (cli_interface.json):
    argument validation, XYZ parsing, radii JSON and frame preparation
    errors, parsed frames of accepted inputs, the default settings, and the
    key sets and CSV header of a full run's output files."""
    import tempfile
    out = dict(args={}, xyz={}, xyz_ok={}, radii={}, frames={},
               inputs=dict(xyz=BAD_XYZ, xyz_ok=GOOD_XYZ, radii=BAD_RADII))
    for argv in BAD_ARGS:
        a = ccs_cli.parser().parse_args(['x.xyz', '--output', '/nonexistent/out', *argv])
        try:
            ccs_cli.validate_args(a)
            out['args'][' '.join(argv)] = None
        except ValueError as exc:
            out['args'][' '.join(argv)] = str(exc)
    with tempfile.TemporaryDirectory() as tmp:
        tmp = Path(tmp)
        a = ccs_cli.parser().parse_args(['x.xyz', '--output', str(tmp)])
        try:
            ccs_cli.validate_args(a)
        except ValueError as exc:
            out['args']['<existing output>'] = str(exc).replace(str(tmp), '{output}')
        for name, text in BAD_XYZ.items():
            f = tmp / f'{name}.xyz'
            f.write_text(text, encoding='utf-8')
            try:
                ccs_cli.read_xyz(f)
                out['xyz'][name] = None
            except ValueError as exc:
                out['xyz'][name] = str(exc).replace(str(f), '{path}')
        for name, text in GOOD_XYZ.items():
            f = tmp / f'{name}.xyz'
            f.write_text(text, encoding='utf-8')
            out['xyz_ok'][name] = [dict(number=fr.number, comment=fr.comment, elements=list(fr.elements),
                                        coordinates=fr.coordinates.tolist()) for fr in ccs_cli.read_xyz(f)]
        for name, raw in BAD_RADII.items():
            f = tmp / f'{name}.json'
            f.write_text(json.dumps(raw), encoding='utf-8')
            try:
                ccs_cli.radius_table(f)
                out['radii'][name] = None
            except ValueError as exc:
                out['radii'][name] = str(exc)
        table = ccs_cli.radius_table(None)
        frame = ccs_cli.XYZFrame
        cases = {
            'only_h_excluded': (frame(1, 'h', ('H', 'H'), np.array([[0., 0, 0], [1, 0, 0]])), dict(exclude_hydrogen=True)),
            'unknown': (frame(2, 'u', ('C', 'Xe', 'Au'), np.array([[0., 0, 0], [1, 0, 0], [2, 0, 0]])), {}),
            'coincident': (frame(3, 'c', ('C', 'O'), np.array([[1., 2, 3], [1, 2, 3]])), {}),
            'overflow': (frame(1, 'o', ('C', 'O'), np.array([[0., 0, 0], [1e308, 0, 0]])), dict(units='nm')),
            'ok_nm': (frame(4, 'ok', ('O', 'H', 'H'), np.array([[0.1, 0, 0], [0.2, 0.05, 0], [0, 0.3, 0.01]])),
                      dict(units='nm')),
            'ok_noh': (frame(5, 'ok', ('O', 'H', 'C'), np.array([[3., 1, 0], [2, 0.5, 0], [0, 3, 0.1]])),
                       dict(exclude_hydrogen=True)),
        }
        for name, (fr, kw) in cases.items():
            try:
                spheres, info = ccs_cli.prepare_frame(fr, table, 1.4, **kw)
                out['frames'][name] = dict(centers=spheres.centers.tolist(), radii=spheres.radii.tolist(), info=info)
            except ValueError as exc:
                out['frames'][name] = str(exc)
        # a full run on a one-atom file: the output files' layout
        xyz = tmp / 'single_carbon.xyz'
        xyz.write_text('1\nsingle carbon\nC 0 0 0\n', encoding='utf-8')
        run = tmp / 'run'
        assert ccs_cli.main([str(xyz), '--rays', '1024', '--directions', '8', '--grid-size', '64', '--repeats', '2',
                             '--output', str(run)]) == 0
        payload = json.loads((run / 'results.json').read_text(encoding='utf-8'))
        rec = payload['records'][0]
        out['results'] = dict(top=sorted(payload), record=sorted(rec), summary=sorted(rec['summary']),
                              run=sorted(rec['runs'][0]), run_pa=sorted(rec['runs'][0]['pa']),
                              run_ehss=sorted(rec['runs'][0]['ehss']), timings=sorted(rec['timings']),
                              settings=payload['settings'], notes=payload['notes'],
                              radii_source=payload['radii_source'], radii=payload['atomic_radii_angstrom'])
        bvh = tmp / 'bvh'
        assert ccs_cli.main([str(xyz), '--rays', '1024', '--repeats', '1', '--pa-method', 'bvh',
                             '--output', str(bvh)]) == 0
        rec = json.loads((bvh / 'results.json').read_text(encoding='utf-8'))['records'][0]
        out['results']['run_pa_bvh'] = sorted(rec['runs'][0]['pa'])
        out['results']['run_bvh'] = sorted(rec['runs'][0])
        header = (run / 'summary.csv').read_text(encoding='utf-8-sig').splitlines()[0]
        out['results']['csv_header'] = header.split(',')
    out['default_settings'] = {k: (str(v) if isinstance(v, Path) else v)
                               for k, v in vars(ccs_cli.parser().parse_args(['x.xyz'])).items()}
    (HERE / 'cli_interface.json').write_text(json.dumps(out, indent=1, ensure_ascii=False) + '\n', encoding='utf-8')


# Reference structures (PDB-derived heavy-atom XYZ files shipped with the
# reference) traced by the reference CLI's solve_frame.
STRUCTURES = [('1AL1', [64]), ('1CLL', [64]), ('1AO6', [64]), ('1BMF', [64, 512])]


def structure_fixtures(ccs_cli, reference):
    """structures.npz: each structure's XYZ text; structures.json: the
    prepared spheres' digest and the reference's solve_frame readouts
    (EHSS + BVH PA, 16,384 rays x 3 replicates, seed 190003) at each cap."""
    import hashlib
    texts, readouts = {}, {}
    table = ccs_cli.radius_table(None)

    def strip(obj):
        if isinstance(obj, dict):
            return {k: strip(v) for k, v in obj.items() if not k.endswith('_s')}
        if isinstance(obj, list):
            return [strip(v) for v in obj]
        return obj
    for name, caps in STRUCTURES:
        path = reference / 'data' / 'inputs' / 'evaluation18' / f'{name}.xyz'
        raw = path.read_bytes()
        texts[name] = np.frombuffer(raw, dtype=np.uint8)
        frame = ccs_cli.read_xyz(path)[0]
        spheres, info = ccs_cli.prepare_frame(frame, table, 1.4)
        entry = dict(atoms=len(spheres.radii), comment=info['comment'],
                     centers_sha256=hashlib.sha256(np.ascontiguousarray(spheres.centers).tobytes()).hexdigest(),
                     radii_sha256=hashlib.sha256(np.ascontiguousarray(spheres.radii).tobytes()).hexdigest(),
                     runs={})
        for cap in caps:
            argv = ['unused.xyz', '--method', 'both', '--pa-method', 'bvh', '--rays', '16384', '--repeats', '3',
                    '--max-collisions', str(cap), '--output', '/nonexistent/x']
            out = ccs_cli.solve_frame(spheres, ccs_cli.parser().parse_args(argv), False)
            entry['runs'][str(cap)] = dict(argv=argv, summary=out['summary'], runs=strip(out['runs']))
        readouts[name] = entry
        print(name, len(spheres.radii), 'atoms', {c: r['summary']['ehss_angstrom2']['mean'] for c, r in entry['runs'].items()})
    np.savez_compressed(HERE / 'structures.npz', **texts)
    (HERE / 'structures.json').write_text(json.dumps(readouts, indent=1) + '\n')


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--reference', default=os.environ.get('EHSS_REFERENCE'),
                    help='reference checkout (default: the EHSS_REFERENCE environment variable)')
    ap.add_argument('--only', choices=['compact', 'cli'], default=None,
                    help='regenerate one fixture file only (the others stay as they are)')
    args = ap.parse_args()
    if not args.reference:
        ap.error('name the reference checkout with --reference or EHSS_REFERENCE')
    sys.path.insert(0, str(Path(args.reference) / 'src'))
    from scipy.stats import qmc
    from support_exchange_transport.inside_out_pa import Spheres, Source
    from support_exchange_transport.ehss_state import EHSSSource, external_source, reverse_pa_source
    from support_exchange_transport.ehss_static import PreparedStaticCPUEHSS
    from support_exchange_transport.ehss_reference import trace as flat_trace
    from support_exchange_transport.pa_spatial import SphereIndex
    from support_exchange_transport import ccs_cli
    if args.only == 'compact':
        compact_fixtures(Spheres)
        print('wrote compact.npz')
        return
    if args.only == 'cli':
        cli_interface_fixtures(ccs_cli)
        structure_fixtures(ccs_cli, Path(args.reference))
        print('wrote cli_interface.json, structures.json, structures.npz')
        return

    # ---- Sobol -------------------------------------------------------------
    sob = {}
    for d, m, seed in SOBOL_CASES:
        eng = qmc.Sobol(d, scramble=True, seed=seed)
        sv, shift = eng._sv.copy(), eng._shift.copy()
        pts = eng.random_base2(m)
        q = pts * 2.0 ** 30
        assert np.array_equal(q, np.round(q))
        key = f'd{d}_m{m}_s{seed}'
        sob[key + '_q'] = q.astype(np.uint32)
        sob[key + '_sv'] = sv.astype(np.uint32)
        sob[key + '_shift'] = shift.astype(np.uint32)
    sob['plain_d7_m8_q'] = (qmc.Sobol(7, scramble=False).random_base2(8) * 2.0 ** 30).astype(np.uint32)
    np.savez_compressed(HERE / 'sobol.npz', **sob)

    # ---- impact-disk sources -------------------------------------------------
    src = {}
    pub = Spheres(np.array([[0., 0., 0.], [4., 0., 0.], [1., 5., 0.], [.5, 1., 6.]]), np.full(4, 3.1),
                  deduplicate=False)
    for name, s, m, seed in [('pub4', pub, 8, 170100001), ('single', Spheres(np.zeros((1, 3)), [3.1]), 6, 91),
                             ('tri', Spheres(*triatomic(), deduplicate=False), 7, 2)]:
        e = external_source(s, m, seed)
        src[name + '_centers'] = s.centers; src[name + '_radii'] = s.radii
        src[name + '_m'] = np.array(m); src[name + '_seed'] = np.array(seed)
        src[name + '_origins'] = e.origins; src[name + '_directions'] = e.directions
        src[name + '_weights'] = e.weights
    np.savez_compressed(HERE / 'source.npz', **src)

    # ---- static BVH arrays (test_ehss_static.py kinds) ------------------------
    trees = {}
    rng = np.random.default_rng(936)
    base = rng.normal(size=(47, 3)) * 4
    radii47 = rng.uniform(.8, 2.5, 47)
    for kind in ('random', 'ties', 'coincident', 'single', 'translated'):
        xyz = base.copy()
        if kind == 'ties': xyz = np.round(xyz)
        if kind == 'coincident': xyz[:] = 0
        if kind == 'single': xyz = xyz[:1]
        if kind == 'translated': xyz = xyz + 1e6
        r = radii47[:len(xyz)]
        trees[f'{kind}_centers'] = xyz; trees[f'{kind}_radii'] = r
        for leaf in (1, 4, 9):
            t = PreparedStaticCPUEHSS(Spheres(xyz, r, deduplicate=False), leaf_size=leaf).model.tree
            for key in ('lo', 'hi', 'end', 'leaf_group', 'offsets', 'ids', 'groups'):
                trees[f'{kind}_l{leaf}_{key}'] = getattr(t, key)
    np.savez_compressed(HERE / 'static_tree.npz', **trees)

    # ---- EHSS trace cases ------------------------------------------------------
    cases = {}

    def record(name, s, source, cap, leaf=4, history=True):
        eng = PreparedStaticCPUEHSS(s, leaf_size=leaf).engine
        r = eng.trace(source, cap, record_history=history)
        cases[name + '_centers'] = s.centers; cases[name + '_radii'] = s.radii
        cases[name + '_origins'] = source.origins; cases[name + '_directions'] = source.directions
        cases[name + '_incoming'] = source.incoming; cases[name + '_weights'] = source.weights
        cases[name + '_last_atom'] = source.last_atom; cases[name + '_initial'] = source.initial_bounces
        cases[name + '_cap'] = np.array(cap); cases[name + '_leaf'] = np.array(leaf)
        cases[name + '_positions'] = r.positions; cases[name + '_outgoing'] = r.outgoing
        cases[name + '_escaped'] = r.escaped; cases[name + '_unresolved'] = r.unresolved
        cases[name + '_bounces'] = r.bounces
        if history:
            cases[name + '_collider_ids'] = trim_history(r.collider_ids, r.bounces)
        cases[name + '_counters'] = np.array([r.metrics['box_tests'], r.metrics['sphere_tests']])
        cases[name + '_omega'] = np.array(r.omega); cases[name + '_tail'] = np.array(r.tail_bound)
        cases[name + '_pa'] = np.array(r.pa)

    c37 = Spheres(*cloud(317, 37, 3, .7, 1.5))
    record('cloud37', c37, external_source(c37, 10, 321), 64)
    record('cloud37_rev', c37, reverse_pa_source(c37, 9, 321), 64)
    trap = Spheres(np.array([[-2., 0., 0.], [2., 0., 0.]]), np.ones(2))
    one = np.array([[1., 0., 0.]])
    record('trap', trap, EHSSSource(np.zeros((1, 3)), one, one, np.ones(1), np.array([-1]), np.array([0]), 'diag'), 7)
    record('single', Spheres(np.array([[2., -1., 4.]]), np.array([1.])),
           external_source(Spheres(np.array([[2., -1., 4.]]), np.array([1.])), 10, 98), 4)
    b = np.array([0., .2, .8, .999]); o = np.column_stack((np.full(4, -3.), b, np.zeros(4)))
    dd = np.tile([1., 0., 0.], (4, 1))
    record('impact', Spheres(np.zeros((1, 3)), np.ones(1)),
           EHSSSource(o, dd, dd, np.ones(4), np.full(4, -1), np.zeros(4), 'controlled'), 64)
    record('pub4', pub, external_source(pub, 10, 170100001), 256)
    c23 = Spheres(*cloud(667, 23, 2, 1.2, 1.2))
    record('cap1', c23, external_source(c23, 10, 190003), 1)
    tri = Spheres(*triatomic(), deduplicate=False)
    record('triatomic', tri, external_source(tri, 12, 0), 64)
    g300 = Spheres(*cloud(4242, 300, 6, 2.5, 3.2))
    record('cloud300', g300, external_source(g300, 11, 7), 64)
    record('cloud300_leaf1', g300, external_source(g300, 9, 8), 64, leaf=1)
    tr = Spheres(base + 1e6, radii47, deduplicate=False)
    record('translated', tr, external_source(tr, 8, 572), 64)
    np.savez_compressed(HERE / 'trace.npz', **cases)

    # ---- independent flat tracer on one case ---------------------------------
    flat = {}
    src37 = external_source(c37, 10, 321)
    fr = flat_trace(c37, src37, 64)
    flat['cloud37_outgoing'] = fr.outgoing; flat['cloud37_bounces'] = fr.bounces
    flat['cloud37_escaped'] = fr.escaped
    np.savez_compressed(HERE / 'flat.npz', **flat)

    # ---- BVH any-hit PA --------------------------------------------------------
    pa = {}
    for name, s, m, seed in [('cloud37', c37, 10, 321), ('cloud300', g300, 11, 7), ('tri', tri, 10, 3)]:
        e = external_source(s, m, seed)
        idx = SphereIndex(s, leaf_size=4)
        hits, boxes, tests = idx.query(Source(e.origins, e.directions, e.last_atom, float(e.weights.sum())))
        pa[name + '_centers'] = s.centers; pa[name + '_radii'] = s.radii
        pa[name + '_origins'] = e.origins; pa[name + '_directions'] = e.directions
        pa[name + '_weights'] = e.weights
        pa[name + '_hits'] = hits; pa[name + '_counters'] = np.array([boxes, tests])
        for key in ('lo', 'hi', 'end', 'first', 'count', 'ids'):
            pa[f'{name}_tree_{key}'] = getattr(idx.tree, key)
    np.savez_compressed(HERE / 'pa.npz', **pa)

    # ---- adaptive finite-grid PA ---------------------------------------------------
    from support_exchange_transport.pa_walsh_geometry import project_grid
    from support_exchange_transport.pa_sparse_blocks import block_disks, block_count
    from support_exchange_transport.inside_out_pa import unit_sphere
    ada = {}
    for name, s, ndir, grid, seed in [('cloud37', c37, 8, 128, 5), ('cloud300', g300, 16, 256, 190003),
                                      ('tri', tri, 8, 512, 0), ('single', Spheres(np.zeros((1, 3)), [3.1]), 4, 64, 2)]:
        ds = unit_sphere(qmc.Sobol(2, scramble=True, seed=seed).random_base2(ndir.bit_length() - 1))
        counts, spacings, xys = [], [], []
        for d in ds:
            xy, lower, spacing, *_ = project_grid(s, d, grid)
            full, partial, _ = block_disks(xy, s.radii, lower, spacing, grid)
            counts.append(int(block_count(full, partial))); spacings.append(spacing); xys.append(xy)
        out = ccs_cli.adaptive_pa(s, ndir, grid, seed)
        ada[name + '_centers'] = s.centers; ada[name + '_radii'] = s.radii
        ada[name + '_args'] = np.array([ndir, grid, seed])
        ada[name + '_counts'] = np.array(counts); ada[name + '_spacings'] = np.array(spacings)
        ada[name + '_xy'] = np.array(xys); ada[name + '_pa'] = np.array(out['pa_angstrom2'])
    np.savez_compressed(HERE / 'pa_adaptive.npz', **ada)

    # ---- CLI solve_frame readouts ------------------------------------------------
    cli = {}

    def strip(obj):
        if isinstance(obj, dict):
            return {k: strip(v) for k, v in obj.items() if not k.endswith('_s')}
        if isinstance(obj, list):
            return [strip(v) for v in obj]
        return obj

    for name, s, extra in [
            ('single', Spheres(np.zeros((1, 3)), np.array([3.1])), ['--pa-method', 'bvh']),
            ('cap1', c23, ['--pa-method', 'bvh', '--repeats', '1', '--max-collisions', '1']),
            ('tri', tri, ['--pa-method', 'bvh', '--rays', '4096', '--repeats', '3', '--seed', '0']),
            ('tri_adaptive', tri, ['--directions', '16', '--grid-size', '256', '--repeats', '2'])]:
        argv = ['unused.xyz', '--rays', '1024', '--repeats', '2', '--output', '/nonexistent/x', *extra]
        a = ccs_cli.parser().parse_args(argv)
        out = ccs_cli.solve_frame(s, a, False)
        cli[name] = dict(argv=argv, centers=s.centers.tolist(), radii=s.radii.tolist(),
                         summary=out['summary'], runs=strip(out['runs']))
    (HERE / 'cli.json').write_text(json.dumps(cli, indent=1) + '\n')
    cli_interface_fixtures(ccs_cli)
    structure_fixtures(ccs_cli, Path(args.reference))
    compact_fixtures(Spheres)
    print('wrote', sorted(p.name for p in HERE.glob('*.npz')), 'cli.json')


if __name__ == '__main__':
    main()
