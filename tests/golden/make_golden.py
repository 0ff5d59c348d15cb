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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--reference', default=os.environ.get('EHSS_REFERENCE'),
                    help='reference checkout (default: the EHSS_REFERENCE environment variable)')
    ap.add_argument('--only', choices=['compact'], default=None,
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
    compact_fixtures(Spheres)
    print('wrote', sorted(p.name for p in HERE.glob('*.npz')), 'cli.json')


if __name__ == '__main__':
    main()
