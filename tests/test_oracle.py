"""The CPU oracle against fixtures generated from the reference itself."""
import json

import numpy as np
import pytest

from oracle import oracle as O
from tests.conftest import GOLDEN

TRACE_CASES = ['cloud37', 'cloud37_rev', 'trap', 'single', 'impact', 'pub4', 'cap1', 'triatomic', 'cloud300',
               'cloud300_leaf1', 'translated']


def test_sobol_scramble_and_points_bit_exact(golden):
    g = golden('sobol.npz')
    keys = sorted({k.rsplit('_', 1)[0] for k in g if k.startswith('d')})
    assert keys
    for key in keys:
        d, m, s = (int(part[1:]) for part in key.split('_'))
        sv, shift = O.sobol_scramble(d, s)
        np.testing.assert_array_equal(sv, g[key + '_sv'], err_msg=key)
        np.testing.assert_array_equal(shift, g[key + '_shift'], err_msg=key)
        np.testing.assert_array_equal(O.sobol_integers(d, m, s), g[key + '_q'], err_msg=key)
    np.testing.assert_array_equal(O.sobol_integers(7, 8, 0, scramble=False), g['plain_d7_m8_q'])


def test_impact_disk_source_matches_reference(golden):
    g = golden('source.npz')
    for name in ('pub4', 'single', 'tri'):
        e = O.external_source(g[name + '_centers'], g[name + '_radii'], int(g[name + '_m']), int(g[name + '_seed']))
        for field in ('origins', 'directions', 'weights'):
            np.testing.assert_array_equal(e[field], g[f'{name}_{field}'], err_msg=f'{name} {field}')


@pytest.mark.parametrize('kind', ['random', 'ties', 'coincident', 'single', 'translated'])
@pytest.mark.parametrize('leaf', [1, 4, 9])
def test_static_tree_arrays_bit_exact(golden, kind, leaf):
    g = golden('static_tree.npz')
    t = O.StaticTree(g[f'{kind}_centers'], g[f'{kind}_radii'], leaf)
    for key in ('lo', 'hi', 'end', 'leaf_group', 'offsets', 'ids', 'groups'):
        np.testing.assert_array_equal(getattr(t, key), g[f'{kind}_l{leaf}_{key}'], err_msg=key)


def _trace_case(g, name, threads=1):
    t = O.StaticTree(g[name + '_centers'], g[name + '_radii'], int(g[name + '_leaf']))
    cap = int(g[name + '_cap'])
    r = O.StaticTree.trace(t, g[name + '_origins'], g[name + '_directions'], g[name + '_last_atom'],
                           g[name + '_initial'], cap, True, threads)
    return t, r, cap


@pytest.mark.parametrize('name', TRACE_CASES)
def test_trace_bit_exact_against_reference_numba(golden, name):
    g = golden('trace.npz')
    t, r, cap = _trace_case(g, name)
    for field in ('positions', 'outgoing', 'escaped', 'unresolved', 'bounces'):
        np.testing.assert_array_equal(r[field], g[f'{name}_{field}'], err_msg=field)
    width = g[name + '_collider_ids'].shape[1]
    np.testing.assert_array_equal(r['collider_ids'][:, :width], g[name + '_collider_ids'])
    assert (r['collider_ids'][:, width:] == -1).all()
    assert [r['box_tests'], r['sphere_tests']] == g[name + '_counters'].tolist()
    src = dict(incoming=g[name + '_incoming'], weights=g[name + '_weights'])
    ro = O.readout(src, r, cap)
    assert ro['ehss_angstrom2'] == float(g[name + '_omega'])
    assert ro['tail_bound_angstrom2'] == float(g[name + '_tail'])
    assert ro['pa_from_same_rays_angstrom2'] == float(g[name + '_pa'])


def test_trace_thread_invariance(golden):
    g = golden('trace.npz')
    _, a, _ = _trace_case(g, 'cloud300', 1)
    _, b, _ = _trace_case(g, 'cloud300', 4)
    for field in ('positions', 'outgoing', 'escaped', 'unresolved', 'bounces', 'collider_ids'):
        np.testing.assert_array_equal(a[field], b[field])
    assert (a['box_tests'], a['sphere_tests']) == (b['box_tests'], b['sphere_tests'])


def test_known_answers():
    # trapped two-sphere path (test_ehss_reference.py:37-44)
    t = O.StaticTree(np.array([[-2., 0, 0], [2., 0, 0]]), np.ones(2))
    r = t.trace(np.zeros((1, 3)), np.array([[1., 0, 0]]), cap=7, record=True)
    assert r['unresolved'][0] and not r['escaped'][0]
    assert r['collider_ids'][0].tolist() == [1, 0, 1, 0, 1, 0, 1]
    # distance order, not atom order; miss at b = 1.01 (test_ehss_reference.py:20-24)
    assert O.entry_distance([-3., 0, 0], [1., 0, 0], [0., 0, 0], 1.) == 2.
    assert np.isinf(O.entry_distance([-3., 1.01, 0], [1., 0, 0], [0., 0, 0], 1.))
    # a 1e-10 gap is not skipped (test_ehss_reference.py:69-73)
    gap = 1e-10
    t2 = O.StaticTree(np.array([[0., 0, 0], [2. + gap, 0, 0]]), np.ones(2))
    r2 = t2.trace(np.array([[1., 0, 0]]), np.array([[1., 0, 0]]), last_atom=np.array([0]),
                  initial_bounces=np.array([1]), cap=2, record=True)
    assert r2['collider_ids'][0].tolist()[:2] == [0, 1]


def test_reference_cpp_kernel_matches_oracle(golden):
    if not O.ref_available():
        pytest.skip('reference C++ kernel not built here')
    g = golden('trace.npz')
    for name in ('cloud37', 'cloud300', 'triatomic'):
        t = O.StaticTree(g[name + '_centers'], g[name + '_radii'], int(g[name + '_leaf']))
        cap = int(g[name + '_cap'])
        for threads in (1, 3):
            r = O.ref_trace(t, g[name + '_origins'], g[name + '_directions'], cap, threads, record=True)
            for field in ('positions', 'outgoing', 'escaped', 'unresolved', 'bounces'):
                np.testing.assert_array_equal(r[field], g[f'{name}_{field}'], err_msg=f'{name} {field}')
            assert [r['box_tests'], r['sphere_tests']] == g[name + '_counters'].tolist()


def test_flat_reference_agrees(golden):
    g = golden('trace.npz'); f = golden('flat.npz')
    r = O.trace_flat(g['cloud37_centers'], g['cloud37_radii'], g['cloud37_origins'], g['cloud37_directions'], cap=64)
    np.testing.assert_array_equal(r['bounces'], g['cloud37_bounces'])
    np.testing.assert_array_equal(r['escaped'], g['cloud37_escaped'])
    np.testing.assert_allclose(r['outgoing'], f['cloud37_outgoing'], rtol=0, atol=1e-10)


@pytest.mark.parametrize('name', ['cloud37', 'cloud300', 'tri'])
def test_pa_tree_and_hits_bit_exact(golden, name):
    g = golden('pa.npz')
    t = O.PATree(g[name + '_centers'], g[name + '_radii'], 4)
    for key in ('lo', 'hi', 'end', 'first', 'count', 'ids'):
        np.testing.assert_array_equal(getattr(t, key), g[f'{name}_tree_{key}'], err_msg=key)
    hits, boxes, tests = t.query(g[name + '_origins'], g[name + '_directions'])
    np.testing.assert_array_equal(hits, g[name + '_hits'])
    assert [boxes, tests] == g[name + '_counters'].tolist()


def test_cli_readout_matches_reference_solve_frame():
    cli = json.loads((GOLDEN / 'cli.json').read_text())
    for name, case in cli.items():
        argv = case['argv']

        def flag(name, default):   # argparse keeps the last occurrence
            hits = [i for i, a in enumerate(argv) if a == name]
            return int(argv[hits[-1] + 1]) if hits else default
        rays, repeats = flag('--rays', 16384), flag('--repeats', 3)
        seed, cap = flag('--seed', 190003), flag('--max-collisions', 64)
        centers, radii = np.array(case['centers']), np.array(case['radii'])
        tree = O.StaticTree(centers, radii, 4); pat = O.PATree(centers, radii, 4)
        adaptive = '--pa-method' not in argv or argv[argv.index('--pa-method') + 1] == 'adaptive'
        omegas = []
        for k in range(repeats):
            s = (seed + 104729 * k) % 2 ** 32
            src = O.external_source(centers, radii, rays.bit_length() - 1, s)
            r = tree.trace(src['origins'], src['directions'], cap=cap)
            ro = O.readout(src, r, cap)
            run = case['runs'][k]
            assert run['seed'] == s
            for key in ('ehss_angstrom2', 'pa_from_same_rays_angstrom2', 'tail_bound_angstrom2', 'unresolved_rays',
                        'collision_histogram', 'collision_contribution_angstrom2'):
                assert ro[key] == run['ehss'][key], (name, k, key)
            if adaptive:
                ada = O.adaptive_pa(centers, radii, flag('--directions', 64), flag('--grid-size', 512), s)
                assert ada['pa_angstrom2'] == run['pa']['pa_angstrom2']
            else:
                hits, _, _ = pat.query(src['origins'], src['directions'])
                assert float(src['weights'][hits].sum()) == run['pa']['pa_angstrom2']
            omegas.append(ro['ehss_angstrom2'])
        assert O.summarize(omegas) == case['summary']['ehss_angstrom2']


@pytest.mark.parametrize('name', ['cloud37', 'cloud300', 'tri', 'single'])
def test_adaptive_pa_bit_exact(golden, name):
    g = golden('pa_adaptive.npz')
    ndir, grid, seed = (int(x) for x in g[name + '_args'])
    r = O.adaptive_pa(g[name + '_centers'], g[name + '_radii'], ndir, grid, seed)
    assert r['counts'] == g[name + '_counts'].tolist()
    assert r['spacings'] == g[name + '_spacings'].tolist()
    assert r['pa_angstrom2'] == float(g[name + '_pa'])
    # the union count from the reference's own projected coordinates
    for xy, sp, c in zip(g[name + '_xy'], g[name + '_spacings'], g[name + '_counts']):
        assert O.union_count(xy, g[name + '_radii'], np.array([-sp * grid / 2] * 2), sp, grid) == c


def test_compact_sources_and_fits_match_reference():
    """Oracle compact-boundary sources on scipy-identical Sobol points, and the
    package's host fit (CompactBoundary.fit), against the reference's own."""
    import types
    from ehss_b200.compact import CompactBoundary
    g = np.load(GOLDEN / 'compact.npz')
    for name in ('cloud37', 'cloud300', 'tri', 'line', 'single'):
        s = types.SimpleNamespace(centers=g[name + '_centers'], radii=g[name + '_radii'])
        for kind in ('sphere', 'ellipsoid', 'box'):
            b = CompactBoundary.fit(s, kind)
            np.testing.assert_array_equal(b.center, g[f'{name}_{kind}_center'])
            np.testing.assert_array_equal(b.rotation, g[f'{name}_{kind}_rotation'])
            np.testing.assert_array_equal(b.axes, g[f'{name}_{kind}_axes'])
            for m, seed in [(6, 11), (9, 190003)]:
                u = O.sobol_points(5 if kind == 'box' else 4, m, seed)
                r = O.compact_source(kind, b.center, b.rotation, b.axes, u)
                key = f'{name}_{kind}_{m}_{seed}'
                for f in ('origins', 'directions', 'weights'):
                    np.testing.assert_array_equal(r[f], g[key + '_' + f], err_msg=key + f)
