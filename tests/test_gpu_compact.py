"""Compact-boundary incidence on the device (CompactBoundary, ehss_compact_source.py)
against the reference's own rays (golden fixtures) and the oracle on identical
Sobol points, and traced end to end through the prepared engine."""
import types

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

NAMES = ['cloud37', 'cloud300', 'tri', 'line', 'single']
KINDS = ['sphere', 'ellipsoid', 'box']
# Device cos/sin are within 2 ulp of numpy's: directions agree to ~4e-16, origins
# (|o| ~ structure size) to ~1e-14 A.  The box rotation is the identity, so its
# face choice and face coordinates are exact; a general ellipsoid rotation adds
# one rounding of the 3x3 products.
RTOL, ATOL = 1e-13, 1e-12


@pytest.fixture(scope='module')
def eb():
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    import ehss_b200
    return ehss_b200


@pytest.fixture(scope='module')
def golden():
    from pathlib import Path
    return np.load(Path(__file__).parent / 'golden' / 'compact.npz')


@pytest.mark.parametrize('kind', KINDS)
@pytest.mark.parametrize('name', NAMES)
def test_device_rays_match_reference_rays(eb, golden, name, kind):
    s = types.SimpleNamespace(centers=golden[name + '_centers'], radii=golden[name + '_radii'])
    b = eb.CompactBoundary.fit(s, kind)
    for m, seed in [(6, 11), (9, 190003)]:
        src = b.source(m, seed)
        key = f'{name}_{kind}_{m}_{seed}'
        np.testing.assert_allclose(src.directions, golden[key + '_directions'], rtol=0, atol=4e-15)
        np.testing.assert_allclose(src.origins, golden[key + '_origins'], rtol=RTOL, atol=ATOL)
        np.testing.assert_allclose(src.weights, golden[key + '_weights'], rtol=RTOL, atol=0)
        assert np.all(src.last_atom == -1) and np.all(src.initial_bounces == 0)


@pytest.mark.parametrize('kind', KINDS)
def test_device_rays_match_oracle_on_device_sobol_points(eb, kind):
    from ehss_b200 import workloads as W
    c, r, _ = W.globule(800, 21)
    s = types.SimpleNamespace(centers=c, radii=r)
    b = eb.CompactBoundary.fit(s, kind)
    o, d, w = (x.cpu().numpy() for x in b.device_rays(12, 4242))
    u = O.sobol_points(5 if kind == 'box' else 4, 12, 4242)
    ref = O.compact_source(kind, b.center, b.rotation, b.axes, u)
    np.testing.assert_allclose(d, ref['directions'], rtol=0, atol=4e-15)
    np.testing.assert_allclose(o, ref['origins'], rtol=RTOL, atol=ATOL)
    np.testing.assert_allclose(w, ref['weights'], rtol=RTOL, atol=0)
    # the rays start outside every sphere
    dist = np.linalg.norm(o[:, None, :] - c[None, ::40, :], axis=2)
    assert np.all(dist >= r[None, ::40] - 1e-9)
    # a partial range is the same rays
    o2, d2, w2 = (x.cpu().numpy() for x in b.device_rays(12, 4242, first=1000, n=77))
    np.testing.assert_array_equal(o2, o[1000:1077])
    np.testing.assert_array_equal(w2, w[1000:1077])


@pytest.mark.parametrize('kind', ['box', 'ellipsoid'])
def test_compact_source_traced_through_the_prepared_engine(eb, kind):
    from ehss_b200 import workloads as W
    c, r, _ = W.globule(600, 5)
    s = eb.Spheres(c, r, deduplicate=False)
    prep = eb.PreparedStaticGPUEHSS(s, boundary=kind)
    assert prep.boundary.kind == kind
    src = prep.boundary.source(12, 190003)
    got = prep.engine.trace(src, 64, record_history=True)
    ref = O.StaticTree(c, r, 4).trace(src.origins, src.directions, cap=64, record=True, threads=4)
    for field in ('positions', 'outgoing', 'escaped', 'unresolved', 'bounces', 'collider_ids'):
        np.testing.assert_array_equal(getattr(got, field), ref[field], err_msg=field)
    ro = O.readout(dict(incoming=src.incoming, weights=src.weights), ref, 64)
    assert got.omega == pytest.approx(ro['ehss_angstrom2'], rel=1e-12)
    # the three boundaries estimate the same cross section (different incidence, same physics)
    disk = eb.PreparedStaticGPUEHSS(s).engine.trace(eb.external_source(s, 14, 7, scene=prep.scene), 64)
    assert abs(got.omega - disk.omega) <= 0.03 * disk.omega


def test_boundary_validation(eb):
    s = types.SimpleNamespace(centers=np.zeros((2, 3)) + [[0, 0, 0], [1, 0, 0]], radii=np.ones(2))
    with pytest.raises(ValueError):
        eb.CompactBoundary.fit(s, 'cube')
    b = eb.CompactBoundary.fit(s, 'box')
    with pytest.raises(ValueError):
        b.source(-1, 0)
    with pytest.raises(ValueError):
        b.source(3, -5)


@pytest.mark.parametrize('kind', ['box', 'ellipsoid', 'sphere'])
def test_fused_boundary_blocks_match_explicit_trace(eb, kind):
    """Boundary rays in the fused kernel (EHSS_BLOCK_RAYS, weighted fixed-point
    sums) against the same rays traced one by one and read out on the host."""
    from ehss_b200 import workloads as W
    from ehss_b200.batch import BatchCCS
    structures = [W.globule(n, 60 + n)[:2] for n in (40, 900)]
    bc = BatchCCS(structures, 12, [7, 8], repeats=2, cap=32, pa=True, graph=False, boundary=kind)
    out = bc.run()
    for (c, r), o in zip(structures, out):
        s = eb.Spheres(c, r, deduplicate=False)
        prep = eb.PreparedStaticGPUEHSS(s, boundary=kind)
        for run in o['runs']:
            seed = bc.plan.jobs[o['structure'] * 2 + run['tag'][1]].seed
            src = prep.boundary.source(12, seed)
            ref = prep.engine.trace(src, 32)
            assert run['ehss_angstrom2'] == pytest.approx(ref.omega, rel=1e-11)
            assert run['tail_bound_angstrom2'] == pytest.approx(ref.tail_bound, rel=1e-11, abs=1e-12)
            assert run['pa_from_same_rays_angstrom2'] == pytest.approx(ref.pa, rel=1e-11)
            assert run['collision_histogram'] == np.bincount(ref.bounces, minlength=33).tolist()
            assert run['unresolved_rays'] == int(ref.unresolved.sum())
            hit = O.PATree(c, r, 4).query(src.origins, src.directions)[0]
            assert run['pa_angstrom2'] == pytest.approx(float(src.weights[hit].sum()), rel=1e-11)
    with pytest.raises(ValueError):
        BatchCCS(structures, 12, [7, 8], boundary=kind, cap_ladder=(64,))


@pytest.mark.parametrize('kind', ['box', 'ellipsoid'])
def test_boundary_blocks_on_varied_shapes(eb, kind):
    """Boundary incidence on elongated, flat and split structures: the rays start
    outside every sphere, exterior and full scenes give identical fused blocks,
    and per-ray outcomes equal the oracle's."""
    from ehss_b200.batch import BatchCCS
    from test_gpu_batched import _shapes
    structures = _shapes(505)
    seeds = list(range(505, 505 + len(structures)))
    kw = dict(repeats=2, cap=64, pa=True, graph=False, boundary=kind)
    a = BatchCCS(structures, 12, seeds, exterior=False, **kw).run()
    b = BatchCCS(structures, 12, seeds, exterior=True, **kw).run()
    keys = ('ehss_angstrom2', 'pa_angstrom2', 'unresolved_rays', 'escaped_rays', 'collision_histogram')
    for x, y in zip(a, b):
        for rx, ry in zip(x['runs'], y['runs']):
            assert {k: rx[k] for k in keys} == {k: ry[k] for k in keys}
    for i in (3, 4, 5):              # rod, sheet, split clusters
        c, r = structures[i]
        s = eb.Spheres(c, r, deduplicate=False)
        prep = eb.PreparedStaticGPUEHSS(s, boundary=kind)
        src = prep.boundary.source(11, 77 + i)
        gap = np.linalg.norm(src.origins[:, None, :] - c[None, :, :], axis=2) - r[None, :]
        assert gap.min() >= -1e-9
        got = prep.engine.trace(src, 64, record_history=True)
        ref = O.StaticTree(c, r, 4).trace(src.origins, src.directions, cap=64, record=True, threads=O.host_cores())
        for field in ('positions', 'outgoing', 'escaped', 'unresolved', 'bounces', 'collider_ids'):
            np.testing.assert_array_equal(getattr(got, field), ref[field], err_msg=f'{i} {field}')
