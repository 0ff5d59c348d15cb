"""Batched and served forms on the device: determinism across mixes, agreement
with single-structure runs, the autotuner, and the served request loop."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def eb():
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    import ehss_b200
    return ehss_b200


def _structures(sizes, seed=0):
    from ehss_b200 import workloads as W
    return [W.globule(n, seed + i)[:2] for i, n in enumerate(sizes)]


def test_batchccs_equals_per_structure_blocks(eb):
    from ehss_b200.batch import BatchCCS
    from ehss_b200.blocks import BlockJob, BlockPlan, seed_schedule
    structures = _structures([20, 700, 150, 3000])
    log2s, seeds = [12, 13, 12, 14], [11, 22, 33, 44]
    bc = BatchCCS(structures, log2s, seeds, repeats=3, cap=64, graph=True)
    out = bc.run()
    again = bc.run()
    for s, ((c, r), lg, sd) in enumerate(zip(structures, log2s, seeds)):
        scene = eb.Scene(c, r)
        plan = BlockPlan([BlockJob(scene, lg, k) for k in seed_schedule(sd, 3)])
        plan.run()
        single = [x['ehss_angstrom2'] for x in plan.collect()]
        assert [x['ehss_angstrom2'] for x in out[s]['runs']] == single
        assert out[s]['ehss_angstrom2'] == again[s]['ehss_angstrom2']


def test_server_results_same_alone_and_in_the_mix(eb):
    from ehss_b200.serve import CCSRequest, CCSServer, DeviceExecutor
    ex = DeviceExecutor()
    structures = _structures([30, 400, 1500, 90], seed=5)
    alone = CCSServer(ex, block_log2=13, target=0.01)
    alone.submit(CCSRequest('x', *structures[1], seed=99))
    ra = alone.run()['x']
    mixed = CCSServer(ex, block_log2=13, target=0.01)
    for rid, (c, r), seed in zip('axbd', structures, (1, 99, 2, 3)):
        mixed.submit(CCSRequest(rid, c, r, seed=seed))
    done = mixed.run()
    assert done['x']['values'] == ra['values']
    assert all(d['converged'] for d in done.values())
    lat = mixed.latency_percentiles()
    assert lat['requests'] == 4 and lat['p99_ms'] >= lat['p50_ms'] > 0


def test_autotuner_returns_a_valid_faster_or_equal_launch(eb):
    from ehss_b200 import autotune
    from ehss_b200.blocks import BlockJob, BlockPlan
    scenes = [eb.Scene(c, r) for c, r in _structures([500, 2000], seed=9)]
    jobs = [BlockJob(sc, 14, k) for sc in scenes for k in range(2)]
    space = dict(block_threads=(64, 128), warps_per_sm=(16, 24), chunk_rays=(128, 256), resolve_batch=(16, 24),
                 smem_stack=(8, 16))
    launch, ms = autotune.tune(jobs, passes=1, use_cache=False, space=space)
    assert ms > 0 and launch['block_threads'] in (64, 128)
    plan = BlockPlan(jobs, launch=launch)
    plan.run()
    ref = BlockPlan(jobs)
    ref.run()
    assert [r['ehss_angstrom2'] for r in plan.collect()] == [r['ehss_angstrom2'] for r in ref.collect()]


def _lattice(k=6, spacing=1.2, radius=1.5):
    g = np.stack(np.meshgrid(*[np.arange(k)] * 3, indexing='ij'), -1).reshape(-1, 3) * spacing
    return g.astype(np.float64), np.full(len(g), radius)


@pytest.mark.parametrize('precision', ['fp64', 'fp32'])
def test_exterior_scenes_give_identical_blocks(eb, precision):
    """Buried atoms left out of the trees change no outcome of any block."""
    from ehss_b200.batch import BatchCCS
    from ehss_b200.blocks import DEFAULT_LAUNCH
    # degenerate cases: duplicated atoms, small atoms nested in large ones, a collinear chain
    dup = (np.repeat(np.array([[0., 0., 0.], [1.5, 0., 0.], [0., 1.5, 0.]]), 3, axis=0), np.full(9, 1.7))
    nest = (np.array([[0., 0., 0.], [0.2, 0., 0.], [0., 0.3, 0.1], [2.5, 0., 0.]]), np.array([3.0, 0.8, 1.2, 2.0]))
    chain = (np.stack([np.arange(30) * 1.1, np.zeros(30), np.zeros(30)], 1), np.full(30, 1.6))
    structures = _structures([1, 3, 40, 700, 3000], seed=31) + [_lattice(), dup, nest, chain]
    seeds = [5, 6, 7, 8, 9, 10, 11, 12, 13]
    kw = dict(repeats=2, cap=64, precision=precision, pa=True, graph=False,
              launch=dict(DEFAULT_LAUNCH, count_tests=True))
    full = BatchCCS(structures, 13, seeds, exterior=False, **kw)
    ext = BatchCCS(structures, 13, seeds, exterior=True, **kw)
    a, b = full.run(), ext.run()
    keys = ('ehss_angstrom2', 'pa_angstrom2', 'pa_from_same_rays_angstrom2', 'unresolved_rays', 'escaped_rays',
            'collision_histogram', 'collision_contribution_angstrom2')
    for x, y in zip(a, b):
        for rx, ry in zip(x['runs'], y['runs']):
            assert {k: rx[k] for k in keys} == {k: ry[k] for k in keys}
    infos = [ext.batch.info(i) for i in range(len(structures))]
    assert all(i.exterior == 1 and 1 <= i.n_active <= i.n_atoms for i in infos)
    assert infos[5].n_active == 216 - 64             # the lattice's 4^3 inner atoms are buried
    assert infos[7].n_active == 2                    # the nested atoms are held by the large one
    assert infos[4].n_active < infos[4].n_atoms      # and so are a globule's core atoms
    assert all(full.batch.info(i).n_active == n for i, n in enumerate(full.n_atoms))
    tests = lambda out: sum(r['sphere_tests'] for o in out for r in o['runs'])
    assert tests(b) < tests(a)


def test_exterior_scene_refused_for_explicit_rays(eb):
    import torch
    from ehss_b200 import _lib
    c, r = _lattice()
    sc = eb.Scene(c, r, exterior=True)
    assert sc.exterior and sc.n_active == 216 - 64
    with pytest.raises(ValueError):
        eb.GPUEHSSTransport(sc)
    n = 4
    o = torch.zeros((n, 3), dtype=torch.float64, device='cuda')
    o[:, 0] = -50.0
    d = torch.zeros((n, 3), dtype=torch.float64, device='cuda')
    d[:, 0] = 1.0
    own = torch.full((n,), -1, dtype=torch.int64, device='cuda')
    blocked = torch.zeros(n, dtype=torch.uint8, device='cuda')
    stats = torch.zeros(_lib.NSTATS, dtype=torch.int64, device='cuda')
    _lib.check(_lib.load().ehss_pa_anyhit(sc.ptr, n, o.data_ptr(), d.data_ptr(), own.data_ptr(), blocked.data_ptr(),
                                          stats.data_ptr(), torch.cuda.current_stream().cuda_stream))
    assert int(stats[_lib.STAT_ERRORS]) == n and int(blocked.sum()) == 0


def _padded(d, cap):
    h = list(d['collision_histogram']) + [0] * (cap + 1 - len(d['collision_histogram']))
    l = list(d['collision_contribution_angstrom2']) + [0.0] * (cap + 1 - len(d['collision_contribution_angstrom2']))
    return h, l


@pytest.mark.parametrize('precision,capacity', [('fp64', 1 << 16), ('fp32', 1 << 16), ('fp32', 3)])
def test_cap_extension_equals_a_run_at_the_larger_cap(eb, precision, capacity):
    """Continuing only the saved unresolved rays gives the totals of a run
    that used the larger cap from the start (capacity 3 forces the re-trace
    with a larger residual buffer)."""
    from ehss_b200 import _lib
    from ehss_b200.blocks import BlockJob, BlockPlan
    prec = {'fp64': _lib.PREC_FP64, 'fp32': _lib.PREC_FP32}[precision]
    scenes = [eb.Scene(c, r, exterior=True) for c, r in _structures([300, 1800], seed=41)]
    jobs = lambda cap: [BlockJob(sc, 12, 100 + k, cap=cap, precision=prec, pa=True, tag=(s, k))
                        for s, sc in enumerate(scenes) for k in range(2)]
    plan = BlockPlan(jobs(3), residual_capacity=capacity)
    plan.run()
    first = plan.collect()
    assert sum(r['unresolved_rays'] for r in first) > 10
    ext = plan.extend_caps((6, 12, 64), tail_fraction=0.0)
    ref = BlockPlan(jobs(64))
    ref.run()
    full = ref.collect()
    for a, b, f in zip(ext, full, first):
        for key in ('ehss_angstrom2', 'tail_bound_angstrom2', 'unresolved_rays', 'escaped_rays',
                    'pa_from_same_rays_angstrom2', 'pa_angstrom2'):
            assert a[key] == b[key], key
        assert _padded(a, 64) == _padded(b, 64)
        caps = [x['cap'] for x in a['cap_attempts']]
        assert caps[0] == 3 and caps == sorted(caps) and a['cap'] == caps[-1]
        assert a['cap'] == 64 or a['unresolved_rays'] == 0
        assert sum(x['continued_rays'] for x in a['cap_attempts'][1:2]) == f['unresolved_rays']


def test_batchccs_cap_ladder_stops_when_the_tail_is_small(eb):
    from ehss_b200.batch import BatchCCS
    structures = _structures([200, 900], seed=43)
    low = BatchCCS(structures, 12, [1, 2], repeats=2, cap=4, cap_ladder=(8, 16, 64), tail_fraction=5e-4, graph=False)
    out = low.run()
    for o in out:
        for run in o['runs']:
            att = run['cap_attempts']
            last = att[-1]
            assert last['tail_bound_angstrom2'] <= 5e-4 * last['ehss_angstrom2'] or last['cap'] == 64
            assert all(x['tail_bound_angstrom2'] > 5e-4 * x['ehss_angstrom2'] for x in att[:-1])


def _shapes(seed):
    """Structures of varied shape, density and radius mix for the exterior identity."""
    rng = np.random.default_rng(seed)
    out = []
    # dense and sparse random clouds with mixed radii
    for n, box in ((400, 12.), (400, 25.), (1500, 22.)):
        c = rng.uniform(-box / 2, box / 2, (n, 3))
        out.append((c, rng.uniform(0.6, 2.8, n)))
    # a rod, a sheet, two separated clusters
    t = rng.uniform(0, 60, 300)
    out.append((np.stack([t, rng.normal(0, 1.2, 300), rng.normal(0, 1.2, 300)], 1), rng.uniform(1.2, 2.0, 300)))
    out.append((np.stack([rng.uniform(0, 30, 500), rng.uniform(0, 30, 500), rng.normal(0, 0.8, 500)], 1),
                np.full(500, 1.7)))
    a = rng.normal(0, 3, (200, 3)); b = rng.normal(0, 3, (200, 3)) + [40., 0., 0.]
    out.append((np.concatenate([a, b]), rng.uniform(1.0, 2.2, 400)))
    # a dense ball of large atoms around a few small ones, with exact duplicates
    c = rng.normal(0, 2.5, (250, 3))
    c = np.concatenate([c, c[:20]])
    out.append((c, np.concatenate([rng.uniform(1.5, 3.0, 250), rng.uniform(0.3, 0.6, 20)])))
    return out


@pytest.mark.parametrize('seed', [101, 202])
def test_exterior_identity_on_varied_shapes(eb, seed):
    """Exterior and full scenes give identical block results (FP32 filter, PA on)
    on clouds, rods, sheets, split clusters and dense balls with duplicates."""
    from ehss_b200.batch import BatchCCS
    structures = _shapes(seed)
    seeds = list(range(seed, seed + len(structures)))
    kw = dict(repeats=2, cap=64, precision='fp32', pa=True, graph=False)
    a = BatchCCS(structures, 14, seeds, exterior=False, **kw).run()
    ext = BatchCCS(structures, 14, seeds, exterior=True, **kw)
    b = ext.run()
    keys = ('ehss_angstrom2', 'pa_angstrom2', 'unresolved_rays', 'escaped_rays', 'collision_histogram',
            'collision_contribution_angstrom2')
    for x, y in zip(a, b):
        for rx, ry in zip(x['runs'], y['runs']):
            assert {k: rx[k] for k in keys} == {k: ry[k] for k in keys}
    assert sum(ext.batch.info(i).n_active for i in range(len(structures))) < sum(len(r) for _, r in structures)


@pytest.mark.parametrize('seed', [303])
def test_fp32_filter_equals_fp64_on_varied_shapes(eb, seed):
    """The FP32 filter with FP64 re-test returns the FP64 path's outcomes on the
    varied shapes, also far from the origin and with radii spanning 0.1-3 A."""
    from ehss_b200.batch import BatchCCS
    rng = np.random.default_rng(seed)
    structures = _shapes(seed)
    c = rng.normal(0, 4, (300, 3)) + [1.0e4, -2.5e4, 3.0e3]          # far from the origin
    structures.append((c, rng.uniform(0.1, 3.0, 300)))
    seeds = list(range(seed, seed + len(structures)))
    kw = dict(repeats=2, cap=64, pa=True, graph=False, exterior=False)
    a = BatchCCS(structures, 14, seeds, precision='fp64', **kw).run()
    b = BatchCCS(structures, 14, seeds, precision='fp32', **kw).run()
    keys = ('ehss_angstrom2', 'pa_angstrom2', 'unresolved_rays', 'escaped_rays', 'collision_histogram',
            'collision_contribution_angstrom2')
    for x, y in zip(a, b):
        for rx, ry in zip(x['runs'], y['runs']):
            assert {k: rx[k] for k in keys} == {k: ry[k] for k in keys}


def test_cap_extension_on_varied_shapes(eb):
    """Cap 2 continued to 5, 17 and 64 equals a run at cap 64 on clouds, rods,
    sheets, split clusters and dense balls with duplicates."""
    from ehss_b200.blocks import BlockJob, BlockPlan
    scenes = [eb.Scene(c, r, exterior=True) for c, r in _shapes(808)]
    jobs = lambda cap: [BlockJob(sc, 12, 300 + s, cap=cap, pa=True, tag=(s, 0)) for s, sc in enumerate(scenes)]
    plan = BlockPlan(jobs(2), residual_capacity=1 << 14)
    plan.run()
    first = plan.collect()
    assert sum(r['unresolved_rays'] for r in first) > 10
    ext = plan.extend_caps((5, 17, 64), tail_fraction=0.0)
    ref = BlockPlan(jobs(64))
    ref.run()
    for a, b in zip(ext, ref.collect()):
        for key in ('ehss_angstrom2', 'tail_bound_angstrom2', 'unresolved_rays', 'escaped_rays',
                    'pa_from_same_rays_angstrom2', 'pa_angstrom2'):
            assert a[key] == b[key], key
        assert _padded(a, 64) == _padded(b, 64)


def test_large_structure_exterior_identity_and_oracle_ccs(eb):
    """A 100,000-atom globule (device-wide key sort, global refit, exposure test
    at scale): exterior and full scenes give identical blocks, and the CCS
    equals the oracle's on the same rays."""
    from ehss_b200 import workloads as W
    from ehss_b200.batch import BatchCCS
    c, r, _ = W.globule(100000, 1)
    kw = dict(repeats=1, cap=64, pa=True, graph=False)
    a = BatchCCS([(c, r)], 12, [9], exterior=False, **kw).run()[0]['runs'][0]
    ext = BatchCCS([(c, r)], 12, [9], exterior=True, **kw)
    b = ext.run()[0]['runs'][0]
    for key in ('ehss_angstrom2', 'pa_angstrom2', 'unresolved_rays', 'escaped_rays', 'collision_histogram'):
        assert a[key] == b[key], key
    info = ext.batch.info(0)
    assert info.n_active < info.n_atoms // 2                       # most of a large globule is buried
    scene = eb.Scene(c, r)
    o, d = (x.cpu().numpy() for x in scene.source_rays(12, 9))
    ref = O.StaticTree(c, r, 4).trace(o, d, cap=64, threads=O.host_cores())
    ro = O.readout(dict(incoming=d, weights=np.full(len(o), np.pi * scene.radius ** 2 / len(o))), ref, 64)
    assert b['ehss_angstrom2'] == pytest.approx(ro['ehss_angstrom2'], rel=1e-12)
    assert b['collision_histogram'] == ro['collision_histogram']
