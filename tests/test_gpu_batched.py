"""Batched and served forms on the device: determinism across mixes, agreement
with single-structure runs, the autotuner, and the served request loop."""
import numpy as np
import pytest

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
