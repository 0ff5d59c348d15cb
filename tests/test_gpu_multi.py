"""The several-GPU splits on one device, rank by rank: the ranks' kernels
never wait on one another, so their launches can run one after the other on
a single GPU, and the sum of their integer results (what the all-reduce
computes) must equal one launch of the whole job bit for bit.

* ray windows: one 2000-atom structure's 20 seed blocks (the precision
  configuration's shape at 2^14 rays per seed) cut into 3 and 8 windows;
* structure shards: a 24-structure mixed batch over 3 ranks.  A shard's
  plan has fewer rays, so it takes smaller chunks; a lane's traversal order
  depends on its warp-mates (leaves are postponed until the warp's lanes
  all hold one), so the diagnostic counters of tests made (box, sphere,
  FP64 re-tests, grazing and fallback queries) can differ, while every
  outcome integer and the per-ray query and error counts are equal."""
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


def test_ray_windows_add_up_to_one_launch(eb):
    from ehss_b200 import distributed as D, workloads as W
    from ehss_b200.blocks import BlockJob, BlockPlan
    c, r, _ = W.globule(2000, 2000)
    scene = eb.Scene(c, r, exterior=True)
    jobs = [BlockJob(scene, 14, seed, cap=64, pa=seed % 2 == 0) for seed in range(20)]
    whole = BlockPlan(jobs)
    whole.enqueue()
    ref = whole.packed.clone()
    for world in (3, 8):
        plan = BlockPlan(jobs)
        windows = D.chunk_windows(plan.chunk_costs(), world)
        total = None
        for first, end in windows:
            plan.window = (first, end)
            plan.enqueue()
            total = plan.packed.clone() if total is None else total + plan.packed
        assert windows[0][0] == 0 and windows[-1][1] == plan.total_chunks
        assert bool((total == ref).all()), world
        # the readout of the summed integers is the whole plan's
        plan.packed.copy_(total)
        a, b = plan.collect(), whole.collect()
        assert [x['ehss_angstrom2'] for x in a] == [x['ehss_angstrom2'] for x in b]
    # an empty window (more ranks than work at the end of a list) traces nothing and leaves zeros
    plan = BlockPlan(jobs)
    plan.window = (7, 7)
    plan.enqueue()
    assert int(plan.packed.abs().sum()) == 0


def test_structure_shards_add_up_to_one_batch(eb):
    import torch
    from ehss_b200 import distributed as D, workloads as W
    spec = W.mixed_batch(24, seed=77)
    structures = [W.globule(n, s)[:2] for n, _, s in spec]
    log2s = [min(lg, 15) for _, lg, _ in spec]
    seeds = [s % 2 ** 32 for _, _, s in spec]
    full = D.ShardedBatch(structures, log2s, seeds, 0, 1, graph=False)
    full.upload()
    full.build()
    full.trace()
    ref = full.exchange().clone()
    np.testing.assert_array_equal(ref.cpu().numpy(), full.batch.plan.packed.cpu().numpy())
    # the merged integers read out as BatchCCS reads its own
    for a, b in zip(full.summaries(), full.batch.download()):
        for key in ('mean', 'sd', 'sem'):
            assert a['ehss_angstrom2'][key] == pytest.approx(b['ehss_angstrom2'][key], rel=1e-14, abs=1e-14)
        assert a['ehss_unresolved_rays_total'] == b['ehss_unresolved_rays_total']
    total = torch.zeros_like(ref)
    owners = []
    for rank in range(3):
        part = D.ShardedBatch(structures, log2s, seeds, rank, 3, graph=False)
        owners.append(part.mine)
        part.upload()
        part.build()
        part.trace()
        total += part.scatter()
    assert sorted(i for m in owners for i in m) == list(range(24))
    from ehss_b200 import _lib
    from ehss_b200.blocks import _RESULT_WORDS, _STATS0
    n_res = 24 * 3 * _RESULT_WORDS
    words = np.arange(n_res) % _RESULT_WORDS
    order_free = (words < _STATS0) | (words == _STATS0 + _lib.STAT_QUERIES) | (words == _STATS0 + _lib.STAT_ERRORS)
    a, b = total.cpu().numpy(), ref.cpu().numpy()
    np.testing.assert_array_equal(a[:n_res][order_free], b[:n_res][order_free])
    np.testing.assert_array_equal(a[n_res:], b[n_res:])          # histograms and ledgers
