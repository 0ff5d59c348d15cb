"""Host logic of the served form and of the multi-GPU sharding (CPU only).

The server's device side is replaced by a fake executor whose block results
are a deterministic function of (structure, seed), like the device's integer
sums; the sharded path runs as two gloo ranks on CPU.
"""
import math
import os
import socket

import numpy as np
import pytest

from ehss_b200.serve import CCSRequest, CCSServer, rel_rmse
from ehss_b200 import distributed as D


class FakeExecutor:
    """Block value = structure-dependent mean + seeded noise; 100 bytes per atom."""

    def __init__(self, noise=0.02):
        self.noise = noise
        self.built, self.released, self.traced = [], [], []

    def footprint(self, n_atoms):
        return 100 * n_atoms

    def build(self, structures):
        handles = []
        for c, r in structures:
            h = (len(r), float(np.round(c.sum(), 6)))
            self.built.append(h)
            handles.append(h)
        return handles

    def trace(self, jobs):
        self.traced.append(len(jobs))
        out = []
        for (n, key), log2, seed in jobs:
            rng = np.random.default_rng([n, int(abs(key) * 1000) % 2 ** 31, seed])
            out.append((100.0 + n + self.noise * (100 + n) * rng.normal(), 0.0))
        return out

    def release(self, handle):
        self.released.append(handle)


def _req(rid, n, seed=1, arrival=0.0):
    rng = np.random.default_rng(n)
    return CCSRequest(rid, rng.normal(size=(n, 3)), np.ones(n), seed=seed, arrival=arrival)


def test_rel_rmse():
    assert math.isinf(rel_rmse([1.0]))
    a = [1.0, 1.1, 0.9, 1.0]
    assert rel_rmse(a) == pytest.approx(np.std(a, ddof=1) / 2 / 1.0)


def test_results_same_alone_and_in_the_mix():
    alone = CCSServer(FakeExecutor(), target=0.01)
    alone.submit(_req('a', 50, seed=7))
    ra = alone.run()['a']
    mixed = CCSServer(FakeExecutor(), target=0.01)
    for rid, n, seed in [('b', 300, 3), ('a', 50, 7), ('c', 12, 9), ('d', 1000, 11)]:
        mixed.submit(_req(rid, n, seed=seed))
    rm = mixed.run()['a']
    assert ra['values'] == rm['values'] and ra['blocks'] == rm['blocks']
    assert rm['converged'] and rm['rel_rmse'] <= 0.01 and rm['blocks'] >= 2


def test_admission_by_memory_and_rejection():
    ex = FakeExecutor()
    server = CCSServer(ex, budget_bytes=100 * 1500, target=0.01)
    server.submit(_req('big', 1000))
    server.submit(_req('big2', 1000))       # does not fit beside 'big'
    server.submit(_req('small', 100))
    server.step()
    assert {s.req.rid for s in server.active} | set(server.done) == {'big', 'small'}
    assert [s.req.rid for s in server.pending] == ['big2']
    done = server.run()
    assert set(done) == {'big', 'big2', 'small'}
    assert done['big2']['admitted_s'] >= done['big']['latency_s'] - 1e-9   # waited for memory
    assert server.used == 0 and len(ex.released) == 3
    with pytest.raises(ValueError):
        server.submit(_req('huge', 5000))


def test_batch_memory_held_until_its_last_member_finishes():
    """Two requests admitted together share one build allocation: when the
    quick one finishes, its bytes stay counted until the slow one is done, so
    a third request that fits only in the freed share waits for the batch."""
    class TwoSpeed(FakeExecutor):
        def trace(self, jobs):
            # 'quick' (10 atoms) converges at once; 'slow' (20 atoms) needs 6 blocks
            out = []
            for (n, key), log2, seed in jobs:
                if n == 10:
                    out.append((100.0, 0.0))
                else:
                    out.append((100.0 + (20.0 if seed % 2 else -20.0), 0.0))
            return out
    ex = TwoSpeed()
    server = CCSServer(ex, budget_bytes=100 * 35, target=0.1, max_blocks=6)
    server.submit(_req('quick', 10))
    server.submit(_req('slow', 20))
    server.submit(_req('third', 10))        # fits only in what 'quick' held
    server.step()
    assert 'quick' in server.done and [s.req.rid for s in server.active] == ['slow']
    assert server.used == 100 * 30          # the batch is still allocated
    server.step()
    assert [s.req.rid for s in server.pending] == ['third']
    while 'slow' not in server.done:
        server.step()
    assert server.used == 0 or [s.req.rid for s in server.active] == ['third']
    done = server.run()
    assert set(done) == {'quick', 'slow', 'third'}
    assert done['third']['admitted_s'] >= done['slow']['latency_s'] - 1e-9
    assert server.used == 0


def test_late_arrivals_join_running_rounds():
    t = [0.0]
    ex = FakeExecutor(noise=0.05)
    server = CCSServer(ex, target=0.01, clock=lambda: t[0])
    server.submit(_req('early', 40, arrival=0.0))
    server.submit(_req('late', 60, arrival=0.5))
    server.step()
    assert [s.req.rid for s in server.active] == ['early']
    t[0] = 0.6
    server.step()
    rids = {s.req.rid for s in server.active} | set(server.done)
    assert 'late' in rids and 'early' in rids
    while server.active or server.pending:
        t[0] += 0.01
        server.step()
    assert server.done['late']['latency_s'] > 0


def test_shard_balances_and_covers():
    costs = [D.estimated_cost(n, 1 << lg) for n, lg in [(20, 14), (5000, 18), (300, 16), (40, 15), (1200, 17)]]
    owner = D.shard(costs, 2)
    assert sorted(set(owner)) == [0, 1]
    loads = [sum(c for c, o in zip(costs, owner) if o == r) for r in (0, 1)]
    assert max(loads) - min(loads) <= max(costs)


def _free_port():
    s = socket.socket()
    s.bind(('127.0.0.1', 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, structures, log2s, seeds, out):
    import torch.distributed as dist
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        def run_local(indices):
            return {i: dict(structure=i, value=float(len(structures[i][1]) * 2 + seeds[i])) for i in indices}
        res = D.run_sharded(structures, log2s, seeds, run_local, rank, world)
        if rank == 0:
            out.put(res)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_sharded_gather_with_two_gloo_ranks():
    import torch.multiprocessing as mp
    structures = [(np.zeros((n, 3)), np.ones(n)) for n in (20, 300, 5000, 45, 1200, 7)]
    log2s = [14, 15, 18, 14, 17, 14]
    seeds = list(range(len(structures)))
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, structures, log2s, seeds, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert [r['structure'] for r in res] == list(range(len(structures)))
    assert [r['value'] for r in res] == [float(len(s[1]) * 2 + i) for i, s in enumerate(structures)]


def test_chunk_windows_cover_the_list_by_cost():
    rng = np.random.default_rng(3)
    for n, world in [(0, 2), (1, 3), (10, 3), (1000, 8), (5, 8)]:
        costs = rng.uniform(0.5, 20.0, n)
        w = D.chunk_windows(costs, world)
        assert len(w) == world and w[0][0] == 0 and w[-1][1] == n
        assert all(a[1] == b[0] for a, b in zip(w, w[1:])) and all(f <= e for f, e in w)
        if n >= 100:
            loads = [costs[f:e].sum() for f, e in w]
            assert max(loads) - min(loads) <= 2 * costs.max()


def test_global_index_partitions_the_batch_layout():
    S, R, W, H1 = 7, 3, 16, 9
    owner = D.shard([D.estimated_cost(n, 1 << 14) for n in (20, 300, 5000, 45, 1200, 7, 90)], 3)
    parts = [D.global_index([i for i, o in enumerate(owner) if o == r], S, R, W, H1) for r in range(3)]
    allidx = np.concatenate(parts)
    assert len(allidx) == S * R * W + 2 * S * R * H1
    np.testing.assert_array_equal(np.sort(allidx), np.arange(len(allidx)))
    # a rank holding every structure in order has the global layout itself
    np.testing.assert_array_equal(D.global_index(list(range(S)), S, R, W, H1), np.arange(len(allidx)))


class _FakeWindowPlan:
    """A plan whose 'kernel' sums integer functions of its rays: chunk c holds
    rays [c*8, c*8 + 8) of one of three blocks; packed = per-block sums."""

    def __init__(self):
        import torch
        self.blocks = [(0, 5), (5, 12), (12, 13)]      # chunk ranges of three blocks
        self.total_chunks = 13
        self.window = None
        self.packed = torch.zeros(6, dtype=torch.int64)

    def chunk_costs(self):
        return [1.0 + (c % 4) for c in range(self.total_chunks)]

    def enqueue(self):
        first, end = self.window if self.window is not None else (0, self.total_chunks)
        self.packed.zero_()
        for b, (lo, hi) in enumerate(self.blocks):
            for c in range(max(lo, first), min(hi, end)):
                for ray in range(c * 8, c * 8 + 8):
                    self.packed[2 * b] += (ray * 2654435761) % 1000003     # a fixed-point 'angle'
                    self.packed[2 * b + 1] += ray % 3 == 0                   # a count


def _window_worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        plan = _FakeWindowPlan()
        windows = D.trace_window_split(plan, rank, world)
        out.put((rank, windows, plan.packed.tolist()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_window_split_sums_equal_one_rank_with_two_gloo_ranks():
    import torch.multiprocessing as mp
    whole = _FakeWindowPlan()
    whole.enqueue()
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_window_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, windows, packed in got:
        assert windows[0][0] == 0 and windows[-1][1] == 13 and windows[0][1] == windows[1][0]
        assert packed == whole.packed.tolist()      # every rank holds the whole plan's integers


class _FakeBatch:
    """Stands in for BatchCCS on CPU: the packed block results are integers
    that depend only on (structure, replicate), laid out as a BlockPlan lays
    them out (result words per block, then histogram, then ledger entries)."""
    W = 16

    def __init__(self, structures, log2s, seeds, repeats=3, cap=64):
        import torch
        self.device = torch.device('cpu')
        self.rays = sum((1 << lg) * repeats for lg in log2s)
        ids = [int(np.round(c.sum() * 1000)) % 100003 for c, _ in structures]
        n = len(structures) * repeats
        res = np.array([[ids[b // repeats] * 7 + (b % repeats) * 3 + w for w in range(self.W)] for b in range(n)])
        hist = np.array([[ids[b // repeats] + k + b % repeats for k in range(cap + 1)] for b in range(n)])
        self.packed_np = np.concatenate([res.ravel(), hist.ravel(), 2 * hist.ravel()]).astype(np.int64)
        self.plan = type('Plan', (), {})()
        self.plan.packed = torch.from_numpy(self.packed_np.copy())

    def upload(self):
        pass

    def build(self):
        pass

    def trace(self):
        pass


def _sharded_worker(rank, world, port, structures, log2s, seeds, out):
    import torch.distributed as dist
    from ehss_b200 import blocks
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        blocks._RESULT_WORDS = _FakeBatch.W
        job = D.ShardedBatch(structures, log2s, seeds, rank, world, repeats=3, cap=8, batch_factory=_FakeBatch)
        packed = job.step().clone()
        out.put((rank, job.mine, packed.numpy().tolist()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_structure_shards_exchange_with_two_gloo_ranks():
    """Each rank holds only its LPT share; after the all-reduce every rank's
    buffer equals the one-rank layout of the whole batch."""
    import torch.multiprocessing as mp
    from ehss_b200 import blocks
    rng = np.random.default_rng(5)
    sizes = (20, 300, 5000, 45, 1200, 7, 90)
    structures = [(rng.normal(size=(n, 3)), np.ones(n)) for n in sizes]
    log2s, seeds = [14, 16, 18, 15, 17, 14, 16], [1, 2, 3, 4, 5, 6, 7]
    saved = blocks._RESULT_WORDS
    blocks._RESULT_WORDS = _FakeBatch.W
    try:
        whole = D.ShardedBatch(structures, log2s, seeds, 0, 1, repeats=3, cap=8, batch_factory=_FakeBatch)
        ref = whole.step().numpy().tolist()
    finally:
        blocks._RESULT_WORDS = saved
    assert ref == whole.batch.packed_np.tolist()
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_sharded_worker, args=(r, 2, port, structures, log2s, seeds, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    mines = sorted(i for _, mine, _ in got for i in mine)
    assert mines == list(range(len(sizes)))
    for rank, mine, packed in got:
        assert packed == ref, rank


def test_sharded_summaries_read_the_merged_integers():
    """summaries() turns the merged block integers into per-structure CCS
    with the blocks' impact-disk weights (pi R^2 / rays, fixed point 2^-36)."""
    from ehss_b200 import blocks, _lib
    from ehss_b200.batch import enclosing_radius
    rng = np.random.default_rng(9)
    structures = [(rng.normal(size=(n, 3)), np.full(n, 1.5)) for n in (12, 40)]
    saved = blocks._RESULT_WORDS
    blocks._RESULT_WORDS = _FakeBatch.W
    try:
        job = D.ShardedBatch(structures, [14, 15], [1, 2], 0, 1, repeats=3, cap=8, batch_factory=_FakeBatch)
        job.step()
        summ = job.summaries()
    finally:
        blocks._RESULT_WORDS = saved
    res = job.batch.packed_np[:2 * 3 * _FakeBatch.W].reshape(6, _FakeBatch.W)
    for s, lg in enumerate((14, 15)):
        R = enclosing_radius(*structures[s])
        w = np.pi * R * R / 2 ** lg
        vals = w * (res[3 * s:3 * s + 3, 0].astype(np.float64) * _lib.FX_SCALE)
        assert summ[s]['ehss_angstrom2']['mean'] == pytest.approx(vals.mean(), rel=1e-15)
        assert summ[s]['ehss_unresolved_rays_total'] == int(res[3 * s:3 * s + 3, 2].sum())


def test_requests_from_xyz_files(tmp_path):
    """XYZ jobs are read and prepared as the command line does and served."""
    from ehss_b200 import ccs_cli
    xyz = tmp_path / 'water.xyz'
    xyz.write_text('3\nwater\nO 0 0 0\nH 0.9572 0 0\nH -0.239987 0.926627 0\n'
                   '3\nsecond\nO 0 0 0\nH 0.96 0 0\nH -0.24 0.93 0\n')
    req = CCSRequest.from_xyz('w2', xyz, frame=2, seed=5)
    spheres, _ = ccs_cli.prepare_frame(ccs_cli.read_xyz(xyz)[1], ccs_cli.radius_table(None), 1.4)
    np.testing.assert_array_equal(req.centers, spheres.centers)
    np.testing.assert_array_equal(req.radii, spheres.radii)
    assert req.seed == 5
    with pytest.raises(ValueError, match='exceeds 2 frames'):
        CCSRequest.from_xyz('w3', xyz, frame=3)
    server = CCSServer(FakeExecutor(), target=0.01)
    server.submit(req)
    assert server.run()['w2']['converged']
