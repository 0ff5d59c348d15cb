"""Builder paths: batches of structures of at most 2048 or 8192 atoms sort their
Morton keys per structure in one block radix sort (two sizes); larger batches
use the device-wide sort.  Both are stable sorts of the same keys, so the scenes must be identical
byte for byte."""
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


def _scene_bytes(batch, i):
    raw = batch.scene_buf.cpu().numpy()
    off = batch.scene_ptrs[i] - batch.scene_buf.data_ptr()
    return raw[off:off + int(batch._sizes[i])]


@pytest.mark.parametrize('largest', [2048, 8192])
@pytest.mark.parametrize('exterior', [False, True])
def test_segment_sort_build_equals_device_sort_build(eb, exterior, largest):
    from ehss_b200 import workloads as W
    from ehss_b200.batch import BatchScenes
    small = [W.globule(n, 70 + i)[:2] for i, n in enumerate([1, 2, 13, 15, 300, 1990, largest - 50])]
    # duplicated atoms: equal keys keep atom order in both sorts
    c, r = small[4]
    small.append((np.concatenate([c, c[:50]]), np.concatenate([r, r[:50]])))
    big = W.globule(9000, 99)[:2]
    a = BatchScenes(small, exterior=exterior)            # per-structure sort
    b = BatchScenes(small + [big], exterior=exterior)    # device-wide sort
    for batch in (a, b):
        batch.scene_buf.zero_()                          # alignment padding is never written
        batch.build()
    for i in range(len(small)):
        assert np.array_equal(_scene_bytes(a, i), _scene_bytes(b, i)), i
        assert a.info(i).n_nodes == b.info(i).n_nodes
    # the big structure alone (4 sort passes over 31 key bits) and in the batch (5 passes over 35)
    alone = BatchScenes([big], exterior=exterior)
    alone.scene_buf.zero_()
    alone.build()
    assert np.array_equal(_scene_bytes(alone, 0), _scene_bytes(b, len(small)))


def _spread10(v):
    v = v.astype(np.uint64) & 0x3ff
    v = (v | (v << 16)) & 0x030000FF
    v = (v | (v << 8)) & 0x0300F00F
    v = (v | (v << 4)) & 0x030C30C3
    v = (v | (v << 2)) & 0x09249249
    return v


def test_device_sort_orders_large_structures_like_a_stable_cpu_sort(eb):
    """Leaf order of structures beyond the per-structure sort (8,193 to
    60,000 atoms, the last 500 duplicating the first 500, so many keys are
    equal): the scene's id map lists the atoms in the stable order of their
    30-bit Morton keys, recomputed here in FP64 from the scene's own centre."""
    from ehss_b200 import workloads as W
    from ehss_b200.batch import BatchScenes
    for n, seed in ((8193, 5), (20000, 6), (60000, 7)):
        c, r, _ = W.globule(n - 500, seed)
        c = np.concatenate([c, c[:500]]); r = np.concatenate([r, r[:500]])
        batch = BatchScenes([(c, r)])
        batch.build()
        raw = _scene_bytes(batch, 0)
        info = batch.info(0)
        assert info.n_atoms == n
        off_ids = int(np.frombuffer(raw[120:128].tobytes(), dtype=np.uint64)[0])
        ids = np.frombuffer(raw[off_ids:off_ids + 4 * n].tobytes(), dtype=np.int32)
        x = c - np.array(info.center[:])                 # the builder's centre-relative coordinates
        lo, hi = x.min(axis=0), x.max(axis=0)
        ext = hi + (-lo)
        u = np.clip(np.where(ext > 0, (x - lo) / np.where(ext > 0, ext, 1), 0.0), 0.0, 1.0)
        q = np.minimum(u * 1024.0, 1023.0).astype(np.uint32)
        key = (_spread10(q[:, 0]) << 2) | (_spread10(q[:, 1]) << 1) | _spread10(q[:, 2])
        np.testing.assert_array_equal(ids, np.argsort(key, kind='stable'))
