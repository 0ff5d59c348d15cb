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
