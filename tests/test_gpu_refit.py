"""Refit of device scenes (ehss_scenes_refit): new coordinates for the same
atoms with the tree topology kept, the device counterpart of the reference's
SphereIndex.refit (pa_spatial.py:166-170) and bottom-up box refit
(_refit, pa_spatial.py:78-95).  A refit scene must trace exactly like a
scene built from the new coordinates, and its boxes must contain its atoms."""
import ctypes as ct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LEAF_BITS, EMPTY = 4, -2 ** 31


@pytest.fixture(scope='module')
def eb():
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    import ehss_b200
    return ehss_b200


def _moved(c, sigma, seed):
    return c + np.random.default_rng(seed).normal(0., sigma, c.shape)


def _align256(x):
    return (x + 255) & ~255


def _scene_arrays(scene):
    """Node records and atom arrays of a full scene, parsed from its device buffer."""
    n = scene.n_atoms
    raw = scene._buf.cpu().numpy()[scene.ptr - scene._buf.data_ptr():][:scene.nbytes]
    alloc = max(n - 1, 1)
    off_nodes = 256
    off_atoms = _align256(off_nodes + alloc * 128)
    off_atoms64 = _align256(off_atoms + n * 16)
    off_ids = _align256(off_atoms64 + n * 32)
    nodes = raw[off_nodes:off_nodes + alloc * 128].view(np.float32).reshape(alloc, 8, 4)
    atoms64 = raw[off_atoms64:off_atoms64 + n * 32].view(np.float64).reshape(n, 4)
    ids = raw[off_ids:off_ids + n * 4].view(np.int32)
    return nodes[:scene.info.n_nodes], atoms64, ids


def _check_boxes(scene):
    """Every reachable slot box contains the spheres of its subtree."""
    nodes, atoms64, ids = _scene_arrays(scene)
    center = np.asarray(scene.center)
    lo_atom = atoms64[:, :3] - center - atoms64[:, 3:4]
    hi_atom = atoms64[:, :3] - center + atoms64[:, 3:4]
    checked = 0

    def subtree(ref):
        if ref < 0:
            code = ~ref
            first, cnt = code >> LEAF_BITS, (code & 15) + 1
            return list(range(first, first + cnt))
        out = []
        for r in nodes[ref, 6].view(np.int32):
            if r != EMPTY:
                out += subtree(int(r))
        return out

    stack = [0]
    while stack:
        i = stack.pop()
        refs = nodes[i, 6].view(np.int32)
        for c, r in enumerate(refs):
            if r == EMPTY:
                continue
            atoms = subtree(int(r))
            lo = np.array([nodes[i, 0, c], nodes[i, 2, c], nodes[i, 4, c]], dtype=np.float64)
            hi = np.array([nodes[i, 1, c], nodes[i, 3, c], nodes[i, 5, c]], dtype=np.float64)
            assert np.all(lo <= lo_atom[atoms].min(axis=0)) and np.all(hi >= hi_atom[atoms].max(axis=0))
            checked += len(atoms)
            if r >= 0:
                stack.append(int(r))
    assert checked >= scene.n_atoms


@pytest.mark.parametrize('n', [1, 5, 14, 15, 600])
def test_refit_scene_equals_a_build_of_the_new_coordinates(eb, n):
    from ehss_b200 import workloads as W
    c0, r, _ = W.globule(max(n, 2), 3) if n > 1 else (np.zeros((1, 3)), np.array([1.7]), None)
    c0, r = c0[:n], r[:n]
    c1 = _moved(c0, 0.3, 7)
    s = eb.Scene(c0, r)
    nodes_before = s.info.n_nodes
    s.refit(c1)
    fresh = eb.Scene(c1, r)
    assert s.info.n_nodes == nodes_before
    for field in ('radius', 'scale', 'rmax'):
        assert getattr(s.info, field) == getattr(fresh.info, field)
    assert list(s.info.center) == list(fresh.info.center)
    _, a64, ids = _scene_arrays(s)
    expect = np.concatenate([c1, r[:, None]], axis=1)
    assert np.array_equal(a64, expect[ids])
    _check_boxes(s)


@pytest.mark.parametrize('precision', ['fp32', 'fp64'])
@pytest.mark.parametrize('sigma', [0.3, 3.0])
def test_refit_traces_and_pa_equal_a_rebuild(eb, precision, sigma):
    from ehss_b200 import workloads as W
    from ehss_b200.state import Spheres
    c0, r, _ = W.globule(900, 11)
    c1 = _moved(c0, sigma, 12)
    s = eb.Scene(c0, r)
    s.refit(c1)
    fresh = eb.Scene(c1, r)
    _check_boxes(s)
    src = eb.external_source(Spheres(c1, r, False), 12, 190003, scene=fresh)
    got = eb.GPUEHSSTransport(s, precision=precision).trace(src, 64, record_history=True)
    ref = eb.GPUEHSSTransport(fresh, precision=precision).trace(src, 64, record_history=True)
    for name in ('positions', 'outgoing', 'escaped', 'unresolved', 'bounces', 'collider_ids'):
        assert np.array_equal(getattr(got, name), getattr(ref, name)), name
    idx = eb.SphereIndex(Spheres(c0, r, False))
    idx.refit(Spheres(c1, r, False))
    blocked, _, _ = idx.query(src)
    blocked_ref, _, _ = eb.SphereIndex(Spheres(c1, r, False)).query(src)
    assert np.array_equal(blocked, blocked_ref)


def test_batch_refit_blocks_equal_a_batch_build(eb):
    from ehss_b200 import workloads as W
    from ehss_b200.batch import BatchScenes
    from ehss_b200.blocks import BlockJob, BlockPlan
    sizes = [1, 9, 14, 40, 700, 2500]
    frames0 = [W.globule(n, 30 + i)[:2] if n > 1 else (np.zeros((1, 3)), np.array([1.7])) for i, n in enumerate(sizes)]
    frames1 = [(_moved(c, 0.3, 40 + i), r) for i, (c, r) in enumerate(frames0)]
    batch = BatchScenes(frames0)
    batch.build()
    batch.refit(frames1)
    fresh = BatchScenes(frames1)
    fresh.build()

    def blocks(b):
        plan = BlockPlan([BlockJob(sc, 12, 1000 + i, cap=64, pa=True) for i, sc in enumerate(b.scenes)])
        plan.run()
        return [(x['ehss_angstrom2'], x['collision_histogram'], x['pa_blocked_rays']) for x in plan.collect()]

    assert blocks(batch) == blocks(fresh)
    for i in range(len(sizes)):
        assert batch.info(i).radius == fresh.info(i).radius


def test_refit_refusals(eb):
    from ehss_b200 import _lib, workloads as W
    from ehss_b200.batch import BatchScenes
    from ehss_b200.state import Spheres
    c, r, _ = W.globule(300, 2)
    with pytest.raises(ValueError, match='fixed primitive identities'):
        eb.Scene(c, r).refit(c[:-1])
    with pytest.raises(ValueError, match='fixed primitive identities'):
        eb.SphereIndex(Spheres(c, r, False)).refit(Spheres(c[:-1], r[:-1], False))
    with pytest.raises(ValueError, match='exterior'):
        eb.Scene(c, r, exterior=True).refit(c)
    with pytest.raises(ValueError, match='exterior'):
        BatchScenes([(c, r)], exterior=True).refit([(c, r)])
    with pytest.raises(ValueError, match='positive finite'):
        eb.Scene(c, r).refit(c, -r)
    # the device check: the C entry point given an exterior scene marks it invalid
    ext = eb.Scene(c, r, exterior=True)
    import torch
    lib = _lib.load()
    xyz = torch.tensor(c, dtype=torch.float64, device='cuda')
    rad = torch.tensor(r, dtype=torch.float64, device='cuda')
    sb, wb = ct.c_uint64(), ct.c_uint64()
    _lib.check(lib.ehss_scene_bytes(len(r), 14, ct.byref(sb), ct.byref(wb)))
    ws = torch.empty(wb.value + 256, dtype=torch.uint8, device='cuda')
    _lib.check(lib.ehss_scenes_refit(1, (ct.c_void_p * 1)(xyz.data_ptr()), (ct.c_void_p * 1)(rad.data_ptr()),
                                     (ct.c_int64 * 1)(len(r)), (ct.c_void_p * 1)(ext.ptr),
                                     (ws.data_ptr() + 255) & ~255, wb.value, None))
    info = _lib.SceneInfo()
    assert lib.ehss_scene_info_get(ext.ptr, ct.byref(info), None) == _lib.ERR_VALUE
    assert b'refit requires a full' in lib.ehss_last_error()


def test_refit_after_rigid_rotation_on_varied_shapes(eb):
    """A rotated and translated copy refit into the old topology traces like a
    rebuilt scene (per-ray outcomes) on clouds, rods, sheets and split clusters."""
    from ehss_b200.state import Spheres
    from test_gpu_batched import _shapes
    rot = np.array([[0., -1., 0.], [1., 0., 0.], [0., 0., 1.]])
    for i, (c0, r) in enumerate(_shapes(606)[:6]):
        c1 = c0 @ rot.T + [7.5, -3.0, 120.0]
        s = eb.Scene(c0, r)
        s.refit(c1)
        fresh = eb.Scene(c1, r)
        _check_boxes(s)
        src = eb.external_source(Spheres(c1, r, False), 11, 60 + i, scene=fresh)
        got = eb.GPUEHSSTransport(s).trace(src, 64, record_history=True)
        ref = eb.GPUEHSSTransport(fresh).trace(src, 64, record_history=True)
        for name in ('positions', 'outgoing', 'escaped', 'unresolved', 'bounces', 'collider_ids'):
            assert np.array_equal(getattr(got, name), getattr(ref, name)), (i, name)
