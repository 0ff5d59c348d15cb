"""Host-side logic that needs no GPU: the C ABI loads and exports what the
header declares, the host Sobol scrambler is bit-exact, block preparation,
argument validation, workload generators and the reference data types."""
import ctypes as ct

from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O


@pytest.fixture(scope='module')
def lib():
    from ehss_b200 import _lib
    return _lib.load()


def test_library_exports_every_header_function(lib):
    from ehss_b200 import _lib
    declared = _lib.header_functions()
    assert len(declared) >= 15
    for name in declared:
        assert hasattr(lib, name), name
    assert set(declared) == set(_lib._SIGNATURES), 'ctypes table and header differ'
    assert lib.ehss_abi_version() == 1


@pytest.mark.parametrize('dim', [1, 2, 4, 5, 8])
def test_host_sobol_scramble_bit_exact(lib, dim):
    for seed in (0, 1, 98, 190003, 2 ** 32 - 1, 2 ** 40 + 5, 2 ** 64 - 1):
        sv = (ct.c_uint32 * (dim * 30))(); sh = (ct.c_uint32 * dim)()
        assert lib.ehss_sobol_scramble(dim, seed, sv, sh) == 0
        ref_sv, ref_sh = O.sobol_scramble(dim, seed)
        np.testing.assert_array_equal(np.array(sv[:]).reshape(dim, 30), ref_sv)
        np.testing.assert_array_equal(np.array(sh[:]), ref_sh)


def test_host_sobol_against_golden_scrambles(lib, golden):
    g = golden('sobol.npz')
    for key in sorted({k.rsplit('_', 1)[0] for k in g if k.startswith('d')}):
        d, m, s = (int(part[1:]) for part in key.split('_'))
        sv = (ct.c_uint32 * (d * 30))(); sh = (ct.c_uint32 * d)()
        assert lib.ehss_sobol_scramble(d, s, sv, sh) == 0
        np.testing.assert_array_equal(np.array(sv[:]).reshape(d, 30), g[key + '_sv'])
        np.testing.assert_array_equal(np.array(sh[:]), g[key + '_shift'])


def test_argument_validation_without_device(lib):
    from ehss_b200 import _lib
    sb, wb = ct.c_uint64(), ct.c_uint64()
    assert lib.ehss_scene_bytes(0, 4, ct.byref(sb), ct.byref(wb)) == _lib.ERR_VALUE
    assert b'atom count' in lib.ehss_last_error()
    assert lib.ehss_scene_bytes(10, 17, ct.byref(sb), ct.byref(wb)) == _lib.ERR_VALUE
    assert lib.ehss_scene_bytes(1000, 4, ct.byref(sb), ct.byref(wb)) == 0
    assert sb.value % 256 == 0 and sb.value >= 256 + 999 * 64 + 1000 * (16 + 32 + 8)
    sv = (ct.c_uint32 * 300)(); sh = (ct.c_uint32 * 10)()
    assert lib.ehss_sobol_scramble(9, 0, sv, sh) == _lib.ERR_VALUE
    assert lib.ehss_trace(None, 1, 0, 1, *([None] * 8), None) == _lib.ERR_VALUE
    one = (ct.c_void_p * 1)(1024)
    assert lib.ehss_scenes_build_ex(1, one, one, (ct.c_int64 * 1)(10), 8, one, (ct.c_uint64 * 1)(1 << 20), 1024,
                                    1 << 20, 2, None) == _lib.ERR_VALUE
    assert b'unknown build flags' in lib.ehss_last_error()
    wb = ct.c_uint64()
    assert lib.ehss_scenes_workspace_bytes(3, (ct.c_int64 * 3)(1 << 30, 1 << 30, 1 << 30), ct.byref(wb)) == _lib.ERR_VALUE
    assert b'at most' in lib.ehss_last_error()
    assert lib.ehss_scenes_build_ex(0, one, one, (ct.c_int64 * 1)(10), 8, one, (ct.c_uint64 * 1)(1 << 20), 1024,
                                    1 << 20, 1, None) == _lib.ERR_VALUE
    with pytest.raises(ValueError):
        _lib.check(_lib.ERR_VALUE)
    # a chunk window must lie inside the prepared chunk list (checked before any device work)
    L = _lib.Launch(128, 8, 256, 28, 0, 0, 5, 0)
    ws = (ct.c_uint64 * 512)()
    for first, end in ((5, 3), (-1, 2), (0, 11)):
        rc = lib.ehss_trace_blocks_window(ct.c_void_p(1024), 1, 10, first, end, ct.c_void_p(1024), ct.c_void_p(1024),
                                          ct.c_void_p(1024), 1, ws, ct.sizeof(ws), ct.byref(L), None)
        assert rc == _lib.ERR_VALUE and b'chunk window' in lib.ehss_last_error()


def test_noalloc_limit_fits_the_fixed_scratch_array(lib):
    """The allocation-free build's stated maximum (EHSS_NOALLOC_MAX_ATOMS)
    must fit its fixed 4 MiB workspace; the workspace size is host arithmetic
    (the builder's own sort has no size that depends on a library version)."""
    limit = 20000
    sb, wb = ct.c_uint64(), ct.c_uint64()
    assert lib.ehss_scene_bytes(limit, 16, ct.byref(sb), ct.byref(wb)) == 0
    assert wb.value <= 4 << 20
    header = (Path(__file__).resolve().parents[1] / 'include' / 'ehss_b200.h').read_text()
    assert f'#define EHSS_NOALLOC_MAX_ATOMS {limit}' in header


def test_blocks_prepare_chunks_and_offsets(lib):
    from ehss_b200 import _lib
    n = 3
    blocks = (_lib.Block * n)()
    for i, (log2, cap) in enumerate([(12, 64), (5, 1), (14, 7)]):
        blocks[i].scene = 0x1000 * (i + 1)
        blocks[i].log2_rays = log2
        blocks[i].cap = cap
        blocks[i].precision = 1
        blocks[i].flags = _lib.BLOCK_EHSS
        blocks[i].hist_offset = -1
    seeds = (ct.c_uint64 * n)(0, 1, 2)
    total = ct.c_int64()
    assert lib.ehss_blocks_prepare(blocks, n, seeds, 256, ct.byref(total)) == 0
    assert total.value == 16 + 1 + 64
    assert [b.chunk_begin for b in blocks] == [0, 16, 17]
    # the fixed-point angle sum of a block must stay below 2^63: at most 2^26 rays
    one = (_lib.Block * 1)()
    one[0].scene, one[0].cap, one[0].precision, one[0].flags, one[0].hist_offset = 0x1000, 8, 1, _lib.BLOCK_EHSS, -1
    one[0].log2_rays = 27
    assert lib.ehss_blocks_prepare(one, 1, (ct.c_uint64 * 1)(5), 256, ct.byref(total)) == _lib.ERR_VALUE
    one[0].log2_rays = 26
    assert lib.ehss_blocks_prepare(one, 1, (ct.c_uint64 * 1)(5), 256, ct.byref(total)) == 0
    assert total.value == (1 << 26) // 256
    assert [b.hist_offset for b in blocks] == [0, 65, 67]
    blocks[1].cap = 0
    assert lib.ehss_blocks_prepare(blocks, n, seeds, 256, ct.byref(total)) == _lib.ERR_VALUE
    assert lib.ehss_blocks_prepare(blocks, n, seeds, 100, ct.byref(total)) == _lib.ERR_VALUE


def test_struct_layouts_match_header():
    from ehss_b200 import _lib
    assert ct.sizeof(_lib.Block) == 560 and _lib.Block.basis.offset == 0 and _lib.Block.base.offset == 480
    assert ct.sizeof(_lib.BlockResult) == 8 * (8 + _lib.NSTATS)
    assert ct.sizeof(_lib.Launch) == 32
    assert ct.sizeof(_lib.SceneInfo) == 96 and _lib.SceneInfo.n_active.offset == 80


def test_workload_generators():
    from ehss_b200 import workloads as W
    from scipy.spatial import cKDTree
    c, r, e = W.globule(650, 4)
    assert c.shape == (650, 3) and len(e) == 650
    assert cKDTree(c).query(c, k=2)[0][:, 1].min() >= 1.0 - 1e-12
    c2, _, _ = W.globule(650, 4)
    np.testing.assert_array_equal(c, c2)
    set_r = set(np.round(r, 6))
    assert set_r <= {round(W.VDW_RADII[x] + 1.4, 6) for x in W.ELEMENTS}
    batch = W.mixed_batch(256, seed=1)
    ns = np.array([b[0] for b in batch]); logs = np.array([b[1] for b in batch])
    assert ns.min() >= 20 and ns.max() <= 5000 and set(logs) <= set(range(14, 19))
    R = W.random_rotation(5)
    np.testing.assert_allclose(R @ R.T, np.eye(3), atol=1e-12)
    assert np.linalg.det(R) == pytest.approx(1.0)
    xyz, rad, el = W.triatomic()
    assert np.linalg.norm(xyz[1] - xyz[0]) == pytest.approx(0.9572)
    assert list(rad) == [2.92, 2.5, 2.5]


def test_state_types_validate_like_reference():
    from ehss_b200 import EHSSSource, Spheres
    with pytest.raises(ValueError):
        Spheres(np.zeros((0, 3)), np.zeros(0))
    with pytest.raises(ValueError):
        Spheres(np.zeros((1, 3)), np.array([-1.]))
    s = Spheres(np.array([[0., 0, 0], [0., 0, 0]]), np.ones(2))
    assert len(s.radii) == 1
    d = np.array([[1., 0, 0]])
    with pytest.raises(ValueError):
        EHSSSource(np.zeros((1, 3)), 2 * d, d, np.ones(1), np.array([-1]), np.array([0]), 'x')
    with pytest.raises(ValueError):
        EHSSSource(np.zeros((1, 3)), d, d, np.ones(1), np.array([-1]), np.array([1]), 'x')


@pytest.mark.parametrize('m,seed', [(3, 0), (8, 190003), (12, 7), (14, 2 ** 32 - 1), (16, 104729)])
def test_coherent_enumeration_is_the_sobol_point_set(lib, m, seed):
    """Block descriptors enumerate exactly scipy's points, neighbours close."""
    from ehss_b200 import _lib
    blocks = (_lib.Block * 1)()
    blocks[0].scene = 0x1000
    blocks[0].log2_rays = m
    blocks[0].cap = 8
    blocks[0].precision = 1
    blocks[0].flags = _lib.BLOCK_EHSS
    blocks[0].hist_offset = -1
    total = ct.c_int64()
    assert lib.ehss_blocks_prepare(blocks, 1, (ct.c_uint64 * 1)(seed), 64, ct.byref(total)) == 0
    basis = np.array([[blocks[0].basis[e][j] for j in range(4)] for e in range(30)], dtype=np.uint32)
    base = np.array(blocks[0].base[:], dtype=np.uint32)
    p = np.arange(1 << m, dtype=np.uint64)
    pts = np.tile(base, (1 << m, 1))
    for e in range(m):
        sel = ((p >> np.uint64(e)) & np.uint64(1)).astype(bool)
        pts[sel] ^= basis[e]
    ref = O.sobol_integers(4, m, seed)
    got_sorted = np.lexsort(pts.T[::-1]); ref_sorted = np.lexsort(ref.T[::-1])
    np.testing.assert_array_equal(pts[got_sorted], ref[ref_sorted])
    if m >= 12:
        # the 32 positions of a warp share the leading digits of all four dimensions
        digits = (m - 5) // 4
        top = pts.reshape(-1, 32, 4) >> np.uint32(30 - digits)
        assert (top == top[:, :1, :]).all(axis=(1, 2)).mean() == 1.0


def test_block_readout_matches_per_block_formulas():
    """BlockPlan.collect's vectorised read-out against the per-block definitions
    omega = w angle_fx 2^-36, pa = w hits, tail = 2 w unresolved (host only)."""
    import torch
    from ehss_b200 import _lib
    from ehss_b200.blocks import BlockJob, BlockPlan, _RESULT_WORDS, _STATS0

    class FakeScene:
        ptr, radius, device, n_atoms = 0x10000, 12.5, torch.device('cpu'), 10

    spec = [(10, 1, 4, True), (12, 2, 8, False), (14, 3, 2, True)]
    jobs = [BlockJob(FakeScene(), lg, seed, cap=cap, pa=pa, tag=i) for i, (lg, seed, cap, pa) in enumerate(spec)]
    plan = BlockPlan(jobs, device=torch.device('cpu'))
    rng = np.random.default_rng(3)
    words = plan.packed.numpy().view(np.uint64)
    n = len(jobs)
    res = rng.integers(0, 2 ** 50, size=(n, _RESULT_WORDS), dtype=np.uint64)
    res[:, _STATS0 + _lib.STAT_ERRORS] = 0
    words[:n * _RESULT_WORDS] = res.ravel()
    words[n * _RESULT_WORDS:] = rng.integers(0, 2 ** 40, size=len(words) - n * _RESULT_WORDS, dtype=np.uint64)
    out = plan.collect()
    hist = words[n * _RESULT_WORDS:n * _RESULT_WORDS + plan.hist_len]
    ledger = words[n * _RESULT_WORDS + plan.hist_len:]
    off = 0
    for j, r, d in zip(jobs, res, out):
        w = np.pi * 12.5 * 12.5 / (1 << j.log2_rays)
        assert d['ehss_angstrom2'] == w * (int(r[0]) * _lib.FX_SCALE)
        assert d['pa_from_same_rays_angstrom2'] == w * int(r[1])
        assert d['tail_bound_angstrom2'] == 2 * w * int(r[2])
        assert d['collision_histogram'] == hist[off:off + j.cap + 1].astype(np.int64).tolist()
        assert d['collision_contribution_angstrom2'] == (ledger[off:off + j.cap + 1].astype(np.float64)
                                                          * _lib.FX_SCALE * w).tolist()
        assert ('pa_angstrom2' in d) == j.pa and (not j.pa or d['pa_angstrom2'] == w * int(r[4]))
        off += j.cap + 1
    res[1, _STATS0 + _lib.STAT_ERRORS] = 2
    words[:n * _RESULT_WORDS] = res.ravel()
    with pytest.raises(_lib.EHSSDeviceError):
        plan.collect()


def test_weighted_readout_of_boundary_blocks():
    """Blocks with caller-made weighted rays report hits, tail and PA from the
    weighted fixed-point sums; impact-disk blocks from counts (host only)."""
    import torch
    from ehss_b200 import _lib
    from ehss_b200.blocks import BlockJob, BlockPlan, _RESULT_WORDS, _STATS0

    class FakeScene:
        ptr, radius, device, n_atoms = 0x10000, 5.0, torch.device('cpu'), 10

    jobs = [BlockJob(FakeScene(), 10, 1, cap=4, pa=True, tag=0), BlockJob(FakeScene(), 10, 2, cap=4, pa=True, tag=1)]
    plan = BlockPlan(jobs, device=torch.device('cpu'))
    plan._weighted = np.array([False, True])          # block 1 as if its rays carried weights
    plan._w = np.array([plan._w[0], 0.25])
    words = plan.packed.numpy().view(np.uint64)
    res = np.zeros((2, _RESULT_WORDS), dtype=np.uint64)
    res[:, 0] = 3 << 36                                 # angle sums
    res[:, 1], res[:, 2], res[:, 4] = 7, 2, 5           # counts
    res[:, 5], res[:, 6], res[:, 7] = 6 << 35, 1 << 36, 9 << 34   # weighted sums: 3.0, 1.0, 2.25
    words[:2 * _RESULT_WORDS] = res.ravel()
    a, b = plan.collect()
    w0 = plan._w[0]
    assert a['pa_from_same_rays_angstrom2'] == w0 * 7 and a['tail_bound_angstrom2'] == 2 * w0 * 2
    assert a['pa_angstrom2'] == w0 * 5 and a['ehss_angstrom2'] == w0 * 3.0
    assert b['pa_from_same_rays_angstrom2'] == 0.25 * 3.0 and b['tail_bound_angstrom2'] == 2 * 0.25 * 1.0
    assert b['pa_angstrom2'] == 0.25 * 2.25 and b['ehss_angstrom2'] == 0.25 * 3.0
    assert b['unresolved_rays'] == 2 and b['collision_histogram'] == [0] * 5
    t = plan.totals(plan.fetch())
    assert list(t['tail']) == [2 * w0 * 2, 2 * 0.25 * 1.0] and list(t['pa']) == [w0 * 5, 0.25 * 2.25]


def test_cap_extension_merge():
    """A block at cap 4 with 3 unresolved rays continued to cap 8: two escape
    (at 5 and 7 bounces), one is still unresolved at 8 (host only)."""
    from ehss_b200.blocks import merge_extension
    st = dict(cap=4, angle_fx=100, escaped=10, unresolved=3, hist=[5, 3, 2, 0, 3], ledger=[0, 40, 60, 0, 0])
    hist = [0] * 9; ledger = [0] * 9
    hist[5], hist[7], hist[8] = 1, 1, 1
    ledger[5], ledger[7] = 11, 13
    cont = merge_extension(st, (24, 2, 1, 3), hist, ledger, 8)
    assert cont == 3 and st['cap'] == 8
    assert st['hist'] == [5, 3, 2, 0, 0, 1, 0, 1, 1] and sum(st['hist']) == 13
    assert st['ledger'] == [0, 40, 60, 0, 0, 11, 0, 13, 0]
    assert (st['angle_fx'], st['escaped'], st['unresolved']) == (124, 12, 1)


def test_enclosing_radius_matches_the_reference_formula(lib):
    """ehss_enclosing_radius (host) equals external_source's R = max(|c - mean| + r) * (1 + 1e-9)
    (ehss_state.py:46-47, numpy operation order) bit for bit."""
    from ehss_b200 import _lib
    from ehss_b200.batch import enclosing_radius
    for s in range(200):
        rng = np.random.default_rng(s)
        n = int(rng.integers(1, 2000))
        c = rng.normal(0, 10 ** rng.uniform(-2, 3), (n, 3)) + rng.normal(0, 10 ** rng.uniform(-2, 4), 3)
        r = rng.uniform(0.5, 3, n)
        center = c.mean(axis=0)
        ref = float(np.max(np.linalg.norm(c - center, axis=1) + r)) * (1. + 1e-9)
        assert enclosing_radius(c, r) == ref
    out = ct.c_double()
    assert lib.ehss_enclosing_radius(0, None, None, ct.byref(out)) == _lib.ERR_VALUE
