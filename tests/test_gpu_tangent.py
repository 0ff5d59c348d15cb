"""Near-tangent rays through the FP32 filter.

Each ray is built to pass one surface sphere at perpendicular distance
r (1 + delta), delta in {0, +-2^-40, +-2^-30, +-2^-26, +-2^-24, +-2^-22,
+-2^-20, +-2^-16}, starting 2 S from the structure's centre.  The filter's
certain-miss, certain-hit and grazing classes rest on error bounds (the fused
kernel's short discriminant under its widened bound, the interval from one
reciprocal square root); on these rays the FP32 and FP64 forms must give the
same outcomes as each other and as the oracle:

* in the fused kernel, as caller-made ray blocks (EHSS_BLOCK_RAYS): identical
  integer results (CCS fixed-point sum, histogram, escaped/unresolved/hit
  counts) in both precisions, and the oracle's read-out;
* in the explicit-ray kernel: identical per-ray outcomes in both precisions
  and equal to the oracle ray by ray."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
DELTAS = [0.0] + [s * 2.0 ** -e for e in (40, 30, 26, 24, 22, 20, 16) for s in (1, -1)]


@pytest.fixture(scope='module')
def eb():
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    import ehss_b200
    return ehss_b200


def _tangent_rays(c, r, center, S, n, seed):
    """n rays, each tangent (up to r * delta) to a sphere near the surface."""
    rng = np.random.default_rng(seed)
    reach = np.linalg.norm(c - center, axis=1) + r
    surface = np.flatnonzero(reach >= 0.85 * reach.max())
    k = rng.choice(surface, n)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    e = rng.normal(size=(n, 3))
    e -= np.sum(e * d, axis=1, keepdims=True) * d
    e /= np.linalg.norm(e, axis=1, keepdims=True)
    delta = np.asarray(DELTAS)[np.arange(n) % len(DELTAS)]
    p = c[k] + (r[k] * (1.0 + delta))[:, None] * e
    # start behind the tangent point, 2 S from the centre (outside every sphere)
    q = p - center
    b = np.sum(q * d, axis=1)
    L = b + np.sqrt(b * b - np.sum(q * q, axis=1) + 4.0 * S * S)
    o = p - L[:, None] * d
    return o, d


class _CallerRays:
    """Caller-made rays for a fused block (the interface blocks.BlockPlan reads
    from a boundary): origins, directions and unit weights."""

    def __init__(self, o, d):
        self.o, self.d = o, d

    def fill_ray_buffer(self, power, seed, buf):
        import torch
        n = 1 << int(power)
        host = np.concatenate([self.o.ravel(), self.d.ravel(), np.ones(n)])
        buf[:7 * n].copy_(torch.from_numpy(host).to(buf.device))

    def max_projected_area(self):
        return float(len(self.o)) * (1.0 + 1e-9)


def test_tangent_rays_fused_blocks_fp32_equal_fp64_and_oracle(eb):
    from ehss_b200 import workloads as W
    from ehss_b200.blocks import BlockJob, BlockPlan
    from ehss_b200 import _lib
    c, r, _ = W.globule(2000, 5)
    scene = eb.Scene(c, r)
    center, S = np.asarray(scene.center), float(scene.radius)
    log2 = 13
    o, d = _tangent_rays(c, r, center, S, 1 << log2, 41)
    assert (np.linalg.norm(o[:, None, :] - c[None, :, :], axis=2) - r[None, :]).min() > 0
    rays = _CallerRays(o, d)
    jobs = [BlockJob(scene, log2, 0, cap=64, precision=p, boundary=rays, tag=p)
            for p in (_lib.PREC_FP32, _lib.PREC_FP64)]
    plan = BlockPlan(jobs)
    plan.run()
    f32, f64 = plan.collect()
    keys = ('ehss_angstrom2', 'collision_histogram', 'unresolved_rays', 'escaped_rays')
    assert {k: f32[k] for k in keys} == {k: f64[k] for k in keys}
    assert f32['stats'][_lib.STAT_GRAZING] > 0          # the filter did meet near-tangent tests
    ref = O.StaticTree(c, r, 4).trace(o, d, cap=64, threads=O.host_cores())
    ro = O.readout(dict(incoming=d, weights=np.ones(len(o))), ref, 64)
    assert f32['collision_histogram'] == ro['collision_histogram']
    assert f32['unresolved_rays'] == ro['unresolved_rays']
    assert f32['ehss_angstrom2'] == pytest.approx(ro['ehss_angstrom2'], rel=1e-12)


def test_tangent_rays_explicit_kernel_per_ray(eb):
    from ehss_b200 import workloads as W
    c, r, _ = W.globule(2000, 5)
    s = eb.Spheres(c, r, deduplicate=False)
    prep = eb.PreparedStaticGPUEHSS(s, precision='fp32')
    center, S = np.asarray(prep.scene.center), float(prep.scene.radius)
    o, d = _tangent_rays(c, r, center, S, 1 << 13, 43)
    n = len(o)
    src = eb.EHSSSource(o, d, d.copy(), np.ones(n), np.full(n, -1, dtype=np.int64), np.zeros(n, dtype=np.int64),
                        'near-tangent rays')
    a = prep.engine.trace(src, 64, record_history=True)
    b = eb.GPUEHSSTransport(prep.scene, precision='fp64').trace(src, 64, record_history=True)
    ref = O.StaticTree(c, r, 4).trace(o, d, cap=64, record=True, threads=O.host_cores())
    for field in ('positions', 'outgoing', 'escaped', 'unresolved', 'bounces', 'collider_ids'):
        np.testing.assert_array_equal(getattr(a, field), getattr(b, field), err_msg=field)
        np.testing.assert_array_equal(getattr(a, field), ref[field], err_msg=field)
    assert a.metrics['grazing_queries'] > 0
