"""The FP32 filter's discriminant bounds, checked on the host.

The device's FILTER tests classify a sphere as a certain miss, a certain hit
or a grazing candidate by comparing an FP32 discriminant with a per-ray bound
Edisc (trace.cu: setup_ray; the fused kernel's shorter form adds
kWidenShortDisc (rmax^2 + A^2)).  Here the same FP32 operation sequences are
replayed in numpy (float32 arithmetic, fma as an exact float64 product and
sum rounded once to float32) on rays built to pass spheres near tangency,
and the computed discriminants are compared with the discriminant of the
FP64 ray (the reference's projection form, evaluated in extended precision):
every error must stay inside its bound.  Host logic only: no device."""
import numpy as np

U32 = 2.0 ** -24


def _f(x):
    return np.asarray(x, dtype=np.float32)


def _fma(a, b, c):
    """fmaf: exact product and sum of float32 inputs, rounded once to float32
    (the float64 sum is exact whenever the float32 result is not a tie)."""
    return (a.astype(np.float64) * b.astype(np.float64) + c.astype(np.float64)).astype(np.float32)


def _rays(n, seed, S=30.0):
    rng = np.random.default_rng(seed)
    r = rng.uniform(1.6, 3.4, n)
    c = rng.normal(size=(n, 3))
    c *= (rng.uniform(0.0, 1.0, n) ** (1 / 3) * (S - r) / np.linalg.norm(c, axis=1))[:, None]
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    e = rng.normal(size=(n, 3))
    e -= np.sum(e * d, axis=1, keepdims=True) * d
    e /= np.linalg.norm(e, axis=1, keepdims=True)
    delta = rng.choice([0.0, 1e-7, -1e-7, 1e-5, -1e-5, 1e-3, -1e-3, 0.3, -0.5], n)
    p = c + (r * (1 + delta))[:, None] * e
    back = rng.uniform(0.2, 2.0, n) * S
    o = p - back[:, None] * d
    keep = np.linalg.norm(o, axis=1) <= 3.0 * S
    return o[keep], d[keep], c[keep], r[keep], S


def _exact_disc(o, d, c, r):
    """r^2 - |x - (x.d / d.d) d|^2 of the FP64 ray, in extended precision."""
    o, d, c, r = (np.asarray(v, dtype=np.longdouble) for v in (o, d, c, r))
    x = o - c
    proj = np.sum(x * d, axis=1) / np.sum(d * d, axis=1)
    p = x - proj[:, None] * d
    return r * r - np.sum(p * p, axis=1)


def _bounds(o32, S, rmax):
    a = np.sqrt(_fma(o32[:, 0], o32[:, 0], _fma(o32[:, 1], o32[:, 1], o32[:, 2] * o32[:, 2])))
    A = _f(a + _f(S))
    Ep = _f(A * _f(32 * U32))
    rm = _f(rmax)
    Edisc = _f(_f(_f(8 * U32) * rm * rm) + _f(_f(2.5) * rm * Ep) + _f(_f(8.0) * Ep * Ep))
    wide = _f(Edisc + _f(_f(16 * U32) * _f(rm * rm + A * A)))
    return Edisc, wide


def test_fp32_discriminants_stay_inside_their_bounds():
    o, d, c, r, S = _rays(400_000, 2024)
    rmax = float(r.max())
    o32, d32, c32, r32 = _f(o), _f(d), _f(c), _f(r)
    vx, vy, vz = (c32[:, i] - o32[:, i] for i in range(3))
    b = _fma(vx, d32[:, 0], _fma(vy, d32[:, 1], vz * d32[:, 2]))
    # cancellation-free form (explicit-ray and any-hit kernels)
    px, py, pz = (_fma(-b, d32[:, i], v) for i, v in enumerate((vx, vy, vz)))
    q = _fma(px, px, _fma(py, py, pz * pz))
    disc_cf = _fma(r32, r32, -q)
    # short form (fused kernel)
    w = _fma(-vx, vx, _fma(-vy, vy, _fma(-vz, vz, r32 * r32)))
    disc_short = _fma(b, b, w)
    Edisc, wide = _bounds(o32, S, rmax)
    true = _exact_disc(o, d, c, r)
    # the bounds matter where a classification depends on them: true disc >= 0,
    # or a computed disc >= 2 Edisc (certain hit)
    for disc, bound in ((disc_cf, Edisc), (disc_short, wide)):
        err = np.abs(disc.astype(np.longdouble) - true)
        rel = (err / bound.astype(np.longdouble))[(true >= 0) | (disc >= 2 * bound)]
        assert rel.size > 100_000
        assert float(rel.max()) < 1.0, float(rel.max())
    # the tests near tangency do occur: true discriminants inside the grazing band
    assert np.count_nonzero(np.abs(true) < 2 * wide) > 1000


def test_certain_hit_interval_covers_the_reciprocal_square_root():
    """Et = 2 (Ep + Edisc y) + 8u (|b| + s), s = disc y, with y within 2 ulp of
    1/sqrt(disc): the interval holds the entry distance of the FP64 ray for
    every y in that range (both ends of it tried)."""
    o, d, c, r, S = _rays(200_000, 7)
    rmax = float(r.max())
    o32, d32, c32, r32 = _f(o), _f(d), _f(c), _f(r)
    vx, vy, vz = (c32[:, i] - o32[:, i] for i in range(3))
    b = _fma(vx, d32[:, 0], _fma(vy, d32[:, 1], vz * d32[:, 2]))
    w = _fma(-vx, vx, _fma(-vy, vy, _fma(-vz, vz, r32 * r32)))
    disc = _fma(b, b, w)
    Edisc, wide = _bounds(o32, S, rmax)
    a = np.sqrt(_fma(o32[:, 0], o32[:, 0], _fma(o32[:, 1], o32[:, 1], o32[:, 2] * o32[:, 2])))
    Ep = _f(_f(a + _f(S)) * _f(32 * U32))
    sel = disc >= 2 * wide
    true_disc = _exact_disc(o, d, c, r)
    ol, dl, cl = (np.asarray(v, dtype=np.longdouble) for v in (o, d, c))
    x = cl - ol
    t_true = np.sum(x * dl, axis=1) / np.sum(dl * dl, axis=1) - np.sqrt(np.maximum(true_disc, 0))
    for ulps in (-2.0, 2.0):
        y = _f(1.0 / np.sqrt(disc[sel].astype(np.float64)) * (1.0 + ulps * 2.0 ** -23))
        s = _f(disc[sel] * y)
        t = _f(b[sel] - s)
        Et = _f(_f(2.0) * _f(Ep[sel] + _f(wide[sel] * y)) + _f(_f(8 * U32) * _f(np.abs(b[sel]) + s)))
        gap = np.abs(t.astype(np.longdouble) - t_true[sel]) / Et.astype(np.longdouble)
        assert float(gap.max()) < 1.0, float(gap.max())
