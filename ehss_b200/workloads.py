"""Seeded synthetic structures for the cross-section workloads.

No benchmark suite or dataset is needed: the workloads are generated here.

* ``triatomic()``      bent triatomic: O at the origin, two H at 0.9572 A,
                       104.52 degrees apart.
* ``globule(n, seed)`` random sequential addition inside an ellipsoid of
                       semi-axis ratio 1 : 0.85 : 0.75 scaled to 0.1 atoms/A^3,
                       minimum pair distance 1.0 A, elements H/C/N/O/S drawn
                       with fractions 0.49/0.32/0.09/0.09/0.01.
* ``mixed_batch(...)`` many globules with log-uniform atom counts and ray
                       budgets (the batched form).
* ``request_stream``   Poisson arrivals of globules or perturbed frames of one
                       ensemble (the served form).

Radii are the reference CLI's van der Waals table plus the 1.4 A He probe
(src/support_exchange_transport/ccs_cli.py:29-31, :120).
"""
from __future__ import annotations

import math

import numpy as np

VDW_RADII = {"H": 1.10, "He": 1.40, "C": 1.70, "N": 1.55, "O": 1.52, "F": 1.47, "Si": 2.10, "P": 1.80,
             "S": 1.80, "Cl": 1.75, "Se": 1.90, "Br": 1.83, "I": 1.98}
PROBE = 1.4
ELEMENTS = ("H", "C", "N", "O", "S")
FRACTIONS = (0.49, 0.32, 0.09, 0.09, 0.01)
DENSITY = 0.1
AXES = np.array([1.0, 0.85, 0.75])
MIN_DIST = 1.0


def radii_for(elements, probe=PROBE):
    return np.array([VDW_RADII[e] + probe for e in elements])


def triatomic():
    angle = np.deg2rad(104.52)
    xyz = np.array([[0., 0., 0.], [0.9572, 0., 0.], [0.9572 * np.cos(angle), 0.9572 * np.sin(angle), 0.]])
    elements = ("O", "H", "H")
    return xyz, radii_for(elements), elements


def random_rotation(seed):
    """Uniform rotation on SO(3) from a seeded unit quaternion."""
    q = np.random.default_rng(seed).normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def globule(n, seed):
    """RSA globule of n atoms; returns (centers [n,3], radii [n], elements)."""
    from scipy.spatial import cKDTree
    rng = np.random.default_rng(seed)
    n = int(n)
    elements = tuple(rng.choice(ELEMENTS, size=n, p=FRACTIONS))
    volume = n / DENSITY
    a = (volume / (4.0 / 3.0 * math.pi * AXES.prod())) ** (1.0 / 3.0)
    semi = a * AXES
    accepted = np.empty((0, 3))
    tree = None
    while len(accepted) < n:
        need = n - len(accepted)
        m = max(64, int(need * 1.3))
        # uniform in the ellipsoid: uniform in the unit ball, scaled per axis
        v = rng.normal(size=(m, 3))
        v /= np.linalg.norm(v, axis=1)[:, None]
        v *= rng.random(m)[:, None] ** (1.0 / 3.0)
        cand = v * semi
        if tree is not None:
            dist, _ = tree.query(cand, k=1, distance_upper_bound=MIN_DIST)
            cand = cand[~(dist < MIN_DIST)]
        # sequential acceptance inside the batch, in proposal order
        keep = np.ones(len(cand), dtype=bool)
        if len(cand) > 1:
            pairs = cKDTree(cand).query_pairs(MIN_DIST - 1e-12, output_type='ndarray')
            if len(pairs):
                pairs = pairs[np.lexsort((pairs[:, 0], pairs[:, 1]))]
                for i, j in pairs:          # i < j: the later proposal loses to an earlier kept one
                    if keep[i] and keep[j]:
                        keep[j] = False
        cand = cand[keep][:need]
        accepted = np.vstack([accepted, cand])
        tree = cKDTree(accepted)
    return accepted, radii_for(elements), elements


def mixed_batch(count=256, seed=2026, n_range=(20, 5000), log2_range=(14, 18)):
    """[(n_atoms, log2_rays, structure_seed)] for the batched form."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(round(math.exp(rng.uniform(math.log(n_range[0]), math.log(n_range[1])))))
        log2 = int(round(rng.uniform(*log2_range)))
        out.append((n, log2, int(rng.integers(0, 2 ** 31))))
    return out


def ensemble_frame(base, frame, sigma=0.3, seed=0):
    """Frame `frame` of an ensemble: base centres plus i.i.d. N(0, sigma^2)."""
    rng = np.random.default_rng([seed, frame])
    return base + rng.normal(scale=sigma, size=base.shape)


def request_stream(count, rate=200.0, seed=7, n_range=(10, 20000), ensemble_atoms=1500, frames=1000):
    """Poisson arrivals: [(arrival_s, kind, n_atoms or frame, structure_seed)]."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for _ in range(count):
        t += rng.exponential(1.0 / rate)
        if rng.random() < 0.5:
            n = int(round(math.exp(rng.uniform(math.log(n_range[0]), math.log(n_range[1])))))
            out.append((t, 'globule', n, int(rng.integers(0, 2 ** 31))))
        else:
            out.append((t, 'frame', int(rng.integers(0, frames)), int(rng.integers(0, 2 ** 31))))
    return out
