"""Deterministic synthetic colonies for benchmarks and scale tests.

A grown colony of radius R holds about 4.4 R^2 rod-shaped cells (301,116 cells
at R = 260 in the reference's published runs) packed at roughly 0.9, in
orientation domains of a few cell lengths.  `dense_colony` lays out such a
state directly instead of growing it for hours: the disc is tiled into square
patches with one random orientation each; inside a patch, cells sit in
parallel lanes one diameter apart, end to end with small gaps, with lengths
drawn uniformly from [l0, 2 l0) (the spread of a dividing population).  Cells
that would cross a patch edge or the disc edge are dropped, so the initial
state has no overlap; every side-by-side and end-to-end neighbour is within
the phase-0 detection reach, so the first step builds the full contact
network and growth drives the ReLCP / BBPGD solver from there on.
"""
from __future__ import annotations

import numpy as np


def dense_colony(radius: float, seed: int = 0, l0: float = 1.0, patch: float = 12.0, lane_gap: float = 0.01,
                 end_gap: float = 0.02, angle_jitter: float = 1e-6) -> dict:
    """Cells of one patch share the patch orientation up to a uniform jitter of
    +-angle_jitter radians per cell.  Exactly parallel neighbours make the
    segment-distance determinant a*c - b^2 pure rounding noise, so their
    closest points (and the reference's, which take the pair in hash-map
    order) depend on the order the two segments are taken in; the jitter keeps
    every pair away from that case."""
    rng = np.random.default_rng(seed)
    jit = np.random.default_rng(seed + 7919)
    d = l0 / 2
    xs, ys, ths, ls = [], [], [], []
    n_p = int(np.ceil(radius / patch)) + 1
    margin = 0.02
    for px in range(-n_p, n_p):
        for py in range(-n_p, n_p):
            cx0, cy0 = px * patch, py * patch
            # skip patches entirely outside the disc
            nearest = np.hypot(np.clip(0.0, cx0, cx0 + patch), np.clip(0.0, cy0, cy0 + patch))
            if nearest > radius:
                continue
            th = rng.uniform(0.0, np.pi)
            t = np.array([np.cos(th), np.sin(th)])
            nrm = np.array([-t[1], t[0]])
            center = np.array([cx0 + patch / 2, cy0 + patch / 2])
            half = patch * 0.71
            lane = -half
            while lane <= half:
                s = -half + rng.uniform(0.0, 1.0)
                while s <= half:
                    L = rng.uniform(l0, 2 * l0 - 1e-6)
                    c = center + nrm * lane + t * (s + L / 2)
                    # rod footprint: segment +- (L/2 - d/2) t, radius d/2
                    a = L / 2 - d / 2
                    ends = np.array([c - a * t, c + a * t])
                    lo = np.array([cx0, cy0]) + d / 2 + margin
                    hi = np.array([cx0 + patch, cy0 + patch]) - d / 2 - margin
                    inside_patch = np.all(ends >= lo) and np.all(ends <= hi)
                    inside_disc = np.all(np.hypot(ends[:, 0], ends[:, 1]) + d / 2 <= radius)
                    if inside_patch and inside_disc:
                        xs.append(c[0])
                        ys.append(c[1])
                        ths.append(th + jit.uniform(-angle_jitter, angle_jitter))
                        ls.append(L)
                    s += L + end_gap
                lane += d + lane_gap
    n = len(xs)
    ths = np.asarray(ths)
    return {
        "x": np.asarray(xs), "y": np.asarray(ys), "z": np.zeros(n),
        "q0": np.cos(ths / 2), "q1": np.zeros(n), "q2": np.zeros(n), "q3": np.sin(ths / 2),
        "length": np.asarray(ls), "l0": np.full(n, l0), "diameter": np.full(n, d),
        "age": np.ones(n, np.int32),
    }


def min_separation(cells: dict, sample: int = 2000, seed: int = 0) -> float:
    """Smallest surface separation between a random sample of cells and all
    cells (brute force over a neighbourhood; for tests of the generator)."""
    rng = np.random.default_rng(seed)
    n = len(cells["x"])
    idx = rng.choice(n, size=min(sample, n), replace=False)
    th = 2 * np.arctan2(cells["q3"], cells["q0"])
    t = np.stack([np.cos(th), np.sin(th)], 1)
    p = np.stack([cells["x"], cells["y"]], 1)
    a = (cells["length"] / 2 - cells["diameter"] / 2)[:, None]
    P0, P1 = p - a * t, p + a * t
    best = np.inf
    for i in idx:
        near = np.nonzero(np.hypot(*(p - p[i]).T) < 3.0)[0]
        near = near[near != i]
        for j in near:
            best = min(best, _seg_dist(P0[i], P1[i], P0[j], P1[j]) - cells["diameter"][i] / 2 - cells["diameter"][j] / 2)
    return float(best)


def _seg_dist(p0, p1, q0, q1) -> float:
    # brute-force sampled segment distance (test helper only)
    s = np.linspace(0, 1, 41)
    a = p0[None, :] + s[:, None] * (p1 - p0)[None, :]
    b = q0[None, :] + s[:, None] * (q1 - q0)[None, :]
    return float(np.min(np.hypot(*(a[:, None, :] - b[None, :, :]).reshape(-1, 2).T)))
