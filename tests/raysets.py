"""Seeded ray sets for traversal parity tests (shared by CPU and GPU tests)."""
from __future__ import annotations

import os

import numpy as np

from rednoise_b200.scenes import glm_normalize

ASSETS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "assets")


def fan_rays():
    """The reference's testBVH fan (tests/tests.cpp:174-197): 20 x 20 rays from (0, 0, 4)."""
    i = np.arange(400)
    a = (i % 20).astype(np.float32) / np.float32(20.0) - np.float32(0.5)
    b = (i // 20).astype(np.float32) / np.float32(20.0) - np.float32(0.5)
    d = glm_normalize(np.stack([a, b, -np.ones(400, np.float32)], 1))
    o = np.tile(np.array([0.0, 0.0, 4.0], np.float32), (400, 1))
    return o, d


def random_rays(n: int, seed: int, lo, hi, axis_fraction: float = 0.1):
    """Origins uniform in the box [lo, hi]; directions uniform on the sphere
    (normalised with glm's float order); a fraction snapped to axis-aligned or
    planar directions (exact zero components) to exercise the slab test's
    inf / NaN paths."""
    rng = np.random.default_rng(seed)
    lo = np.asarray(lo, np.float32)
    hi = np.asarray(hi, np.float32)
    o = (lo + (hi - lo) * rng.random((n, 3))).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    k = int(n * axis_fraction)
    if k:
        sel = rng.choice(n, size=k, replace=False)
        zero = rng.integers(0, 3, size=(k, 2))
        d[sel, zero[:, 0]] = 0.0
        half = sel[: k // 2]
        d[half, zero[: k // 2, 1]] = 0.0
        d[sel[(d[sel] == 0).all(axis=1)], 2] = -1.0
    return o, glm_normalize(d)


def towards_rays(n: int, seed: int, v9: np.ndarray, origin_lo, origin_hi):
    """Rays aimed at random points on random triangles (so most of them hit),
    including points on shared edges and vertices."""
    rng = np.random.default_rng(seed)
    tri = rng.integers(0, v9.shape[0], size=n)
    t = v9[tri].reshape(n, 3, 3).astype(np.float64)
    w = rng.random((n, 3))
    edge = rng.random(n) < 0.15  # aim exactly at an edge midpoint or vertex
    w[edge, rng.integers(0, 3, size=int(edge.sum()))] = 0.0
    w /= w.sum(axis=1, keepdims=True)
    p = (t * w[:, :, None]).sum(axis=1)
    lo = np.asarray(origin_lo, np.float64)
    hi = np.asarray(origin_hi, np.float64)
    o = lo + (hi - lo) * rng.random((n, 3))
    d = (p - o).astype(np.float32)
    return o.astype(np.float32), glm_normalize(d)


def scene_bounds(v9: np.ndarray, pad: float = 0.5):
    pts = v9.reshape(-1, 3)
    return pts.min(axis=0) - pad, pts.max(axis=0) + pad
