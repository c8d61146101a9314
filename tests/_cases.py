"""Seeded point clouds and helpers shared by the tests."""
from __future__ import annotations

import numpy as np


def sphere_cloud(n: int, seed: int = 0, dtype=np.float32, noise: float = 1e-3) -> np.ndarray:
    rng = np.random.default_rng(seed)
    p = rng.normal(size=(n, 3))
    p /= np.linalg.norm(p, axis=1, keepdims=True)
    p = p * 0.8 + rng.normal(scale=noise, size=p.shape)
    return p.astype(dtype)


def edge_cloud(n: int = 1500, seed: int = 1, dtype=np.float32) -> np.ndarray:
    """Points on split planes, duplicates, tiny signed values, the box faces
    and outside the [-1, 1] box: the cases where a float key could disagree
    with the reference's `x >= centre` comparisons."""
    rng = np.random.default_rng(seed)
    p = rng.uniform(-0.95, 0.95, size=(n, 3))
    planes = np.array([0.0, 0.5, -0.5, 0.25, -0.25, 0.125, 0.75, -0.75, 2.0 ** -14,
                       -2.0 ** -14, 1.0 - 2.0 ** -14])
    k = n // 6
    p[:k, 0] = rng.choice(planes, size=k)
    p[k:2 * k, 1] = rng.choice(planes, size=k)
    p[2 * k:3 * k, 2] = rng.choice(planes, size=k)
    p[3 * k:3 * k + 20] = p[3 * k]                      # 20 identical points
    p[3 * k + 20:3 * k + 30] = [1e-9, -1e-9, 0.0]        # tiny signed values
    p[3 * k + 30:3 * k + 40] = [-1e-30, 1e-30, -0.0]
    p[3 * k + 40:3 * k + 50] = rng.uniform(1.0, 1.5, size=(10, 3))    # outside
    p[3 * k + 50:3 * k + 60] = rng.uniform(-1.5, -1.0, size=(10, 3))
    p[3 * k + 60:3 * k + 70] = [1.0, -1.0, 1.0]          # box corner
    # near-duplicates: differ only below the depth-15 resolution
    base = rng.uniform(-0.5, 0.5, size=(10, 3))
    p[3 * k + 70:3 * k + 80] = base
    p[3 * k + 80:3 * k + 90] = base + 2.0 ** -18
    return p.astype(dtype)


def smooth_normals(points: np.ndarray, seed: int = 2, zero_frac: float = 0.0) -> np.ndarray:
    """Area-weighted outward normals (the shape of a CAGR mu), optionally
    with some exact zeros (zero node weights exercise the centroid fallback)."""
    rng = np.random.default_rng(seed)
    c = points.astype(np.float64) - points.astype(np.float64).mean(0)
    nrm = c / np.maximum(np.linalg.norm(c, axis=1, keepdims=True), 1e-12)
    nrm += rng.normal(scale=0.1, size=nrm.shape)
    mu = nrm * (4.0 / points.shape[0])
    if zero_frac > 0:
        mu[rng.uniform(size=points.shape[0]) < zero_frac] = 0.0
    return mu.astype(points.dtype)


def random_values(n: int, dim: int, seed: int = 3, dtype=np.float32) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return rng.normal(size=(n, dim)).astype(dtype)


def rel_errors(ours: np.ndarray, ref: np.ndarray):
    """(relative L2 error, max error relative to max |ref|)."""
    ours = np.asarray(ours, np.float64)
    ref = np.asarray(ref, np.float64)
    den2 = max(np.linalg.norm(ref), 1e-300)
    denm = max(np.abs(ref).max(), 1e-300)
    return np.linalg.norm(ours - ref) / den2, np.abs(ours - ref).max() / denm
