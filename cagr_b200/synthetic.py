"""Seeded synthetic point clouds for the five benchmark workloads.

No public dataset is needed or used: every cloud is drawn with
``numpy.random.default_rng(seed)`` from an analytic surface, with the shapes,
sizes and noise levels of the workloads:

* ``sphere``  -- 5,000 points, area-uniform on the unit sphere, noise 1e-3.
* ``torus``   -- 100,000 points on a torus (R=1, r=0.3) with density
  proportional to (1 + 0.8 cos phi) along the tube angle, noise 2e-3.
* ``union8``  -- 1,000,000 points, area-uniform on the surface of the union of
  8 seeded primitives (spheres, axis-aligned boxes, capped cylinders; sizes
  U[0.1, 0.4], centres U[-1, 1]^3), noise 1e-3.
* ``thin``    -- 200,000 points on a closed 1 x 1 x 0.01 box plus a hollow
  cylinder (radius 0.5, wall 0.005), with 1 % uniform outliers.
* ``blobs``   -- 4,000,000 points on the 0.5 level set of a sum of 32
  isotropic Gaussian blobs, with sampling density varying 10x across the box,
  noise 5e-4.

``normalize`` maps a cloud into the reference's working box exactly as
main_CAGR.py:42-47 does (centre the bounding box, scale its longest side to
2/1.1).
"""
from __future__ import annotations

import numpy as np

WORKLOADS = ("sphere", "torus", "union8", "thin", "blobs")
DEFAULT_SIZES = {"sphere": 5_000, "torus": 100_000, "union8": 1_000_000,
                 "thin": 200_000, "blobs": 4_000_000}


def normalize(points: np.ndarray, bbox_scale: float = 1.1) -> np.ndarray:
    """main_CAGR.py:42-45: (p - bbox_centre) * 2 / (bbox_len * 1.1), float64."""
    p = np.asarray(points, np.float64)
    lo, hi = p.min(0), p.max(0)
    center = (lo + hi) / 2.0
    length = (hi - lo).max()
    return (p - center) * (2.0 / (length * bbox_scale))


def _unit(rng, n):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def sphere(n: int = 5_000, seed: int = 0, noise: float = 1e-3) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return _unit(rng, n) + rng.normal(scale=noise, size=(n, 3))


def torus(n: int = 100_000, seed: int = 1, R: float = 1.0, r: float = 0.3,
          noise: float = 2e-3) -> np.ndarray:
    """Density (per unit area) proportional to 1 + 0.8 cos(phi); the area
    element is (R + r cos phi) dtheta dphi, so phi is drawn by rejection from
    (R + r cos phi)(1 + 0.8 cos phi) and theta uniformly."""
    rng = np.random.default_rng(seed)
    out = []
    bound = (R + r) * 1.8
    need = n
    while need > 0:
        phi = rng.uniform(0, 2 * np.pi, size=2 * need + 64)
        acc = rng.uniform(0, bound, size=phi.shape) < (R + r * np.cos(phi)) * (1 + 0.8 * np.cos(phi))
        phi = phi[acc][:need]
        th = rng.uniform(0, 2 * np.pi, size=phi.shape)
        x = (R + r * np.cos(phi)) * np.cos(th)
        y = (R + r * np.cos(phi)) * np.sin(th)
        z = r * np.sin(phi)
        out.append(np.stack([x, y, z], 1))
        need -= phi.shape[0]
    p = np.concatenate(out)[:n]
    return p + rng.normal(scale=noise, size=p.shape)


# ---- union of primitives -----------------------------------------------------

def _prim_sample(rng, kind, c, s, n):
    """n area-uniform samples on one primitive's surface plus its area."""
    if kind == 0:  # sphere, radius s
        return c + s * _unit(rng, n), 4 * np.pi * s * s
    if kind == 1:  # axis-aligned box, half extents s (3,)
        areas = np.array([s[1] * s[2], s[1] * s[2], s[0] * s[2], s[0] * s[2],
                          s[0] * s[1], s[0] * s[1]]) * 4
        face = rng.choice(6, size=n, p=areas / areas.sum())
        u = rng.uniform(-1, 1, size=(n, 3)) * s
        ax = face // 2
        sign = np.where(face % 2 == 0, -1.0, 1.0)
        u[np.arange(n), ax] = sign * s[ax]
        return c + u, areas.sum()
    # capped cylinder along z: radius s[0], half height s[1]
    rad, hh = s[0], s[1]
    a_side = 2 * np.pi * rad * 2 * hh
    a_cap = np.pi * rad * rad
    tot = a_side + 2 * a_cap
    part = rng.choice(3, size=n, p=[a_side / tot, a_cap / tot, a_cap / tot])
    th = rng.uniform(0, 2 * np.pi, size=n)
    z = rng.uniform(-hh, hh, size=n)
    rr = np.where(part == 0, rad, rad * np.sqrt(rng.uniform(0, 1, size=n)))
    z = np.where(part == 1, -hh, np.where(part == 2, hh, z))
    return c + np.stack([rr * np.cos(th), rr * np.sin(th), z], 1), tot


def _prim_inside(kind, c, s, p):
    d = p - c
    if kind == 0:
        return (d * d).sum(1) < s * s
    if kind == 1:
        return np.all(np.abs(d) < s, axis=1)
    return ((d[:, 0] ** 2 + d[:, 1] ** 2) < s[0] ** 2) & (np.abs(d[:, 2]) < s[1])


def union8(n: int = 1_000_000, seed: int = 2, noise: float = 1e-3, k: int = 8) -> np.ndarray:
    """Area-uniform samples on the boundary of the union of k primitives:
    samples on each primitive's surface in proportion to its area, minus those
    strictly inside another primitive, repeated until n are kept."""
    rng = np.random.default_rng(seed)
    prims = []
    for _ in range(k):
        kind = int(rng.integers(0, 3))
        c = rng.uniform(-1, 1, size=3)
        if kind == 0:
            s = rng.uniform(0.1, 0.4)
        elif kind == 1:
            s = rng.uniform(0.1, 0.4, size=3)
        else:
            s = rng.uniform(0.1, 0.4, size=2)
        prims.append((kind, c, s))
    areas = np.array([_prim_sample(rng, kd, c, s, 1)[1] for kd, c, s in prims])
    out, have = [], 0
    while have < n:
        batch = max(1024, int((n - have) * 1.3))
        counts = rng.multinomial(batch, areas / areas.sum())
        for i, (kd, c, s) in enumerate(prims):
            if counts[i] == 0:
                continue
            p, _ = _prim_sample(rng, kd, c, s, counts[i])
            keep = np.ones(p.shape[0], bool)
            for j, (kd2, c2, s2) in enumerate(prims):
                if j != i:
                    keep &= ~_prim_inside(kd2, c2, s2, p)
            out.append(p[keep])
            have += int(keep.sum())
    p = np.concatenate(out)
    p = p[rng.permutation(p.shape[0])[:n]]
    return p + rng.normal(scale=noise, size=p.shape)


def thin(n: int = 200_000, seed: int = 3, outlier_frac: float = 0.01) -> np.ndarray:
    """Closed box 1 x 1 x 0.01 plus a hollow cylinder (radius 0.5, wall 0.005,
    height 1, axis along x through the box centre) and uniform outliers."""
    rng = np.random.default_rng(seed)
    n_out = int(round(n * outlier_frac))
    n_surf = n - n_out
    box, a_box = _prim_sample(rng, 1, np.zeros(3), np.array([0.5, 0.5, 0.005]), 1)
    # hollow cylinder = outer + inner lateral surfaces + two annular caps
    ro, ri, hh = 0.5, 0.495, 0.5
    a_cyl = 2 * np.pi * (ro + ri) * 2 * hh + 2 * np.pi * (ro * ro - ri * ri)
    nb = rng.binomial(n_surf, a_box / (a_box + a_cyl))
    pb, _ = _prim_sample(rng, 1, np.zeros(3), np.array([0.5, 0.5, 0.005]), nb)
    nc = n_surf - nb
    a_parts = np.array([2 * np.pi * ro * 2 * hh, 2 * np.pi * ri * 2 * hh,
                        np.pi * (ro * ro - ri * ri), np.pi * (ro * ro - ri * ri)])
    part = rng.choice(4, size=nc, p=a_parts / a_parts.sum())
    th = rng.uniform(0, 2 * np.pi, size=nc)
    x = rng.uniform(-hh, hh, size=nc)
    rr = np.where(part == 0, ro, np.where(part == 1, ri,
                  np.sqrt(rng.uniform(ri * ri, ro * ro, size=nc))))
    x = np.where(part == 2, -hh, np.where(part == 3, hh, x))
    pc = np.stack([x, rr * np.cos(th), rr * np.sin(th)], 1)
    surf = np.concatenate([pb, pc])
    lo, hi = surf.min(0), surf.max(0)
    outl = rng.uniform(lo, hi, size=(n_out, 3))
    p = np.concatenate([surf, outl])
    return p[rng.permutation(n)]


def blobs(n: int = 4_000_000, seed: int = 4, noise: float = 5e-4, k: int = 32) -> np.ndarray:
    """Points on {f = 0.5}, f = sum_i exp(-|x - c_i|^2 / (2 s_i^2)): random
    starts are pulled onto the level set by Newton steps along grad f, kept if
    they converged, and thinned by rejection so that the density varies 10x
    (linearly in x) across the box."""
    rng = np.random.default_rng(seed)
    C = rng.uniform(-1, 1, size=(k, 3))
    S = rng.uniform(0.15, 0.35, size=k)

    inv2 = 1.0 / (S * S)
    cc = (C * C).sum(1)

    def f_grad(p):
        # |p - c|^2 = |p|^2 - 2 p.c + |c|^2 and grad f = -sum_i g_i (p - c_i) / s_i^2,
        # as matrix products over the k blobs
        r2 = np.maximum((p * p).sum(1)[:, None] - 2.0 * (p @ C.T) + cc[None], 0.0)
        g = np.exp(-0.5 * r2 * inv2[None])
        f = g.sum(1)
        gw = g * inv2[None]
        grad = gw @ C - p * gw.sum(1)[:, None]
        return f, grad

    out, have = [], 0
    while have < n:
        m = min(400_000, max(50_000, 2 * (n - have)))
        # start near blob surfaces: centre + radius ~ s * 1.2 in a random direction
        idx = rng.integers(0, k, size=m)
        p = C[idx] + _unit(rng, m) * (S[idx] * rng.uniform(0.8, 2.0, size=m))[:, None]
        # Newton steps on the points not yet on the level set (|f - 1/2| < 1e-6)
        act = np.arange(m)
        ok = np.zeros(m, bool)
        for _ in range(13):
            f, g = f_grad(p[act])
            done = np.abs(f - 0.5) < 1e-6
            ok[act[done]] = True
            act, f, g = act[~done], f[~done], g[~done]
            if act.size == 0:
                break
            gg = (g * g).sum(1) + 1e-12
            p[act] = p[act] - ((f - 0.5) / gg)[:, None] * g
        p = p[ok]
        # density ratio 10x across x in [-1.5, 1.5]
        dens = 0.1 + 0.9 * np.clip((p[:, 0] + 1.5) / 3.0, 0, 1)
        p = p[rng.uniform(0, 1, size=p.shape[0]) < dens]
        out.append(p)
        have += p.shape[0]
    p = np.concatenate(out)[:n]
    return p + rng.normal(scale=noise, size=p.shape)


def make(name: str, n: int | None = None, seed: int | None = None) -> np.ndarray:
    """Raw (un-normalised) float64 cloud for a workload name."""
    fn = {"sphere": sphere, "torus": torus, "union8": union8, "thin": thin, "blobs": blobs}[name]
    kw = {}
    if n is not None:
        kw["n"] = n
    if seed is not None:
        kw["seed"] = seed
    return fn(**kw)
