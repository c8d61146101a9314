"""Mesh-to-mesh distances for the reconstruction comparisons.  TEST
INFRASTRUCTURE (the tests and bench.py's CPU-baseline leg use it).

read_ply reads the binary little-endian PLYs both reconstructors write (float
x, y, z vertices; uchar-counted int faces).  hausdorff(A, B) samples each
mesh's surface and measures each sample's exact distance to the other mesh's
nearest triangles (the k nearest by centroid, point-to-triangle distance after
Ericson, Real-Time Collision Detection, 5.1.5)."""
from __future__ import annotations

import numpy as np


def read_ply(path: str):
    with open(path, "rb") as fp:
        header = []
        while True:
            line = fp.readline().decode("ascii").strip()
            header.append(line)
            if line == "end_header":
                break
        assert "format binary_little_endian 1.0" in header
        nv = int(next(h for h in header if h.startswith("element vertex")).split()[-1])
        nf = int(next(h for h in header if h.startswith("element face")).split()[-1])
        v = np.frombuffer(fp.read(12 * nv), np.float32).reshape(nv, 3)
        rec = np.frombuffer(fp.read(13 * nf), np.uint8).reshape(nf, 13)
        assert (rec[:, 0] == 3).all()
        f = rec[:, 1:].copy().view(np.int32).reshape(nf, 3)
    return v.astype(np.float64), f


def _closest_on_triangles(p, a, b, c):
    """Closest points on triangles (a, b, c) to points p, all [n, 3]."""
    ab, ac, ap = b - a, c - a, p - a
    d1, d2 = (ab * ap).sum(1), (ac * ap).sum(1)
    bp = p - b
    d3, d4 = (ab * bp).sum(1), (ac * bp).sum(1)
    cp = p - c
    d5, d6 = (ab * cp).sum(1), (ac * cp).sum(1)
    va = d3 * d6 - d5 * d4
    vb = d5 * d2 - d1 * d6
    vc = d1 * d4 - d3 * d2
    denom = va + vb + vc
    with np.errstate(divide="ignore", invalid="ignore"):
        v = vb / denom
        w = vc / denom
        out = a + ab * v[:, None] + ac * w[:, None]
        # edge and vertex regions
        t_ab = d1 / (d1 - d3)
        t_ac = d2 / (d2 - d6)
        t_bc = (d4 - d3) / ((d4 - d3) + (d5 - d6))
    r = np.empty(len(p), np.int8)
    r[:] = 0
    conds = [
        (d1 <= 0) & (d2 <= 0),                                     # vertex a
        (d3 >= 0) & (d4 <= d3),                                    # vertex b
        (d6 >= 0) & (d5 <= d6),                                    # vertex c
        (vc <= 0) & (d1 >= 0) & (d3 <= 0),                         # edge ab
        (vb <= 0) & (d2 >= 0) & (d6 <= 0),                         # edge ac
        (va <= 0) & ((d4 - d3) >= 0) & ((d5 - d6) >= 0),           # edge bc
    ]
    vals = [a, b, c, a + ab * t_ab[:, None], a + ac * t_ac[:, None],
            b + (c - b) * t_bc[:, None]]
    done = np.zeros(len(p), bool)
    for cond, val in zip(conds, vals):
        m = cond & ~done
        out[m] = val[m]
        done |= m
    return out


def sample_surface(v, f, n, rng):
    a, b, c = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    area = 0.5 * np.linalg.norm(np.cross(b - a, c - a), axis=1)
    t = rng.choice(len(f), size=n, p=area / area.sum())
    r1, r2 = rng.random(n), rng.random(n)
    s = np.sqrt(r1)
    return a[t] * (1 - s)[:, None] + b[t] * (s * (1 - r2))[:, None] + c[t] * (s * r2)[:, None]


def point_to_mesh(p, v, f, k=16):
    from scipy.spatial import cKDTree
    a, b, c = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    k = min(k, len(f))
    _, nb = cKDTree((a + b + c) / 3).query(p, k=k, workers=-1)
    nb = nb.reshape(len(p), k)
    best = np.full(len(p), np.inf)
    for j in range(k):
        t = nb[:, j]
        q = _closest_on_triangles(p, a[t], b[t], c[t])
        best = np.minimum(best, np.linalg.norm(p - q, axis=1))
    return best


def hausdorff(mesh_a, mesh_b, n=200_000, seed=0):
    """(symmetric Hausdorff, mean symmetric distance), in the meshes' units."""
    rng = np.random.default_rng(seed)
    pa = sample_surface(*mesh_a, n, rng)
    pb = sample_surface(*mesh_b, n, rng)
    dab = point_to_mesh(pa, *mesh_b)
    dba = point_to_mesh(pb, *mesh_a)
    return max(dab.max(), dba.max()), 0.5 * (dab.mean() + dba.mean())
