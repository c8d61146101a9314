"""CPU: the marching-cubes case table and the oracle's marching cubes.

The table (generated by the library, host-side, no GPU needed) must give
closed, consistently oriented, outward surfaces; the oracle's marching cubes
is the checker the GPU path is compared with bit for bit.
"""
import os
import tempfile

import numpy as np
import pytest

from cagr_b200 import build as B


@pytest.fixture(scope="module")
def table():
    if not os.path.exists(B.LIB_PATH):
        B.build()
    from cagr_b200.mesh import mc_table
    return mc_table()


def grid_field(fn, n=24, lo=-1.2, hi=1.2):
    h = (hi - lo) / (n - 1)
    c = lo + h * np.arange(n)
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    return fn(x, y, z).astype(np.float32), (lo, lo, lo), h


def edge_counts(faces):
    d = {}
    for f in faces:
        for a, b in ((f[0], f[1]), (f[1], f[2]), (f[2], f[0])):
            d[(a, b)] = d.get((a, b), 0) + 1
    return d


def assert_closed_oriented(faces):
    d = edge_counts(faces)
    for (a, b), c in d.items():
        assert c == 1, "a directed edge used twice: inconsistent orientation"
        assert d.get((b, a), 0) == 1, "an edge without its opposite: not closed"


def signed_volume(v, f):
    a, b, c = v[f[:, 0]].astype(np.float64), v[f[:, 1]].astype(np.float64), v[f[:, 2]].astype(np.float64)
    return float(np.einsum("ij,ij->i", a, np.cross(b, c)).sum() / 6.0)


def test_table_shape(table):
    tri, ntri = table
    assert tri.shape == (256, 36) and ntri.shape == (256,)
    assert ntri[0] == 0 and ntri[255] == 0
    assert ntri.max() <= 12
    # every triangle uses only crossed edges of its case
    for cs in range(256):
        for t in range(ntri[cs]):
            for e in map(int, tri[cs, 3 * t:3 * t + 3]):
                a, u, w = e >> 2, e & 1, (e >> 1) & 1
                others = [x for x in range(3) if x != a]
                c0 = [0, 0, 0]
                c0[others[0]], c0[others[1]] = u, w
                c1 = list(c0)
                c1[a] = 1
                i0 = c0[0] + 2 * c0[1] + 4 * c0[2]
                i1 = c1[0] + 2 * c1[1] + 4 * c1[2]
                assert ((cs >> i0) & 1) != ((cs >> i1) & 1)


def test_sphere_mesh_is_a_closed_outward_sphere(oracle, table):
    vals, org, h = grid_field(lambda x, y, z: 1.0 - np.sqrt(x * x + y * y + z * z))
    v, f = oracle.marching_cubes(vals, org, h, 0.0, *table)
    assert len(f) > 100
    assert_closed_oriented(f)
    E = len(edge_counts(f)) // 2
    assert len(v) - E + len(f) == 2                       # genus 0
    r = np.linalg.norm(v, axis=1)
    assert np.abs(r - 1).max() < h                         # on the sphere to a cell
    assert abs(signed_volume(v, f) - 4 / 3 * np.pi) < 0.05  # outward, right volume


@pytest.mark.parametrize("seed", [0, 1, 2, 3])
def test_random_blob_fields_give_closed_oriented_meshes(oracle, table, seed):
    """Sums of random Gaussians: ambiguous faces and cells occur; the face rule
    must keep neighbouring cells consistent."""
    rng = np.random.default_rng(seed)
    C = rng.uniform(-0.6, 0.6, size=(12, 3))
    S = rng.uniform(0.1, 0.25, size=12)

    def f(x, y, z):
        acc = np.zeros_like(x)
        for c, s in zip(C, S):
            acc += np.exp(-((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) / (2 * s * s))
        return acc

    vals, org, h = grid_field(f, n=40)
    v, faces = oracle.marching_cubes(vals, org, h, 0.5, *table)
    assert len(faces) > 0
    assert_closed_oriented(faces)
    assert signed_volume(v, faces) > 0


def test_checkerboard_field_is_closed(oracle, table):
    """Alternating corners: every face ambiguous."""
    n = 8
    g = np.indices((n, n, n)).sum(0) % 2
    vals = np.where(g == 1, 1.0, -1.0).astype(np.float32)
    vals[0, :, :] = vals[-1, :, :] = vals[:, 0, :] = vals[:, -1, :] = vals[:, :, 0] = \
        vals[:, :, -1] = -1.0
    v, f = oracle.marching_cubes(vals, (0, 0, 0), 1.0, 0.0, *table)
    assert_closed_oriented(f)


def test_ply_round_trip():
    from cagr_b200.mesh import read_ply, write_ply
    rng = np.random.default_rng(5)
    v = rng.normal(size=(50, 3)).astype(np.float32)
    f = rng.integers(0, 50, size=(80, 3)).astype(np.int32)
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "m.ply")
        write_ply(p, v, f)
        v2, f2 = read_ply(p)
    assert np.array_equal(v, v2) and np.array_equal(f, f2)
