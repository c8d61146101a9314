"""The reference's marching-cubes case table (tests/golden/mc_reference_tables.npz,
written from gaussrecon_src/MarchingCubes.cpp:32-324 by the reference's own
code) and the oracle's restatement of its per-cube lookup.

* the fixture equals the tables of the reference build (oracle/_ref, when it
  is present), and its edge masks are exactly the edges each case crosses
  under the reference's corner order and edge numbering (Cube.cpp:86-108);
* the oracle's reference-layout marching cubes gives, cell by cell, the
  triangles of the reference's MarchingCubes::AddTriangleIndices on the same
  8 corner values (values equal to the iso-value included);
* a table with an entry on an edge its case does not cross is rejected.
"""
import ctypes
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FIXTURE = os.path.join(ROOT, "tests", "golden", "mc_reference_tables.npz")
REF_MC = os.path.join(ROOT, "oracle", "_ref", "libref_mc.so")
CORNERS = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]


def _tables():
    z = np.load(FIXTURE)
    return z["edge_mask"], z["triangles"]


def _edge_corners(e):
    ax, a, b = e >> 2, e & 1, (e >> 1) & 1
    lo = [0, 0, 0]
    lo[0 if ax else 1] = a
    lo[2 if ax != 2 else 1] = b
    hi = list(lo)
    hi[ax] = 1
    return tuple(lo), tuple(hi)


def _ref_lib():
    if not os.path.exists(REF_MC):
        pytest.skip("the reference's marching cubes is not built (make -C oracle ref-mc)")
    return ctypes.CDLL(REF_MC)


def test_fixture_masks_are_the_crossed_edges():
    edge_mask, tri = _tables()
    for idx in range(256):
        below = {CORNERS[k] for k in range(8) if (idx >> k) & 1}
        crossed = sum(1 << e for e in range(12)
                      if (_edge_corners(e)[0] in below) != (_edge_corners(e)[1] in below))
        assert edge_mask[idx] == crossed, idx
        row = tri[idx]
        n = int(np.argmax(row == -1))
        assert n % 3 == 0 and n <= 15 and (row[n:] == -1).all()
        assert all((crossed >> int(e)) & 1 for e in row[:n]), idx


def test_fixture_equals_the_reference_build():
    lib = _ref_lib()
    em = np.zeros(256, np.int32)
    tr = np.zeros(256 * 16, np.int32)
    lib.ref_mc_tables(em.ctypes.data_as(ctypes.c_void_p), tr.ctypes.data_as(ctypes.c_void_p))
    edge_mask, tri = _tables()
    assert np.array_equal(em, edge_mask)
    assert np.array_equal(tr.reshape(256, 16), tri.astype(np.int32))


def _field(rng, shape, iso):
    v = rng.normal(size=shape).astype(np.float32)
    v[rng.random(shape) < 0.1] = iso        # corners exactly on the iso-value
    return v


def test_oracle_restates_the_reference_per_cube(oracle):
    lib = _ref_lib()
    lib.ref_mc_cell.restype = ctypes.c_int
    lib.ref_mc_cell.argtypes = [ctypes.c_void_p, ctypes.c_float, ctypes.c_void_p]
    _, tri = _tables()
    rng = np.random.default_rng(90)
    iso = np.float32(0.125)
    shape = (7, 9, 11)
    v = _field(rng, shape, iso)
    nz, ny, nx = shape
    verts, faces = oracle.marching_cubes_reftable(v, (0, 0, 0), 1.0, float(iso), tri)
    # vertex id -> (grid point, axis), in the oracle's numbering
    below = v < iso
    owner = []
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                for ax, (di, dj, dk) in enumerate(((1, 0, 0), (0, 1, 0), (0, 0, 1))):
                    i2, j2, k2 = i + di, j + dj, k + dk
                    if i2 < nx and j2 < ny and k2 < nz and below[k, j, i] != below[k2, j2, i2]:
                        owner.append(((i, j, k), ax))
    assert len(owner) == len(verts)
    got = [tuple(owner[x] for x in f) for f in faces]
    want = []
    idx = np.zeros(15, np.int32)
    for k in range(nz - 1):
        for j in range(ny - 1):
            for i in range(nx - 1):
                v8 = np.array([v[k + z, j + y, i + x] for z in (0, 1) for y in (0, 1)
                               for x in (0, 1)], np.float32)
                n = lib.ref_mc_cell(v8.ctypes.data_as(ctypes.c_void_p), iso,
                                    idx.ctypes.data_as(ctypes.c_void_p))
                for t in range(n):
                    tri_edges = []
                    for e in idx[3 * t:3 * t + 3]:
                        lo, _ = _edge_corners(int(e))
                        tri_edges.append(((i + lo[0], j + lo[1], k + lo[2]), int(e) >> 2))
                    want.append(tuple(tri_edges))
    assert len(want) > 100
    assert got == want


def test_oracle_rejects_an_uncrossed_edge(oracle):
    _, tri = _tables()
    bad = tri.copy()
    bad[1, :3] = (0, 4, 1)   # case 1 crosses edges 0, 4, 8 only
    v = np.array([[[0, 1], [1, 1]], [[1, 1], [1, 1]]], np.float32)
    with pytest.raises(ValueError):
        oracle.marching_cubes_reftable(v, (0, 0, 0), 1.0, 0.5, bad)


def test_mesh_distance_helper_is_exact_on_triangles():
    """oracle/mesh_distance.py's point-to-triangle distance equals the minimum
    over a dense barycentric sampling of each triangle (to the sampling step)."""
    from oracle.mesh_distance import _closest_on_triangles
    rng = np.random.default_rng(91)
    n = 200
    a, b, c = (rng.normal(size=(n, 3)) for _ in range(3))
    p = rng.normal(size=(n, 3)) * 2
    q = _closest_on_triangles(p, a, b, c)
    d = np.linalg.norm(p - q, axis=1)
    s = np.linspace(0, 1, 161)
    u, w = np.meshgrid(s, s)
    keep = u + w <= 1
    u, w = u[keep], w[keep]
    pts = a[:, None] + (b - a)[:, None] * u[None, :, None] + (c - a)[:, None] * w[None, :, None]
    brute = np.linalg.norm(pts - p[:, None], axis=2).min(1)
    assert (d <= brute + 1e-12).all()
    assert np.abs(d - brute).max() < 0.05
