"""GPU: grid field evaluation, marching cubes and the reconstruction pipeline.

* cagr_field_grid equals the operator at explicit query points (the oracle
  traversal at the grid nodes), within the FP32 tolerance;
* cagr_marching_cubes equals the oracle's marching cubes on the same field
  values bit for bit (vertices and faces);
* reconstruct() on a sphere cloud with outward normals gives a closed,
  outward-oriented surface on the sphere.
"""
import numpy as np
import pytest

from tests._cases import rel_errors, smooth_normals, sphere_cloud

pytestmark = pytest.mark.gpu


def _grid_points(n, lo, hi):
    h = (hi - lo) / (n - 1)
    c = lo + h * np.arange(n)
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    return np.stack([x.ravel(), y.ravel(), z.ravel()], 1), h


@pytest.mark.parametrize("n", [17, 32])
def test_field_grid_matches_explicit_queries(cuda_lib, oracle, n):
    import torch
    from cagr_b200 import WindingNumberTreecode
    from cagr_b200.mesh import field_grid
    pts = sphere_cloud(3000, seed=50)
    mu = smooth_normals(pts, seed=51)
    wn = WindingNumberTreecode(torch.from_numpy(pts).cuda())
    wn.scatter(torch.from_numpy(mu).cuda())
    _, h = _grid_points(n, -1.1, 1.1)
    # the grid nodes as the kernel forms them: fma(index, spacing, origin) in float32
    c = (np.arange(n) * np.float64(np.float32(h)) + np.float64(np.float32(-1.1))).astype(np.float32)
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    qf = np.stack([x.ravel(), y.ravel(), z.ravel()], 1)
    got = field_grid(wn, (n, n, n), (-1.1, -1.1, -1.1), h, 0.02).cpu().numpy().reshape(-1)
    tr = oracle.build_tree(pts)
    ref = oracle.forward("A3", tr, pts, mu, np.full(len(qf), 0.02, np.float32), queries=qf,
                         continuous=True)[:, 0]
    l2, mx = rel_errors(got, ref)
    assert l2 <= 2e-5 and mx <= 2e-4, (l2, mx)


def test_marching_cubes_bit_exact_against_oracle(cuda_lib, oracle):
    import torch
    from cagr_b200.mesh import marching_cubes, mc_table
    rng = np.random.default_rng(52)
    n = 48
    C = rng.uniform(-0.6, 0.6, size=(16, 3))
    S = rng.uniform(0.08, 0.25, size=16)
    q, h = _grid_points(n, -1.0, 1.0)
    f = np.zeros(len(q))
    for c, s in zip(C, S):
        f += np.exp(-((q - c) ** 2).sum(1) / (2 * s * s))
    vals = f.reshape(n, n, n).astype(np.float32)
    v_gpu, f_gpu = marching_cubes(torch.from_numpy(vals).cuda(), (-1, -1, -1), h, 0.5)
    v_ref, f_ref = oracle.marching_cubes(vals, (-1, -1, -1), h, 0.5, *mc_table())
    assert len(f_ref) > 1000
    assert np.array_equal(f_gpu.cpu().numpy(), f_ref)
    assert np.array_equal(v_gpu.cpu().numpy(), v_ref)


@pytest.mark.parametrize("shape", [(20, 24, 300), (9, 130, 257), (3, 2, 129)])
def test_marching_cubes_non_cubic_multi_unit_rows(cuda_lib, oracle, shape):
    """x-rows longer than one 128-point unit (cells whose +x corner is the next
    unit's first point), non-cubic grids, thin slabs."""
    import torch
    from cagr_b200.mesh import marching_cubes, mc_table
    nz, ny, nx = shape
    rng = np.random.default_rng(54 + nx)
    h = 0.01
    z, y, x = np.meshgrid(np.arange(nz) * h, np.arange(ny) * h, np.arange(nx) * h, indexing="ij")
    f = np.zeros(x.shape)
    for _ in range(20):
        c = rng.uniform(0, 1, 3) * np.array([nx, ny, nz]) * h
        s = rng.uniform(0.02, 0.3)
        f += np.exp(-((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) / (2 * s * s))
    vals = f.astype(np.float32)
    iso = float(np.median(vals))
    v_gpu, f_gpu = marching_cubes(torch.from_numpy(vals).cuda(), (0.0, 0.0, 0.0), h, iso)
    v_ref, f_ref = oracle.marching_cubes(vals, (0.0, 0.0, 0.0), h, iso, *mc_table())
    assert len(f_ref) > 0
    assert np.array_equal(f_gpu.cpu().numpy(), f_ref)
    assert np.array_equal(v_gpu.cpu().numpy(), v_ref)


def test_reconstruct_sphere(cuda_lib):
    import torch
    from cagr_b200.mesh import reconstruct
    pts = sphere_cloud(20000, seed=53)
    nrm = pts / np.linalg.norm(pts, axis=1, keepdims=True)
    mu = (nrm * (4 * np.pi * 0.8 ** 2 / len(pts))).astype(np.float32)   # outward, area-weighted
    rec = reconstruct(torch.from_numpy(pts).cuda(), torch.from_numpy(mu).cuda(), grid=64)
    v = rec.vertices.cpu().numpy()
    f = rec.faces.cpu().numpy()
    assert len(f) > 1000
    r = np.linalg.norm(v, axis=1)
    assert abs(np.median(r) - 0.8) < 0.02
    # closed and outward
    edges = {}
    for t in f:
        for a, b in ((t[0], t[1]), (t[1], t[2]), (t[2], t[0])):
            edges[(a, b)] = edges.get((a, b), 0) + 1
    assert all(c == 1 and edges.get((b, a), 0) == 1 for (a, b), c in edges.items())
    a, b, c = (v[f[:, k]].astype(np.float64) for k in range(3))
    vol = np.einsum("ij,ij->i", a, np.cross(b, c)).sum() / 6
    assert vol > 0


def test_small_buffers_report_the_sizes_and_nothing_beyond_them(cuda_lib):
    """With buffers smaller than the mesh the call writes nothing beyond them,
    returns CAGR_ERR_OVERFLOW and the sizes; buffers of those sizes then give
    the mesh the Python wrapper returns."""
    import ctypes

    import torch
    from cagr_b200 import _lib
    from cagr_b200.mesh import marching_cubes
    g = 48
    ax = np.linspace(-1, 1, g)
    X, Y, Z = np.meshgrid(ax, ax, ax, indexing="ij")
    vals = np.ascontiguousarray((1.0 - (X ** 2 + Y ** 2 + Z ** 2)).transpose(2, 1, 0), np.float32)
    V = torch.from_numpy(vals).cuda()
    h = 2.0 / (g - 1)
    v_ref, f_ref = marching_cubes(V, (-1, -1, -1), h, 0.5)
    org = (ctypes.c_double * 3)(-1.0, -1.0, -1.0)
    nv, nf = ctypes.c_int64(), ctypes.c_int64()
    cap_v, cap_f = 100, 100
    verts = torch.full((cap_v + 8, 3), 7.0, device="cuda")
    faces = torch.full((cap_f + 8, 3), -7, dtype=torch.int32, device="cuda")
    rc = _lib.lib().cagr_marching_cubes(ctypes.c_void_p(V.data_ptr()), g, g, g, org, h, 0.5,
                                        ctypes.c_void_p(verts.data_ptr()), cap_v,
                                        ctypes.c_void_p(faces.data_ptr()), cap_f,
                                        ctypes.byref(nv), ctypes.byref(nf), None)
    torch.cuda.synchronize()
    assert rc == 4 and nv.value == v_ref.shape[0] and nf.value == f_ref.shape[0]
    assert (verts[cap_v:] == 7.0).all() and (faces[cap_f:] == -7).all()
    assert torch.equal(verts[:cap_v], v_ref[:cap_v])


@pytest.mark.parametrize("shape", [(33, 40, 47), (9, 5, 300)])
def test_reference_table_mode_bit_exact_against_oracle(cuda_lib, oracle, shape):
    """cagr_marching_cubes_table with the reference's own case table
    (MarchingCubes.cpp:32-324, from the golden fixture) equals the oracle's
    restatement of the reference's per-cube lookup bit for bit: same vertices,
    same triangles in the same order (values exactly at the iso-value included,
    rows longer than one 128-point unit)."""
    import os
    import torch
    from cagr_b200.mesh import marching_cubes
    tri = np.load(os.path.join(os.path.dirname(__file__), "golden",
                               "mc_reference_tables.npz"))["triangles"]
    rng = np.random.default_rng(53)
    vals = rng.normal(size=shape).astype(np.float32)
    vals[rng.random(shape) < 0.05] = 0.25
    org, h = (-1.0, -0.5, 0.25), 0.03125
    v_gpu, f_gpu = marching_cubes(torch.from_numpy(vals).cuda(), org, h, 0.25, table=tri)
    v_ref, f_ref = oracle.marching_cubes_reftable(vals, org, h, 0.25, tri)
    assert len(f_ref) > 1000
    assert np.array_equal(f_gpu.cpu().numpy(), f_ref)
    assert np.array_equal(v_gpu.cpu().numpy(), v_ref)


def test_reference_table_mode_rejects_a_bad_table(cuda_lib):
    import os
    import torch
    from cagr_b200.mesh import marching_cubes
    tri = np.load(os.path.join(os.path.dirname(__file__), "golden",
                               "mc_reference_tables.npz"))["triangles"].copy()
    tri[1, :3] = (0, 4, 1)        # case 1 crosses edges 0, 4 and 8 only
    vals = torch.zeros(4, 4, 4, device="cuda")
    with pytest.raises(RuntimeError, match="not an edge the case crosses"):
        marching_cubes(vals, (0, 0, 0), 1.0, 0.5, table=tri)


@pytest.mark.parametrize("table_mode", [False, True])
@pytest.mark.parametrize("shape", [(6, 7, 256), (4, 3, 260), (5, 9, 133), (7, 6, 129)])
def test_non_finite_values_bit_exact_against_oracle(cuda_lib, oracle, shape, table_mode):
    """NaN (outside in both modes), +inf, -inf and values exactly at the
    iso-value in the field: vertices and triangles equal the oracle's bit for
    bit (NaN positions where an edge has a NaN end), for rows whose length is
    a multiple of 4 (16-byte row loads; 260: a last unit of 4 points) and rows
    that are not (133, 129: a last unit of 5 points and of 1)."""
    import os
    import torch
    from cagr_b200.mesh import marching_cubes, mc_table
    rng = np.random.default_rng(54)
    nz, ny, nx = shape
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    vals = (np.sin(0.3 * x) + np.cos(0.5 * y) * np.sin(0.7 * z)).astype(np.float32)
    u = rng.random(shape)
    vals[u < 0.03] = np.nan
    vals[(u >= 0.03) & (u < 0.04)] = np.inf
    vals[(u >= 0.04) & (u < 0.05)] = -np.inf
    vals[(u >= 0.05) & (u < 0.07)] = 0.125
    vals[:, :, : nx // 3][rng.random((nz, ny, nx // 3)) < 0.5] = np.nan  # stretches of NaN
    org, h, iso = (0.5, -0.25, 1.0), 0.0625, 0.125
    if table_mode:
        tri = np.load(os.path.join(os.path.dirname(__file__), "golden",
                                   "mc_reference_tables.npz"))["triangles"]
        v_gpu, f_gpu = marching_cubes(torch.from_numpy(vals).cuda(), org, h, iso, table=tri)
        v_ref, f_ref = oracle.marching_cubes_reftable(vals, org, h, iso, tri)
    else:
        v_gpu, f_gpu = marching_cubes(torch.from_numpy(vals).cuda(), org, h, iso)
        v_ref, f_ref = oracle.marching_cubes(vals, org, h, iso, *mc_table())
    assert len(f_ref) > 100 and np.isnan(v_ref).any()
    assert np.array_equal(f_gpu.cpu().numpy(), f_ref)
    assert np.array_equal(v_gpu.cpu().numpy(), v_ref, equal_nan=True)


@pytest.mark.parametrize("table_mode", [False, True])
def test_rows_not_on_16_byte_boundaries(cuda_lib, oracle, table_mode):
    """Rows whose length is a multiple of 4 but whose grid starts 4 bytes past
    a 16-byte boundary (a view into a larger buffer) take the scalar-load count
    pass; the mesh equals the oracle's bit for bit, and equals the mesh of the
    same values from an aligned copy (the bulk-copy count pass)."""
    import os
    import torch
    from cagr_b200.mesh import marching_cubes, mc_table
    rng = np.random.default_rng(55)
    shape = (9, 10, 264)
    vals = rng.normal(size=shape).astype(np.float32)
    vals[rng.random(shape) < 0.02] = np.nan
    buf = torch.empty(vals.size + 1, dtype=torch.float32, device="cuda")
    buf[1:] = torch.from_numpy(vals.ravel()).cuda()
    view = buf[1:].view(shape)
    assert view.data_ptr() % 16 == 4
    aligned = torch.from_numpy(vals).cuda()
    org, h, iso = (0.0, 0.0, 0.0), 0.125, 0.2
    tri = None
    if table_mode:
        tri = np.load(os.path.join(os.path.dirname(__file__), "golden",
                                   "mc_reference_tables.npz"))["triangles"]
        v_ref, f_ref = oracle.marching_cubes_reftable(vals, org, h, iso, tri)
    else:
        v_ref, f_ref = oracle.marching_cubes(vals, org, h, iso, *mc_table())
    v1, f1 = marching_cubes(view, org, h, iso, table=tri)
    v2, f2 = marching_cubes(aligned, org, h, iso, table=tri)
    assert len(f_ref) > 1000
    for v, f in ((v1, f1), (v2, f2)):
        assert np.array_equal(f.cpu().numpy(), f_ref)
        assert np.array_equal(v.cpu().numpy(), v_ref, equal_nan=True)
