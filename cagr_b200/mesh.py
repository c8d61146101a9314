"""Field evaluation on a regular grid, iso-value, marching cubes, PLY output.

The reconstruction back end of the reference is the GaussRecon driver
(mayueji/CAGR CUDA-based/ext/gaussrecon_src/main_GaussRecon_cuda.cu:256-494):
normals scaled to a fixed area (n / |n| * 1e-5, :276-288), node moments,
``multiply_by_A3`` with the continuous kernel at the grid corners and at the
samples (:427-466), iso-value = the median of the field at the samples
(:485-486), then marching cubes and a binary PLY.  The benchmark workloads
ask for regular G^3 grids, so here the grid is regular and everything up to
the mesh stays on the GPU:

    field  = -cagr_field_grid(A3, continuous)     (grid nodes, Morton order)
    iso    = -(median of A3 at the samples)
    mesh   = cagr_marching_cubes(field, iso)       (inside = field > iso)
"""
from __future__ import annotations

import ctypes
import dataclasses
import struct
import time

import numpy as np
import torch

from . import _lib
from ._lib import OPS, check
from .wn_treecode import WindingNumberTreecode, _ptr, _stream


def field_grid(wn: WindingNumberTreecode, dims, origin, spacing: float, width,
               op: str = "A3", continuous: bool = True) -> torch.Tensor:
    """Operator `op` (moments currently in slot 0) at the nodes of a regular grid:
    returns [nz, ny, nx] in the tree dtype."""
    nx, ny, nz = (int(d) for d in dims)
    out = torch.empty(nz, ny, nx, dtype=wn.dtype, device=wn.device)
    org = (ctypes.c_double * 3)(*[float(o) for o in origin])
    wt, ws = (None, float(width)) if isinstance(width, (int, float)) else (width.contiguous(), 0.0)
    with torch.cuda.device(wn.device):
        check(_lib.lib().cagr_field_grid(
            wn.handle, OPS[op], nx, ny, nz, org, float(spacing), _ptr(wt), ws,
            _lib.FLAG_CONTINUOUS if continuous else 0, _ptr(out), _stream(wn.device)),
            "cagr_field_grid")
    return out


def marching_cubes(values: torch.Tensor, origin, spacing: float, iso: float,
                   table: np.ndarray | None = None):
    """Iso-surface {values = iso} of a [nz, ny, nx] float32 CUDA grid: (vertices
    [V,3] float32, faces [F,3] int32), outward = toward values below iso.

    table: None (the library's generated case table, inside = values > iso) or
    a [256, 16] case table in the reference's layout (PoissonRecon's
    MarchingCubes::triangles: case bit k = corner {0,1,3,2,4,5,7,6}[k] below
    iso, edge ids 4a + u + 2v, -1 terminated), used as given: inside = values
    < iso, each cell's triangles in the table's order and winding
    (cagr_marching_cubes_table).

    One pass over the grid: the mesh goes straight into buffers sized by an
    estimate (a surface crossing the grid in every layer, 8 vertices per
    cell column of the largest face); a larger mesh is reported with its sizes
    and extracted again into buffers of exactly those sizes."""
    if not values.is_cuda or values.dtype != torch.float32 or values.dim() != 3:
        raise RuntimeError("values must be a float32 CUDA tensor [nz, ny, nx]")
    v = values.contiguous()
    nz, ny, nx = v.shape
    org = (ctypes.c_double * 3)(*[float(o) for o in origin])
    L = _lib.lib()
    if table is not None:
        tab = np.ascontiguousarray(table, np.int8)
        if tab.shape != (256, 16):
            raise RuntimeError("table must be [256, 16] int8")

        def run(*a):
            return L.cagr_marching_cubes_table(*a[:7], tab.ctypes.data_as(ctypes.c_void_p),
                                               *a[7:])
        name = "cagr_marching_cubes_table"
    else:
        run, name = L.cagr_marching_cubes, "cagr_marching_cubes"
    nv, nf = ctypes.c_int64(), ctypes.c_int64()
    est_v = 8 * max(nx * ny, ny * nz, nz * nx)
    cap = (est_v, 2 * est_v + 1024)
    with torch.cuda.device(v.device):
        s = _stream(v.device)
        for _ in range(2):
            verts = torch.empty(max(cap[0], 1), 3, dtype=torch.float32, device=v.device)
            faces = torch.empty(max(cap[1], 1), 3, dtype=torch.int32, device=v.device)
            rc = run(_ptr(v), nx, ny, nz, org, float(spacing), float(iso), _ptr(verts), cap[0],
                     _ptr(faces), cap[1], ctypes.byref(nv), ctypes.byref(nf), s)
            if rc == 4 and (nv.value > cap[0] or nf.value > cap[1]):   # CAGR_ERR_OVERFLOW
                cap = (nv.value, nf.value)
                continue
            check(rc, name)
            break
    return verts[:nv.value], faces[:nf.value]


def mc_table():
    """The marching-cubes case table: (tri [256, 36] int8 edge ids, ntri [256] uint8)."""
    tri = np.zeros((256, 36), np.int8)
    ntri = np.zeros(256, np.uint8)
    check(_lib.lib().cagr_mc_table(tri.ctypes.data_as(ctypes.c_void_p),
                                   ntri.ctypes.data_as(ctypes.c_void_p)), "cagr_mc_table")
    return tri, ntri


def write_ply(path: str, vertices: np.ndarray, faces: np.ndarray) -> None:
    """Binary little-endian PLY: float x, y, z per vertex and a uchar-counted int
    index list per face (the element layout the reference writes,
    gaussrecon_src/Octree.cpp:1259-1267)."""
    v = np.ascontiguousarray(vertices, np.float32)
    f = np.ascontiguousarray(faces, np.int32)
    header = ("ply\nformat binary_little_endian 1.0\n"
              f"element vertex {len(v)}\nproperty float x\nproperty float y\nproperty float z\n"
              f"element face {len(f)}\nproperty list uchar int vertex_indices\nend_header\n")
    rec = np.empty(len(f), dtype=[("n", "u1"), ("i", "<i4", (3,))])
    rec["n"] = 3
    rec["i"] = f
    with open(path, "wb") as fh:
        fh.write(header.encode("ascii"))
        fh.write(v.astype("<f4").tobytes())
        fh.write(rec.tobytes())


def read_ply(path: str):
    """Reads what write_ply writes (vertices, faces)."""
    with open(path, "rb") as fh:
        data = fh.read()
    end = data.index(b"end_header\n") + len(b"end_header\n")
    head = data[:end].decode("ascii").split("\n")
    nv = int([h for h in head if h.startswith("element vertex")][0].split()[-1])
    nf = int([h for h in head if h.startswith("element face")][0].split()[-1])
    v = np.frombuffer(data, "<f4", count=3 * nv, offset=end).reshape(nv, 3)
    rec = np.frombuffer(data, dtype=[("n", "u1"), ("i", "<i4", (3,))], count=nf,
                        offset=end + 12 * nv)
    return v.copy(), rec["i"].copy()


@dataclasses.dataclass
class Reconstruction:
    vertices: torch.Tensor    # [V, 3] float32, in the points' (normalised) frame
    faces: torch.Tensor       # [F, 3] int32
    iso: float
    field: torch.Tensor       # [G, G, G]
    seconds: dict


def reconstruct(points: torch.Tensor, mu: torch.Tensor, grid: int = 128,
                lo: float = -1.2, hi: float = 1.2, width: float = 0.01,
                area: float | None = None, tree: WindingNumberTreecode | None = None,
                max_tree_depth: int = 15, far_field: str = "reference", degree: int = 5,
                theta: float = 0.5, op: str = "A3") -> Reconstruction:
    """Surface of oriented points on a regular grid**3 over [lo, hi]^3.

    points [N,3] float32 CUDA (normalised), mu [N,3] area-weighted normals (the
    CAGR solve's output).  area: if given, normals are rescaled to n / |n| * area
    with that weight per point, as the GaussRecon driver does (area 1e-5,
    main_GaussRecon_cuda.cu:276-288); if None, mu is used as it is (weights |mu|).
    far_field / degree / theta: the far-field mode of a tree built here.
    op: the field operator, "A3" as the CUDA GaussRecon driver or "A" as the
    CPU one (main_GaussRecon_cpu.cpp), continuous kernel either way.
    """
    if op not in ("A3", "A"):
        raise ValueError("op must be 'A3' or 'A'")
    dev = points.device
    sec = {}
    t0 = time.perf_counter()
    wn = tree if tree is not None else WindingNumberTreecode(
        points, max_tree_depth, far_field=far_field, degree=degree, theta=theta)
    torch.cuda.synchronize(dev)
    sec["tree"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    if area is not None:
        n = mu / torch.clamp(torch.linalg.norm(mu, dim=1, keepdim=True), min=1e-12)
        attrs = (n * area).contiguous()
        weights = torch.full((points.shape[0],), float(area), device=dev, dtype=points.dtype)
    else:
        attrs, weights = mu.contiguous(), None
    wn.scatter(attrs, weights=weights)
    samples = wn.multiply(op, float(width), continuous=True)[:, 0]
    n = samples.shape[0]
    # grid value = -field and iso = -(median field at the samples), as the GaussRecon
    # program sets them (main_GaussRecon_cuda.cu:478,485-486): with outward normals
    # the field is lower inside, so inside = value > iso
    iso = -float(torch.kthvalue(samples.float(), n // 2 + 1).values)  # nth_element(n/2)
    spacing = (hi - lo) / (grid - 1)
    field = field_grid(wn, (grid, grid, grid), (lo, lo, lo), spacing, float(width), op=op)
    field.neg_()
    torch.cuda.synchronize(dev)
    sec["field"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    verts, faces = marching_cubes(field.float(), (lo, lo, lo), spacing, iso)
    torch.cuda.synchronize(dev)
    sec["marching_cubes"] = time.perf_counter() - t0
    return Reconstruction(verts, faces, iso, field, sec)
