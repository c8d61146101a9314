"""Python face of the CPU oracle.  TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this module; it is the checker, never the product.  The
product (``cagr_b200``) runs on the GPU and fails loudly without its CUDA
library.

Two back ends, same calling convention:

* ``Oracle`` -- the C restatement in ``oracle/cagr_oracle.c`` (always built).
* ``RefOracle`` -- the reference's own sources compiled as host C++ into
  ``oracle/_ref/libwnref.so`` by ``make -C oracle ref`` (only where the
  reference checkout exists; the library itself travels with the repo).

Tree arrays use the reference layout (mayueji/CAGR,
CUDA-based/ext/wn_treecode/wn_treecode_cpu/wn_treecode_cpu_torch_interface.cpp:42-102):
``parent[M] i64, children[M,8] i64 (-1 = none), is_leaf[M] bool,
half_w[M] (input dtype), npts[M] i64, node2point_index[L] i64,
node2point_indexstart[M] i64``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_LIB_PATH = os.path.join(HERE, "_ref", "libwnref.so")
def _reference_root() -> str | None:
    """The reference checkout to compile from: $CAGR_REFERENCE_ROOT, else the
    one the build recipe (oracle/Makefile) names; None when neither exists."""
    root = os.environ.get("CAGR_REFERENCE_ROOT")
    if not root:
        try:
            root = subprocess.run(["make", "-s", "-C", HERE, "ref-root"], capture_output=True,
                                  text=True, timeout=30).stdout.strip()
        except (OSError, subprocess.SubprocessError):
            root = None
    return root if root and os.path.isdir(root) else None


REF_ROOT = _reference_root()

# Operator codes shared by both libraries.
OPS = {"A": 0, "AT": 1, "A3": 2, "A21": 3, "A22": 4, "A23": 5,
       "A2T1": 6, "A2T2": 7, "A2T3": 8, "G": 9}
ATTR_DIM = {"A": 3, "AT": 1, "A3": 3, "A21": 3, "A22": 3, "A23": 3,
            "A2T1": 1, "A2T2": 1, "A2T3": 1, "G": 3}
OUT_DIM = {"A": 1, "AT": 3, "A3": 1, "A21": 1, "A22": 1, "A23": 1,
           "A2T1": 3, "A2T2": 3, "A2T3": 3, "G": 3}

_p = ctypes.c_void_p
_i64 = ctypes.c_int64


def build_oracle(force: bool = False) -> None:
    """Compile the C restatement (and, when the reference checkout exists,
    the reference host build and its CUDA kernels for sm_100a)."""
    if force or not os.path.exists(LIB_PATH) or (
            os.path.getmtime(LIB_PATH) < os.path.getmtime(os.path.join(HERE, "cagr_oracle.c"))):
        subprocess.check_call(["make", "-s", "-C", HERE, "all"])
    if REF_ROOT and (force or not os.path.exists(REF_LIB_PATH)):
        subprocess.check_call(["make", "-s", "-C", HERE, "ref", f"REF_ROOT={REF_ROOT}"])
    gpu_lib = os.path.join(HERE, "_ref", "libwnref_gpu.so")
    if REF_ROOT and (force or not os.path.exists(gpu_lib)):
        subprocess.check_call(["make", "-s", "-C", HERE, "ref-gpu", f"REF_ROOT={REF_ROOT}"])
    # the reference's marching-cubes tables and its CPU reconstructor (baselines)
    for target, path in (("ref-mc", "libref_mc.so"), ("ref-gaussrecon", "main_GaussRecon_cpu")):
        if REF_ROOT and (force or not os.path.exists(os.path.join(HERE, "_ref", path))):
            if force and os.path.exists(os.path.join(HERE, "_ref", path)):
                os.remove(os.path.join(HERE, "_ref", path))
            subprocess.check_call(["make", "-s", "-C", HERE, target, f"REF_ROOT={REF_ROOT}"])


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


@dataclass
class Tree:
    parent: np.ndarray
    children: np.ndarray
    is_leaf: np.ndarray
    half_w: np.ndarray
    npts: np.ndarray
    n2p: np.ndarray
    n2p_start: np.ndarray
    depth: int
    num_leaves: int

    @property
    def num_nodes(self) -> int:
        return int(self.parent.shape[0])

    def as_tuple(self):
        """Same order as the reference's build_tree return value."""
        return (self.parent, self.children, self.is_leaf, self.half_w, self.npts,
                self.n2p, self.n2p_start)


@dataclass
class Moments:
    attrs: np.ndarray   # [M, C]
    rep: np.ndarray     # [M, 3]
    weights: np.ndarray  # [M]


class Oracle:
    """The C restatement (oracle/cagr_oracle.c)."""

    def __init__(self, path: str = LIB_PATH):
        if not os.path.exists(path):
            build_oracle()
        self.lib = ctypes.CDLL(path)
        L = self.lib
        for suf in ("f32", "f64"):
            f = getattr(L, f"oracle_build_tree_{suf}")
            f.restype = _p
            f.argtypes = [_p, _i64, _i64, _i64]
            f = getattr(L, f"oracle_moments_{suf}")
            f.restype = None
            f.argtypes = [_i64] + [_p] * 8 + [_i64] + [_p] * 3
            f = getattr(L, f"oracle_multiply_{suf}")
            f.restype = ctypes.c_int
            f.argtypes = [ctypes.c_int, _p, _p, _i64] + [_p] * 11 + [ctypes.c_int, _p, _p]
        L.oracle_tree_sizes.argtypes = [_p] * 5
        L.oracle_tree_fill.argtypes = [_p] * 8
        L.oracle_tree_free.argtypes = [_p]
        L.oracle_direct_f64.restype = ctypes.c_int
        L.oracle_direct_f64.argtypes = [ctypes.c_int, _p, _p, _i64, _p, _p, _i64, _p,
                                        ctypes.c_int]

    # -- tree ---------------------------------------------------------------
    def build_tree(self, points: np.ndarray, max_depth: int = 15, leaf_size: int = 1) -> Tree:
        points = np.ascontiguousarray(points)
        suf = "f64" if points.dtype == np.float64 else "f32"
        points = points.astype(np.float64 if suf == "f64" else np.float32, copy=False)
        n = points.shape[0]
        h = getattr(self.lib, f"oracle_build_tree_{suf}")(_ptr(points), n, max_depth, leaf_size)
        if not h:
            raise MemoryError("oracle tree build failed")
        try:
            m, nl, d, ln = (ctypes.c_int64() for _ in range(4))
            self.lib.oracle_tree_sizes(h, ctypes.byref(m), ctypes.byref(nl), ctypes.byref(d),
                                       ctypes.byref(ln))
            M, Ln = m.value, ln.value
            parent = np.empty(M, np.int64)
            children = np.empty((M, 8), np.int64)
            is_leaf = np.empty(M, np.bool_)
            half_w = np.empty(M, np.float64)
            npts = np.empty(M, np.int64)
            n2p = np.empty(Ln, np.int64)
            n2p_start = np.empty(M, np.int64)
            self.lib.oracle_tree_fill(h, _ptr(parent), _ptr(children), _ptr(is_leaf),
                                      _ptr(half_w), _ptr(npts), _ptr(n2p), _ptr(n2p_start))
        finally:
            self.lib.oracle_tree_free(h)
        return Tree(parent, children, is_leaf, half_w.astype(points.dtype), npts, n2p,
                    n2p_start, d.value, nl.value)

    # -- node moments -------------------------------------------------------
    def moments(self, tree: Tree, points: np.ndarray, weights: np.ndarray,
                attrs: np.ndarray) -> Moments:
        dt = points.dtype
        suf = "f64" if dt == np.float64 else "f32"
        points = np.ascontiguousarray(points, dt)
        weights = np.ascontiguousarray(weights, dt)
        attrs = np.ascontiguousarray(attrs, dt).reshape(points.shape[0], -1)
        c = attrs.shape[1]
        M = tree.num_nodes
        out_a = np.zeros((M, c), dt)
        out_r = np.zeros((M, 3), dt)
        out_w = np.zeros(M, dt)
        getattr(self.lib, f"oracle_moments_{suf}")(
            M, _ptr(tree.children), _ptr(tree.is_leaf), _ptr(tree.npts), _ptr(tree.n2p),
            _ptr(tree.n2p_start), _ptr(points), _ptr(weights), _ptr(attrs), c, _ptr(out_a),
            _ptr(out_r), _ptr(out_w))
        return Moments(out_a, out_r, out_w)

    # -- traversal ------------------------------------------------------------
    def multiply(self, op: str, queries: np.ndarray, widths: np.ndarray, points: np.ndarray,
                 attrs: np.ndarray, tree: Tree, mom: Moments, continuous: bool = False,
                 counts: bool = False):
        dt = points.dtype
        suf = "f64" if dt == np.float64 else "f32"
        queries = np.ascontiguousarray(queries, dt)
        widths = np.ascontiguousarray(widths, dt)
        attrs = np.ascontiguousarray(attrs, dt).reshape(points.shape[0], -1)
        assert attrs.shape[1] == ATTR_DIM[op], (op, attrs.shape)
        nq = queries.shape[0]
        out = np.zeros((nq, OUT_DIM[op]), dt)
        terms = np.zeros(nq, np.int64) if counts else None
        visits = np.zeros(nq, np.int64) if counts else None
        half_w = np.ascontiguousarray(tree.half_w, dt)
        rc = getattr(self.lib, f"oracle_multiply_{suf}")(
            OPS[op], _ptr(queries), _ptr(widths), nq, _ptr(np.ascontiguousarray(points)),
            _ptr(attrs), _ptr(tree.n2p), _ptr(tree.n2p_start), _ptr(tree.children),
            _ptr(np.ascontiguousarray(mom.attrs, dt)), _ptr(tree.is_leaf), _ptr(half_w),
            _ptr(np.ascontiguousarray(mom.rep, dt)), _ptr(tree.npts), _ptr(out),
            int(continuous), _ptr(terms), _ptr(visits))
        if rc != 0:
            raise RuntimeError(f"oracle traversal failed ({rc})")
        if counts:
            return out, terms, visits
        return out

    def direct(self, op: str, queries: np.ndarray, widths: np.ndarray, points: np.ndarray,
               attrs: np.ndarray, continuous: bool = False) -> np.ndarray:
        """FP64 direct sum over all sources (no tree)."""
        q = np.ascontiguousarray(queries, np.float64)
        w = np.ascontiguousarray(widths, np.float64)
        p = np.ascontiguousarray(points, np.float64)
        a = np.ascontiguousarray(attrs, np.float64).reshape(p.shape[0], -1)
        assert a.shape[1] == ATTR_DIM[op]
        out = np.zeros((q.shape[0], OUT_DIM[op]), np.float64)
        rc = self.lib.oracle_direct_f64(OPS[op], _ptr(q), _ptr(w), q.shape[0], _ptr(p), _ptr(a),
                                        p.shape[0], _ptr(out), int(continuous))
        if rc != 0:
            raise RuntimeError("oracle direct sum failed")
        return out

    def interp(self, op: str, queries: np.ndarray, widths: np.ndarray, points: np.ndarray,
               attrs: np.ndarray, tree: Tree, degree: int = 5, theta: float = 0.5,
               direct_max: int = 64, order: np.ndarray | None = None,
               continuous: bool = False, kind: str | None = None, counts: bool = False):
        """The library's interpolated far-field mode (CAGR_FAR_INTERP) in FP64:
        Chebyshev proxy grids of degree `degree` per node, acceptance per group
        of 32 queries taken in `order` (oracle_interp_f64 in cagr_oracle.c).
        op: one of OPS or "A2_FUSED", "A2T_SUM" (attrs [n,3]: three scalar
        columns), "A2T_SUM_SHARED" (attrs [n,1]), "COUNT"."""
        code = {**OPS, "A2_FUSED": 10, "A2T_SUM": 11, "COUNT": 12, "A2T_SUM_SHARED": 13}[op]
        q = np.ascontiguousarray(queries, np.float64)
        w = np.ascontiguousarray(widths, np.float64)
        p = np.ascontiguousarray(points, np.float64)
        a = np.ascontiguousarray(attrs, np.float64).reshape(p.shape[0], -1)
        if kind is None:
            kind = "triple" if op == "A2T_SUM" else ("scalar" if a.shape[1] == 1 else "vec")
        k = {"vec": 0, "scalar": 1, "triple": 2}[kind]
        nq = q.shape[0]
        co = 1 if op in ("A", "A3", "A21", "A22", "A23", "COUNT") else 3
        out = np.zeros((nq, co), np.float64)
        terms = np.zeros(nq, np.int64)
        o = None if order is None else np.ascontiguousarray(order, np.int64)
        f = self.lib.oracle_interp_f64
        f.restype = ctypes.c_int
        f.argtypes = [ctypes.c_int, ctypes.c_int, _p, _p, _p, _i64, _p, _p, _i64, ctypes.c_int] + \
            [_p] * 5 + [_i64, ctypes.c_int, ctypes.c_double, ctypes.c_int, _p, _p]
        rc = f(code, int(continuous), _ptr(q), _ptr(w), _ptr(o), nq, _ptr(p), _ptr(a), p.shape[0], k,
               _ptr(tree.children), _ptr(np.ascontiguousarray(tree.is_leaf, np.uint8)),
               _ptr(tree.npts), _ptr(tree.n2p), _ptr(tree.n2p_start), tree.num_nodes, int(degree),
               float(theta), int(direct_max), _ptr(out), _ptr(terms))
        if rc != 0:
            raise RuntimeError("oracle interpolated traversal failed")
        return (out, terms) if counts else out

    def marching_cubes(self, values: np.ndarray, origin, spacing: float, iso: float,
                       tri: np.ndarray, ntri: np.ndarray):
        """Regular-grid marching cubes with a given case table (the checker of
        cagr_marching_cubes).  values: [nz, ny, nx] float32."""
        v = np.ascontiguousarray(values, np.float32)
        nz, ny, nx = v.shape
        tri = np.ascontiguousarray(tri, np.int8).reshape(-1)
        ntri = np.ascontiguousarray(ntri, np.uint8)
        f = self.lib.oracle_marching_cubes
        f.restype = ctypes.c_int
        f.argtypes = [_p, ctypes.c_int, ctypes.c_int, ctypes.c_int] + [ctypes.c_double] * 4 + \
            [ctypes.c_float, _p, _p, _p, _i64, _p, _i64, _p, _p]
        nv, nf = ctypes.c_int64(), ctypes.c_int64()
        args = [_ptr(v), nx, ny, nz, float(origin[0]), float(origin[1]), float(origin[2]),
                float(spacing), float(iso), _ptr(tri), _ptr(ntri)]
        if f(*args, None, 0, None, 0, ctypes.byref(nv), ctypes.byref(nf)) != 0:
            raise MemoryError("oracle marching cubes")
        verts = np.zeros((nv.value, 3), np.float32)
        faces = np.zeros((nf.value, 3), np.int32)
        if f(*args, _ptr(verts), nv.value, _ptr(faces), nf.value, ctypes.byref(nv),
             ctypes.byref(nf)) != 0:
            raise MemoryError("oracle marching cubes")
        return verts, faces

    def marching_cubes_reftable(self, values: np.ndarray, origin, spacing: float, iso: float,
                                triangles: np.ndarray):
        """Regular-grid marching cubes with a case table in the reference's
        layout (triangles [256, 16], MarchingCubes.cpp's GetIndex and
        AddTriangleIndices restated; the checker of cagr_marching_cubes_table).
        values: [nz, ny, nx] float32."""
        v = np.ascontiguousarray(values, np.float32)
        nz, ny, nx = v.shape
        tri = np.ascontiguousarray(triangles, np.int8).reshape(-1)
        assert tri.size == 256 * 16
        f = self.lib.oracle_marching_cubes_reftable
        f.restype = ctypes.c_int
        f.argtypes = [_p, ctypes.c_int, ctypes.c_int, ctypes.c_int] + [ctypes.c_double] * 4 + \
            [ctypes.c_float, _p, _p, _i64, _p, _i64, _p, _p]
        nv, nf = ctypes.c_int64(), ctypes.c_int64()
        args = [_ptr(v), nx, ny, nz, float(origin[0]), float(origin[1]), float(origin[2]),
                float(spacing), float(iso), _ptr(tri)]
        for _ in range(2):
            verts = np.zeros((max(nv.value, 0), 3), np.float32)
            faces = np.zeros((max(nf.value, 0), 3), np.int32)
            rc = f(*args, _ptr(verts) if verts.size else None, nv.value,
                   _ptr(faces) if faces.size else None, nf.value, ctypes.byref(nv),
                   ctypes.byref(nf))
            if rc == -1:
                raise MemoryError("oracle marching cubes")
            if rc == -2:
                raise ValueError("table entry is not an edge the case crosses")
        return verts, faces

    # -- the reference's per-call composition ----------------------------------
    def forward(self, op: str, tree: Tree, points: np.ndarray, values: np.ndarray,
                widths: np.ndarray, queries: np.ndarray | None = None,
                continuous: bool = False) -> np.ndarray:
        """One ``WindingNumberTreecode.forward_*`` call
        (wn_treecode_func.py:45-392): weights = |values| per point, node
        moments, then the traversal with queries = points by default."""
        dt = points.dtype
        values = np.ascontiguousarray(values, dt).reshape(points.shape[0], -1)
        weights = point_weights(values)
        mom = self.moments(tree, points, weights, values)
        q = points if queries is None else queries
        return self.multiply(op, q, widths, points, values, tree, mom, continuous)


def point_weights(values: np.ndarray) -> np.ndarray:
    """|value| per point: sqrt((v0*v0 + v1*v1) + v2*v2) in the input precision,
    the reference's ``(normals ** 2).sum(-1).sqrt()`` (wn_treecode_func.py:131)."""
    v = values.reshape(values.shape[0], -1)
    s = v[:, 0] * v[:, 0]
    for j in range(1, v.shape[1]):
        s = s + v[:, j] * v[:, j]
    return np.sqrt(s).astype(values.dtype)


class RefOracle:
    """The reference's own sources compiled as host C++ (oracle/_ref)."""

    def __init__(self, path: str = REF_LIB_PATH):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref`")
        self.lib = ctypes.CDLL(path)
        L = self.lib
        for suf in ("f32", "f64"):
            f = getattr(L, f"wnref_build_tree_{suf}")
            f.restype = _p
            f.argtypes = [_p, _i64, _i64, _i64]
            getattr(L, f"wnref_tree_sizes_{suf}").argtypes = [_p] * 5
            getattr(L, f"wnref_tree_fill_{suf}").argtypes = [_p] * 8
            getattr(L, f"wnref_tree_free_{suf}").argtypes = [_p]
            f = getattr(L, f"wnref_scatter_{suf}")
            f.restype = None
            f.argtypes = [_i64] + [_p] * 5 + [_i64] + [_p] * 4 + [_i64] + [_p] * 3
            f = getattr(L, f"wnref_multiply_{suf}")
            f.restype = ctypes.c_int
            f.argtypes = [ctypes.c_int, _p, _p, _i64] + [_p] * 11 + [ctypes.c_int]
        L.wnref_cpu_scatter_f32.restype = None
        L.wnref_cpu_scatter_f32.argtypes = [_i64] + [_p] * 5 + [_i64] + [_p] * 4 + [_i64] + [_p] * 3
        L.wnref_cpu_multiply_f32.restype = ctypes.c_int
        L.wnref_cpu_multiply_f32.argtypes = [ctypes.c_int, _p, _p, _i64] + [_p] * 11 + [ctypes.c_int]

    def build_tree(self, points: np.ndarray, max_depth: int = 15, leaf_size: int = 1) -> Tree:
        points = np.ascontiguousarray(points)
        suf = "f64" if points.dtype == np.float64 else "f32"
        dt = np.float64 if suf == "f64" else np.float32
        points = points.astype(dt, copy=False)
        L = self.lib
        h = getattr(L, f"wnref_build_tree_{suf}")(_ptr(points), points.shape[0], max_depth,
                                                  leaf_size)
        try:
            m, nl, d, ln = (ctypes.c_int64() for _ in range(4))
            getattr(L, f"wnref_tree_sizes_{suf}")(h, ctypes.byref(m), ctypes.byref(nl),
                                                  ctypes.byref(d), ctypes.byref(ln))
            M, Ln = m.value, ln.value
            parent = np.empty(M, np.int64)
            children = np.empty((M, 8), np.int64)
            is_leaf = np.empty(M, np.bool_)
            half_w = np.empty(M, dt)
            npts = np.empty(M, np.int64)
            n2p = np.empty(Ln, np.int64)
            n2p_start = np.empty(M, np.int64)
            getattr(L, f"wnref_tree_fill_{suf}")(h, _ptr(parent), _ptr(children), _ptr(is_leaf),
                                                 _ptr(half_w), _ptr(npts), _ptr(n2p),
                                                 _ptr(n2p_start))
        finally:
            getattr(L, f"wnref_tree_free_{suf}")(h)
        return Tree(parent, children, is_leaf, half_w, npts, n2p, n2p_start, d.value, nl.value)

    def moments(self, tree: Tree, points: np.ndarray, weights: np.ndarray, attrs: np.ndarray,
                tree_depth: int = 15, cpu_kernels: bool = False) -> Moments:
        dt = points.dtype
        suf = "f64" if dt == np.float64 else "f32"
        attrs = np.ascontiguousarray(attrs, dt).reshape(points.shape[0], -1)
        c = attrs.shape[1]
        M = tree.num_nodes
        out_a = np.zeros((M, c), dt)
        out_r = np.zeros((M, 3), dt)
        out_w = np.zeros(M, dt)
        f = self.lib.wnref_cpu_scatter_f32 if cpu_kernels else getattr(self.lib,
                                                                        f"wnref_scatter_{suf}")
        f(M, _ptr(tree.parent), _ptr(tree.children), _ptr(np.ascontiguousarray(points)),
          _ptr(np.ascontiguousarray(weights, dt)), _ptr(attrs), c, _ptr(tree.n2p),
          _ptr(tree.n2p_start), _ptr(tree.npts), _ptr(tree.is_leaf), tree_depth, _ptr(out_a),
          _ptr(out_r), _ptr(out_w))
        return Moments(out_a, out_r, out_w)

    def multiply(self, op: str, queries: np.ndarray, widths: np.ndarray, points: np.ndarray,
                 attrs: np.ndarray, tree: Tree, mom: Moments, continuous: bool = False,
                 cpu_kernels: bool = False) -> np.ndarray:
        dt = points.dtype
        suf = "f64" if dt == np.float64 else "f32"
        queries = np.ascontiguousarray(queries, dt)
        widths = np.ascontiguousarray(widths, dt)
        attrs = np.ascontiguousarray(attrs, dt).reshape(points.shape[0], -1)
        nq = queries.shape[0]
        out = np.zeros((nq, OUT_DIM[op]), dt)
        f = self.lib.wnref_cpu_multiply_f32 if cpu_kernels else getattr(self.lib,
                                                                         f"wnref_multiply_{suf}")
        rc = f(OPS[op], _ptr(queries), _ptr(widths), nq, _ptr(np.ascontiguousarray(points)),
               _ptr(attrs), _ptr(tree.n2p), _ptr(tree.n2p_start), _ptr(tree.children),
               _ptr(np.ascontiguousarray(mom.attrs, dt)), _ptr(tree.is_leaf),
               _ptr(np.ascontiguousarray(tree.half_w, dt)), _ptr(np.ascontiguousarray(mom.rep, dt)),
               _ptr(tree.npts), _ptr(out), int(continuous))
        if rc != 0:
            raise RuntimeError(f"reference traversal rejected op {op}")
        return out

    def forward(self, op: str, tree: Tree, points: np.ndarray, values: np.ndarray,
                widths: np.ndarray, queries: np.ndarray | None = None,
                continuous: bool = False, tree_depth: int = 15) -> np.ndarray:
        dt = points.dtype
        values = np.ascontiguousarray(values, dt).reshape(points.shape[0], -1)
        weights = point_weights(values)
        mom = self.moments(tree, points, weights, values, tree_depth)
        q = points if queries is None else queries
        return self.multiply(op, q, widths, points, values, tree, mom, continuous)
