"""GPU: the reference's own entry points, served by this library.

1. The low-level Python boundary: ``cagr_b200._cpu.build_tree`` and the
   ``cagr_b200._cuda`` functions with the names, argument order and shapes of
   the reference's pybind modules, driven by exactly the calls the
   reference's operator object makes (CUDA-based/ext/wn_treecode/
   wn_treecode_func.py: constructor :4-43, every forward_* :45-392: |value|
   weights, scatter_point_attrs_to_nodes, multiply_by_X).  Results must be the
   bits of cagr_b200.WindingNumberTreecode with the same weights.  Where a
   checkout of the reference is available (CAGR_REFERENCE_ROOT), the
   unmodified wn_treecode_func.py itself runs with these modules.
2. The C++ main_GaussReconCUDA (cagr_b200/cli/main_gaussrecon.cpp, linked to
   libcagr_b200.so) with the reference's command line: its mesh must be the
   mesh of the same steps made through the Python API.
"""
import importlib.util
import os
import subprocess
import sys
import types

import numpy as np
import pytest

from tests._cases import random_values, smooth_normals, sphere_cloud

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True, scope="module")
def _release_cached_trees():
    """The drop-in module caches the device trees of the points it has seen;
    release them when this module is done (later tests check the pool)."""
    yield
    from cagr_b200 import _cuda
    _cuda.clear_cache()

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
OPS = ["A", "AT", "A3", "A2", "A21", "A22", "A23", "A2T1", "A2T2", "A2T3", "G"]
SCALAR = {"AT", "A2T1", "A2T2", "A2T3"}


class ReferenceCalls:
    """The reference operator object's calls, in its order and argument order
    (wn_treecode_func.py:4-43 and :45-392), on a pair of extension modules."""

    def __init__(self, cpu, cuda, points, max_tree_depth=15):
        packed = cpu.build_tree(points.cpu(), max_tree_depth)
        packed = [t.to(points.device) for t in packed]
        (self.node_parent_list, self.node_children_list, self.node_is_leaf_list,
         self.node_half_w_list, self.num_points_in_node, self.node2point_index,
         self.node2point_indexstart) = packed
        self.cuda = cuda
        self.points = points
        self.tree_depth = max_tree_depth

    def forward(self, name, values, widths):
        point_weights = (values ** 2).sum(-1).sqrt()
        node_attrs, node_reppoints, _ = self.cuda.scatter_point_attrs_to_nodes(
            self.node_parent_list, self.node_children_list, self.points, point_weights, values,
            self.node2point_index, self.node2point_indexstart, self.num_points_in_node,
            self.node_is_leaf_list, self.tree_depth)
        return getattr(self.cuda, "multiply_by_" + name)(
            self.points, widths, self.points, values, self.node2point_index,
            self.node2point_indexstart, self.node_children_list, node_attrs,
            self.node_is_leaf_list, self.node_half_w_list, node_reppoints,
            self.num_points_in_node)


def _inputs(dtype=np.float32):
    import torch
    pts = sphere_cloud(20000, seed=30, dtype=dtype)
    P = torch.from_numpy(pts).cuda()
    mu = torch.from_numpy(smooth_normals(pts, seed=31)).cuda()
    s = torch.from_numpy(random_values(len(pts), 1, seed=32, dtype=dtype)).cuda()
    w = torch.from_numpy(np.random.default_rng(33).uniform(0.005, 0.02, len(pts)).astype(dtype)).cuda()
    return P, mu, s, w


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_reference_calls_give_the_bits_of_the_operator_object(cuda_lib, dtype):
    import torch
    from cagr_b200 import WindingNumberTreecode, _cpu, _cuda
    P, mu, s, w = _inputs(dtype)
    ref = ReferenceCalls(_cpu, _cuda, P)
    wn = WindingNumberTreecode(P)
    # the tree arrays are the reference layout of the same tree
    assert torch.equal(ref.node_children_list, wn.node_children_list)
    assert torch.equal(ref.node2point_index, wn.node2point_index)
    for op in OPS:
        vals = s if op in SCALAR else mu
        got = ref.forward(op, vals, w)
        wn.scatter(vals, weights=(vals ** 2).sum(-1).sqrt())
        want = wn.multiply("A2_FUSED" if op == "A2" else op, w)
        assert got.shape == want.shape and got.dtype == want.dtype, op
        assert torch.equal(got, want), op
    # the moments scatter_point_attrs_to_nodes returns are the library's
    a, r, wts = _cuda.scatter_point_attrs_to_nodes(
        ref.node_parent_list, ref.node_children_list, P, (mu ** 2).sum(-1).sqrt(), mu,
        ref.node2point_index, ref.node2point_indexstart, ref.num_points_in_node,
        ref.node_is_leaf_list, 15)
    wn.scatter(mu, weights=(mu ** 2).sum(-1).sqrt())
    a2, r2, w2 = wn.scatter_export()
    assert torch.equal(a, a2) and torch.equal(r, r2) and torch.equal(wts, w2)


def test_reference_checks_raise_like_torch_check(cuda_lib):
    from cagr_b200 import _cpu, _cuda
    P, mu, s, w = _inputs()
    ref = ReferenceCalls(_cpu, _cuda, P)
    with pytest.raises(RuntimeError, match="contiguous"):
        _cuda.multiply_by_A(P, w, P, mu.t().contiguous().t(), ref.node2point_index,
                            ref.node2point_indexstart, ref.node_children_list, mu,
                            ref.node_is_leaf_list, ref.node_half_w_list, mu,
                            ref.num_points_in_node)
    with pytest.raises(RuntimeError, match="CUDA"):
        ref.cuda.scatter_point_attrs_to_nodes(
            ref.node_parent_list, ref.node_children_list, P.cpu(), w, mu,
            ref.node2point_index, ref.node2point_indexstart, ref.num_points_in_node,
            ref.node_is_leaf_list, 15)
    with pytest.raises(RuntimeError, match="CPU"):
        _cpu.build_tree(P, 15)
    with pytest.raises(RuntimeError):
        _cpu.multiply_by_A(P.cpu())


@pytest.mark.skipif(not os.environ.get("CAGR_REFERENCE_ROOT"),
                    reason="no checkout of the reference (CAGR_REFERENCE_ROOT)")
def test_the_unmodified_reference_operator_object(cuda_lib):
    """wn_treecode_func.py from the reference checkout, unchanged, with its
    `wn_treecode._cpu` / `wn_treecode._cuda` imports bound to this library."""
    import torch
    from cagr_b200 import WindingNumberTreecode, _cpu, _cuda
    path = os.path.join(os.environ["CAGR_REFERENCE_ROOT"], "CUDA-based", "ext", "wn_treecode",
                        "wn_treecode_func.py")
    pkg = types.ModuleType("wn_treecode")
    pkg._cpu, pkg._cuda = _cpu, _cuda
    names = ("wn_treecode", "wn_treecode._cpu", "wn_treecode._cuda")
    saved = {k: sys.modules.get(k) for k in names}
    sys.modules.update({"wn_treecode": pkg, "wn_treecode._cpu": _cpu, "wn_treecode._cuda": _cuda})
    try:
        spec = importlib.util.spec_from_file_location("wn_treecode.wn_treecode_func", path)
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        P, mu, s, w = _inputs()
        theirs = mod.WindingNumberTreecode(P)
        wn = WindingNumberTreecode(P)
        for op in ("A21", "A22", "A23", "A2T1", "G"):
            vals = s if op in SCALAR else mu
            got = getattr(theirs, f"forward_{op}")(vals, w)
            wn.scatter(vals, weights=(vals ** 2).sum(-1).sqrt())
            assert torch.equal(got, wn.multiply(op, w)), op
    finally:
        for k, v in saved.items():
            if v is None:
                sys.modules.pop(k, None)
            else:
                sys.modules[k] = v


def test_cpp_gaussrecon_driver_matches_the_python_pipeline(cuda_lib, tmp_path):
    import torch
    from cagr_b200 import WindingNumberTreecode
    from cagr_b200.build import GAUSSRECON_PATH, build_gaussrecon
    from cagr_b200.mesh import field_grid, marching_cubes, read_ply
    if not os.path.exists(GAUSSRECON_PATH):
        build_gaussrecon()
    g = np.load(os.path.join(GOLDEN, "bunny.npz"))
    xyz = np.ascontiguousarray(g["points"], np.float32)
    nml = np.ascontiguousarray(g["mu_reference"], np.float32)
    inp = tmp_path / "bunny_oriented.xyz"
    with open(inp, "w") as fh:
        for p, n in zip(xyz, nml):
            fh.write(" ".join(repr(float(v)) for v in (*p, *n)) + "\n")
    out = tmp_path / "bunny.ply"
    depth = 7
    res = subprocess.run([GAUSSRECON_PATH, "-i", str(inp), "-o", str(out), "-w", "0.01",
                          "-m", "1", "-d", str(depth)], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr
    verts, faces = read_ply(str(out))
    assert len(faces) > 1000
    # the same steps through the Python API, in float32 as the driver computes them
    f32 = np.float32
    lo, hi = xyz.min(0), xyz.max(0)
    scale = f32((hi - lo).max()) * f32(1.1)
    corner = ((hi + lo - scale) / f32(2)).astype(f32)
    pts = (f32(2) * ((xyz - corner) / scale) - f32(1)).astype(f32)
    length = np.maximum(np.sqrt((nml[:, 0] * nml[:, 0] + nml[:, 1] * nml[:, 1]) + nml[:, 2] * nml[:, 2]),
                        f32(1e-12)).astype(f32)
    attrs = (nml / length[:, None] * f32(1e-5)).astype(f32)
    P = torch.from_numpy(pts).cuda()
    wn = WindingNumberTreecode(P)
    wn.scatter(torch.from_numpy(attrs).cuda(),
               weights=torch.full((len(pts),), 1e-5, device="cuda"))
    samples = wn.multiply("A3", 0.01, continuous=True)[:, 0]
    iso = -float(torch.kthvalue(samples, len(pts) // 2 + 1).values)
    G = (1 << depth) + 1
    field = field_grid(wn, (G, G, G), (-1.0, -1.0, -1.0), 2.0 / (G - 1), 0.01).neg_()
    v, f = marching_cubes(field, (-1.0, -1.0, -1.0), 2.0 / (G - 1), iso)
    v = ((v.cpu().numpy() + f32(1)) * f32(0.5) * scale + corner).astype(f32)
    assert np.array_equal(f.cpu().numpy(), faces)
    assert np.array_equal(v, verts)
    # and the surface lies on the input samples (a few grid cells at most)
    from scipy.spatial import cKDTree
    d, _ = cKDTree(xyz).query(verts)
    assert np.median(d) < 2 * scale / (G - 1)


REF_GAUSSRECON = os.path.join(os.path.dirname(GOLDEN), os.pardir, "oracle", "_ref",
                              "main_GaussRecon_cpu")


@pytest.mark.parametrize("op,depth", [("A", 6), ("A", 7), ("A3", 7)])
def test_cpp_driver_mesh_is_near_the_reference_cpu_reconstruction(cuda_lib, tmp_path, op, depth):
    """The reference's own CPU reconstructor (main_GaussRecon_cpu built from its
    sources by `make -C oracle ref-gaussrecon`: adaptive octree, host treecode,
    octree marching cubes) and main_GaussReconCUDA (regular grid of depth -d,
    operator A as the CPU driver or A3 as the CUDA one) on the reference's
    published bunny output: the two surfaces agree to a fraction of a grid cell
    on average and to about two cells at worst (distances over the bounding-box
    diagonal)."""
    from cagr_b200.build import GAUSSRECON_PATH, build_gaussrecon
    from oracle.mesh_distance import hausdorff, read_ply
    if not os.path.exists(REF_GAUSSRECON):
        pytest.skip("the reference reconstructor is not built (make -C oracle ref-gaussrecon)")
    if not os.path.exists(GAUSSRECON_PATH):
        build_gaussrecon()
    g = np.load(os.path.join(GOLDEN, "bunny.npz"))
    inp = tmp_path / "bunny_oriented.xyz"
    np.savetxt(inp, np.hstack([g["points"], g["mu_reference"]]), fmt="%.17g")
    ours, ref = tmp_path / "ours.ply", tmp_path / "ref.ply"
    r = subprocess.run([GAUSSRECON_PATH, "-i", str(inp), "-o", str(ours), "-d", str(depth),
                        "--op", op], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([REF_GAUSSRECON, "-i", str(inp), "-o", str(ref)], capture_output=True,
                       text=True, timeout=300, cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    mo, mr = read_ply(str(ours)), read_ply(str(ref))
    diag = float(np.linalg.norm(mr[0].max(0) - mr[0].min(0)))
    H, mean = hausdorff(mo, mr, n=100_000)
    print(f"op {op} depth {depth}: Hausdorff / diagonal {H / diag:.5f}, mean {mean / diag:.6f}")
    assert H / diag < 0.02 and mean / diag < 0.002, (H / diag, mean / diag)
