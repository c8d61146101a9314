"""Regenerates the golden fixtures in this directory.

Every array here is produced by the REFERENCE's own code -- mayueji/CAGR's
wn_treecode_cpu_treeutils.cpp tree builder and wn_treecode_cuda_kernels.cu
kernels compiled for the host by `make -C oracle ref` (oracle/_ref) -- so the
fixtures pin both the oracle restatement (tests/test_oracle.py) and the CUDA
path (tests/test_gpu_golden.py) to the reference's behaviour without needing
the reference checkout at test time.

    make -C oracle ref && python tests/golden/make_golden.py

bunny.npz holds CUDA-based/input/bunny.xyz and CUDA-based/results/bunny.xyz,
the reference's one published solve output (its mu for that input).
"""
from __future__ import annotations

import os
import sys
import zlib

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import OPS, REF_ROOT, RefOracle, point_weights  # noqa: E402
from tests._cases import edge_cloud, random_values, smooth_normals, sphere_cloud  # noqa: E402

if REF_ROOT is None:
    sys.exit("make_golden.py reads the reference checkout: set CAGR_REFERENCE_ROOT "
             "(or REF_ROOT in oracle/Makefile)")

CASES = {
    # name: (points factory, max_depth, leaf_size, run operators)
    "sphere_f32": (lambda: sphere_cloud(600, seed=100), 15, 1, True),
    "edge_f32": (lambda: edge_cloud(900, seed=101), 15, 1, True),
    "sphere_f64": (lambda: sphere_cloud(400, seed=102, dtype=np.float64), 15, 1, True),
    "leaf8_depth6": (lambda: sphere_cloud(700, seed=103), 6, 8, True),
}


def make_case(ref: RefOracle, name, make, max_depth, leaf_size, run_ops):
    pts = make()
    dt = pts.dtype
    n = pts.shape[0]
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    tree = ref.build_tree(pts, max_depth, leaf_size)
    mu = smooth_normals(pts, seed=104, zero_frac=0.1)
    s = random_values(n, 1, seed=105, dtype=dt)
    s[::9] = 0
    widths = rng.uniform(0.01, 0.05, size=n).astype(dt)
    out = dict(points=pts, max_depth=np.int64(max_depth), leaf_size=np.int64(leaf_size),
               depth=np.int64(tree.depth), num_leaves=np.int64(tree.num_leaves),
               parent=tree.parent, children=tree.children, is_leaf=tree.is_leaf,
               half_w=tree.half_w, npts=tree.npts, n2p=tree.n2p, n2p_start=tree.n2p_start,
               mu=mu, s=s, widths=widths)
    m3 = ref.moments(tree, pts, point_weights(mu), mu, tree_depth=max_depth)
    m1 = ref.moments(tree, pts, point_weights(s), s, tree_depth=max_depth)
    out.update(mom3_attrs=m3.attrs, mom3_rep=m3.rep, mom3_w=m3.weights,
               mom1_attrs=m1.attrs, mom1_rep=m1.rep, mom1_w=m1.weights)
    if run_ops:
        for op in OPS:
            vals, mom = (s, m1) if op in ("AT", "A2T1", "A2T2", "A2T3") else (mu, m3)
            out[f"out_{op}"] = ref.multiply(op, pts, widths, pts, vals, tree, mom)
            if op in ("A", "A3", "A21"):
                out[f"out_{op}_cont"] = ref.multiply(op, pts, widths, pts, vals, tree, mom,
                                                     continuous=True)
        q = rng.uniform(-1.1, 1.1, size=(300, 3)).astype(dt)
        wq = np.full(300, 0.03, dt)
        out["queries"] = q
        out["qwidths"] = wq
        out["out_A3_cont_queries"] = ref.multiply("A3", q, wq, pts, mu, tree, m3,
                                                  continuous=True)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(f"{name}: {n} points, {tree.num_nodes} nodes, depth {tree.depth}")


def make_bunny():
    base = os.path.join(REF_ROOT, "CUDA-based")
    inp = np.loadtxt(os.path.join(base, "input", "bunny.xyz"))
    res = np.loadtxt(os.path.join(base, "results", "bunny.xyz"))
    assert np.array_equal(inp[:, :3], res[:, :3])
    np.savez_compressed(os.path.join(HERE, "bunny.npz"), points=inp[:, :3],
                        mu_reference=res[:, 3:6])
    print(f"bunny: {inp.shape[0]} points")


def make_bunny_solves(ref: RefOracle):
    """The reference solve (main_CAGR.py schedule, restated in oracle/solve.py) run
    with the reference's own kernels on the bunny input: the full 40-iteration
    schedule at preset l1, and a 10-iteration steepest-descent schedule at l0."""
    from oracle.solve import PRESET_WIDTHS, normalize, solve
    g = np.load(os.path.join(HERE, "bunny.npz"))
    p = normalize(g["points"])
    mu_l1 = solve(p, *PRESET_WIDTHS["l1"], impl=ref)
    mu_l0_10 = solve(p, *PRESET_WIDTHS["l0"], impl=ref, iters=10)
    np.savez_compressed(os.path.join(HERE, "bunny_solve.npz"), mu_l1_40=mu_l1,
                        mu_l0_10=mu_l0_10)
    print("bunny_solve: l1 x 40 iterations, l0 x 10 iterations")


def main():
    ref = RefOracle()
    for name, (make, md, ls, ops) in CASES.items():
        make_case(ref, name, make, md, ls, ops)
    make_bunny()
    make_bunny_solves(ref)


if __name__ == "__main__":
    main()
