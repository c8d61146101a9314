"""GPU: the CUDA path against the reference's own outputs (tests/golden).

The fixtures were produced by the reference's tree builder and kernels
compiled for the host; here the C ABI must reproduce the tree and node
moments bit for bit and every operator within the FP32 / FP64 tolerances.
"""
import glob
import os

import numpy as np
import pytest

from tests._cases import rel_errors

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz"))
               if not os.path.basename(p).startswith(("bunny", "mc_")))
OPS = ["A", "AT", "A3", "A21", "A22", "A23", "A2T1", "A2T2", "A2T3", "G"]
TREE_KEYS = ["parent", "children", "is_leaf", "half_w", "npts", "n2p", "n2p_start"]


def load(name):
    return dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))


def tree_for(g):
    import torch
    from cagr_b200 import WindingNumberTreecode
    return WindingNumberTreecode(torch.from_numpy(g["points"]).cuda(),
                                 max_tree_depth=int(g["max_depth"]),
                                 leaf_size=int(g["leaf_size"]))


@pytest.mark.parametrize("case", CASES)
def test_tree_and_moments(cuda_lib, case):
    import torch
    g = load(case)
    wn = tree_for(g)
    got = [t.cpu().numpy() for t in (wn.node_parent_list, wn.node_children_list,
                                     wn.node_is_leaf_list, wn.node_half_w_list,
                                     wn.num_points_in_node, wn.node2point_index,
                                     wn.node2point_indexstart)]
    for key, arr in zip(TREE_KEYS, got):
        assert np.array_equal(arr, g[key]), key
    assert wn.depth == int(g["depth"])
    for vals, tag, dim in ((g["mu"], "mom3", 3), (g["s"], "mom1", 1)):
        wn.scatter(torch.from_numpy(vals).cuda())
        a, r, w = (t.cpu().numpy() for t in wn.scatter_export(0, dim))
        assert np.array_equal(a, g[f"{tag}_attrs"]), tag
        assert np.array_equal(r, g[f"{tag}_rep"]), tag
        assert np.array_equal(w, g[f"{tag}_w"]), tag


@pytest.mark.parametrize("case", CASES)
def test_operators(cuda_lib, case):
    import torch
    g = load(case)
    wn = tree_for(g)
    tol = (2e-5, 2e-4) if g["points"].dtype == np.float32 else (1e-12, 1e-11)
    widths = torch.from_numpy(g["widths"]).cuda()
    for op in OPS:
        vals = g["s"] if op in ("AT", "A2T1", "A2T2", "A2T3") else g["mu"]
        v = torch.from_numpy(vals).cuda()
        got = getattr(wn, f"forward_{op}")(v, widths).cpu().numpy()
        l2, mx = rel_errors(got, g[f"out_{op}"])
        assert l2 <= tol[0] and mx <= tol[1], (op, l2, mx)
        if f"out_{op}_cont" in g:
            wn.scatter(v)
            got = wn.multiply(op, widths, continuous=True).cpu().numpy()
            l2, mx = rel_errors(got, g[f"out_{op}_cont"])
            assert l2 <= tol[0] and mx <= tol[1], (op, "cont", l2, mx)
    wn.scatter(torch.from_numpy(g["mu"]).cuda())
    got = wn.multiply("A3", torch.from_numpy(g["qwidths"]).cuda(),
                      queries=torch.from_numpy(g["queries"]).cuda(), continuous=True)
    l2, mx = rel_errors(got.cpu().numpy(), g["out_A3_cont_queries"])
    assert l2 <= tol[0] and mx <= tol[1], ("A3 queries", l2, mx)
