"""GPU: cagr_scatter_noalloc, the node-moment entry point that allocates nothing.

It exists for callers that cannot call cudaMalloc when they need node
moments (under a device-memory budget owned by another allocator, or holding
only the reference's tree arrays).  Its scratch
is a fixed device array shared by every call, so this test runs it twice in a
row -- with different inputs and dtypes -- and checks each result against the
allocating path (cagr_scatter + cagr_scatter_export), which computes the same
sums in the same order: the results must be identical.  The file name sorts
last so a stop-at-first-failure run has run everything else first.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cloud(n, seed, dtype):
    rng = np.random.default_rng(seed)
    p = rng.normal(size=(n, 3))
    p = 0.8 * p / np.linalg.norm(p, axis=1, keepdims=True)
    p[::17] = p[1::17]                     # duplicates: multi-point leaves at depth 15
    return p.astype(dtype)


def _noalloc(wn, values, weights=None):
    import torch
    from cagr_b200 import _lib
    L = _lib.lib()
    M = wn.num_nodes
    dim = values.shape[1]
    a = torch.empty(M, dim, dtype=wn.dtype, device="cuda")
    r = torch.empty(M, 3, dtype=wn.dtype, device="cuda")
    w = torch.empty(M, dtype=wn.dtype, device="cuda")
    P = lambda t: None if t is None else ctypes.c_void_p(t.data_ptr())  # noqa: E731
    rc = L.cagr_scatter_noalloc(
        P(wn.node_parent_list), P(wn.node_children_list), P(wn.node_is_leaf_list),
        P(wn.num_points_in_node), P(wn.node2point_index), P(wn.node2point_indexstart), M,
        _lib.CAGR_F64 if wn.dtype == torch.float64 else _lib.CAGR_F32, P(wn.points),
        P(weights), P(values), dim, P(a), P(r), P(w),
        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    _lib.check(rc, "cagr_scatter_noalloc")
    return a, r, w


def _allocating(wn, values):
    wn.scatter(values)
    return wn.scatter_export(0, values.shape[1])


def test_noalloc_matches_allocating_path_twice(cuda_lib):
    import torch
    from cagr_b200 import WindingNumberTreecode
    cases = [(np.float32, 3, 31), (np.float64, 1, 32)]   # two calls in a row
    for dtype, dim, seed in cases:
        pts = _cloud(20000, seed, dtype)
        wn = WindingNumberTreecode(torch.from_numpy(pts).cuda())
        vals = torch.from_numpy(
            np.random.default_rng(seed).normal(size=(len(pts), dim)).astype(dtype)).cuda()
        vals[::11] = 0                                    # zero weights: centroid fallback
        got = _noalloc(wn, vals)
        ref = _allocating(wn, vals)
        torch.cuda.synchronize()
        for g, e, name in zip(got, ref, ("node_attrs", "reppoints", "node_weights")):
            assert torch.equal(g, e), (dtype.__name__, name)


def test_noalloc_with_caller_weights(cuda_lib):
    """The caller-supplied point weights (some zero) give the allocating path's
    moments with the same weights, bit for bit."""
    import torch
    from cagr_b200 import WindingNumberTreecode
    for dtype, dim, seed in [(np.float32, 3, 33), (np.float64, 1, 34)]:
        pts = _cloud(15000, seed, dtype)
        rng = np.random.default_rng(seed)
        wn = WindingNumberTreecode(torch.from_numpy(pts).cuda())
        vals = torch.from_numpy(rng.normal(size=(len(pts), dim)).astype(dtype)).cuda()
        wts = np.abs(rng.normal(size=len(pts))).astype(dtype)
        wts[::7] = 0                                      # zero weights: centroid fallback
        wts = torch.from_numpy(wts).cuda()
        got = _noalloc(wn, vals, wts)
        wn.scatter(vals, weights=wts)
        ref = wn.scatter_export(0, dim)
        torch.cuda.synchronize()
        for g, e, name in zip(got, ref, ("node_attrs", "reppoints", "node_weights")):
            assert torch.equal(g, e), (dtype.__name__, name)


def test_noalloc_rejects_trees_beyond_its_capacity(cuda_lib):
    from cagr_b200 import _lib
    L = _lib.lib()
    dummy = ctypes.c_void_p(256)
    rc = L.cagr_scatter_noalloc(dummy, dummy, dummy, dummy, dummy, dummy, (1 << 21) + 1,
                                _lib.CAGR_F32, dummy, None, dummy, 3, dummy, dummy, dummy, None)
    assert rc == 1
    assert b"exceeds the no-alloc scratch capacity" in L.cagr_last_error()
