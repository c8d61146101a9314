"""Drop-in for the reference's compiled extension ``wn_treecode._cuda``.

The reference's operator object (CUDA-based/ext/wn_treecode/wn_treecode_func.py)
calls a pybind module whose functions take torch tensors
(wn_treecode_cuda_torch_interface.cu, table at :779-793):

    scatter_point_attrs_to_nodes(node_parent_list, node_children_list, points,
        point_weights, point_attrs, node2point_index, node2point_indexstart,
        num_points_in_node, node_is_leaf_list, tree_depth)
        -> [node_attrs, node_reppoints, node_weights]                     (:41-134)
    multiply_by_X(query_points, query_width, points, point_attrs,
        node2point_index, node2point_indexstart, node_children_list, node_attrs,
        node_is_leaf_list, node_half_w_list, node_reppoints, num_points_in_node)
        -> [N', 1] (A, A3, A21, A22, A23) or [N', 3] (AT, G, A2, A2T1..3)  (:137-777)

This module has the same names, argument order, shapes, dtypes and checks
(a non-CUDA or non-contiguous input raises RuntimeError, as TORCH_CHECK does),
and runs on libcagr_b200.so through its C ABI.  The tree arrays it receives
are the reference layout; the library keeps its own device tree of the same
points (bit-identical to the reference's, built once per points tensor and
cached), and the node moments passed to multiply_by_X are loaded into it
(cagr_scatter_import), so the evaluation uses exactly the moments given.
``multiply_by_A3`` is the discontinuous kernel, as the reference's pybind
entry; ``multiply_by_A2`` returns [A21 | A22 | A23] (the reference's kernel
for it writes its three outputs through one comma expression, :835-837).
"""
from __future__ import annotations

import math

import torch

from . import _lib
from ._lib import OPS, check
from .wn_treecode import WindingNumberTreecode, _ptr, _stream

__all__ = ["scatter_point_attrs_to_nodes", "multiply_by_A", "multiply_by_A3", "multiply_by_AT",
           "multiply_by_G", "multiply_by_A2", "multiply_by_A21", "multiply_by_A22",
           "multiply_by_A23", "multiply_by_A2T1", "multiply_by_A2T2", "multiply_by_A2T3"]

_trees: dict = {}
_MAX_CACHED = 4


def _check_input(x: torch.Tensor, name: str) -> None:
    if not x.is_cuda:
        raise RuntimeError(f"{name} must be a CUDA tensor")
    if not x.is_contiguous():
        raise RuntimeError(f"{name} must be contiguous")


def _tree_for(points: torch.Tensor, num_nodes: int, depth) -> WindingNumberTreecode:
    """The library's tree of `points` (cached per tensor, its version counter
    and node count; the cache holds the tensor, so its storage is not reused).
    depth: the build's max_depth, or a callable giving it on a cache miss."""
    key = (points.data_ptr(), tuple(points.shape), points.dtype, points.device,
           points._version, int(num_nodes))
    hit = _trees.get(key)
    if hit is not None:
        return hit[1]
    d = int(depth() if callable(depth) else depth)
    wn = WindingNumberTreecode(points, max_tree_depth=d)
    if wn.num_nodes != num_nodes:
        wn.close()
        raise RuntimeError(f"the tree arrays ({num_nodes} nodes) are not the octree of these "
                           f"points at depth {d} ({wn.num_nodes} nodes)")
    if len(_trees) >= _MAX_CACHED:
        _trees.pop(next(iter(_trees)))[1].close()
    _trees[key] = (points, wn)
    return wn


def scatter_point_attrs_to_nodes(node_parent_list, node_children_list, points, point_weights,
                                 point_attrs, node2point_index, node2point_indexstart,
                                 num_points_in_node, node_is_leaf_list, tree_depth):
    """[node_attrs [M, C], node_reppoints [M, 3], node_weights [M]] (cuda_iface.cu:41-134)."""
    for x, nm in ((node_parent_list, "node_parent_list"), (node_children_list, "node_children_list"),
                  (points, "points"), (point_weights, "point_weights"), (point_attrs, "point_attrs"),
                  (node2point_index, "node2point_index"),
                  (node2point_indexstart, "node2point_indexstart"),
                  (num_points_in_node, "num_points_in_node"),
                  (node_is_leaf_list, "node_is_leaf_list")):
        _check_input(x, nm)
    attr_dim = point_attrs.shape[1]
    assert attr_dim in (1, 3)
    wn = _tree_for(points, node_parent_list.shape[0], tree_depth)
    wn.scatter(point_attrs.to(points.dtype).contiguous(),
               weights=point_weights.to(points.dtype).contiguous())
    return wn.scatter_export(slot=0, attr_dim=attr_dim)


def _multiply(op: str, query_points, query_width, points, point_attrs, node2point_index,
              node2point_indexstart, node_children_list, node_attrs, node_is_leaf_list,
              node_half_w_list, node_reppoints, num_points_in_node, out_dim: int):
    for x, nm in ((query_points, "query_points"), (query_width, "query_width"), (points, "points"),
                  (point_attrs, "point_attrs"), (node2point_index, "node2point_index"),
                  (node2point_indexstart, "node2point_indexstart"),
                  (node_children_list, "node_children_list"), (node_attrs, "node_attrs"),
                  (node_is_leaf_list, "node_is_leaf_list"), (node_half_w_list, "node_half_w_list"),
                  (node_reppoints, "node_reppoints"), (num_points_in_node, "num_points_in_node")):
        _check_input(x, nm)
    M = node_attrs.shape[0]
    # without a preceding scatter: the deepest node of the given tree is the
    # depth it was built to (a shallower cap would have stopped there, a deeper
    # one splits nothing more, as no deeper node exists)
    wn = _tree_for(points, M, lambda: int(round(-math.log2(float(node_half_w_list.min())))))
    dim = point_attrs.shape[1]
    dev = points.device
    with torch.cuda.device(dev):
        check(_lib.lib().cagr_scatter_import(
            wn.handle, 0, _ptr(node_attrs), _ptr(node_reppoints), _ptr(point_attrs), dim,
            _stream(dev)), "cagr_scatter_import")
    nq = query_points.shape[0]
    out = torch.zeros(nq, out_dim, dtype=points.dtype, device=dev)
    if nq == 0:
        return out
    # the tree's own points as queries: the walk groups them along its curve
    same = query_points.data_ptr() == points.data_ptr() and query_points.shape == points.shape
    q = None if same else query_points
    with torch.cuda.device(dev):
        check(_lib.lib().cagr_multiply(
            wn.handle, OPS[op], _ptr(q), None, nq, _ptr(query_width), 0.0, 0, _ptr(out),
            out.stride(0), _stream(dev)), f"cagr_multiply({op})")
    return out


def multiply_by_A(*args):
    return _multiply("A", *args, out_dim=1)


def multiply_by_A3(*args):
    return _multiply("A3", *args, out_dim=1)


def multiply_by_AT(*args):
    return _multiply("AT", *args, out_dim=3)


def multiply_by_G(*args):
    return _multiply("G", *args, out_dim=3)


def multiply_by_A2(*args):
    return _multiply("A2_FUSED", *args, out_dim=3)


def multiply_by_A21(*args):
    return _multiply("A21", *args, out_dim=1)


def multiply_by_A22(*args):
    return _multiply("A22", *args, out_dim=1)


def multiply_by_A23(*args):
    return _multiply("A23", *args, out_dim=1)


def multiply_by_A2T1(*args):
    return _multiply("A2T1", *args, out_dim=3)


def multiply_by_A2T2(*args):
    return _multiply("A2T2", *args, out_dim=3)


def multiply_by_A2T3(*args):
    return _multiply("A2T3", *args, out_dim=3)


def clear_cache() -> None:
    """Frees the cached device trees."""
    while _trees:
        _trees.popitem()[1][1].close()
