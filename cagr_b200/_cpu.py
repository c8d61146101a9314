"""Drop-in for ``build_tree`` of the reference's extension ``wn_treecode._cpu``.

The reference builds its octree on the host for both of its back ends
(wn_treecode_func.py:23, ``wn_treecode._cpu.build_tree(points.cpu(),
tree_depth)``; wn_treecode_cpu_torch_interface.cpp:104-118 -> :42-102) and
returns seven CPU tensors.  Here the same tree (bit for bit) is built on the
GPU by libcagr_b200.so and returned in that layout on the host:

    build_tree(points_cpu [N, 3] float32/float64, max_depth)
      -> [node_parent_list [M] i64, node_children_list [M, 8] i64,
          node_is_leaf_list [M] bool, node_half_w_list [M] (points dtype),
          num_points_in_node [M] i64, node2point_index [L] i64,
          node2point_indexstart [M] i64]

The reference module's host treecode (scatter and multiply on CPU tensors)
has no counterpart: this library evaluates on the GPU only, and those names
raise RuntimeError.
"""
from __future__ import annotations

import torch

from .wn_treecode import WindingNumberTreecode


def build_tree(points_tensor: torch.Tensor, max_depth: int):
    if points_tensor.is_cuda:
        raise RuntimeError("points_tensor must be a CPU tensor")
    if not points_tensor.is_contiguous():
        raise RuntimeError("points_tensor must be contiguous")
    if points_tensor.dtype not in (torch.float32, torch.float64):
        raise RuntimeError(f"build_tree not implemented for dtype '{points_tensor.dtype}'")
    if not torch.cuda.is_available():
        raise RuntimeError("build_tree builds the octree on the GPU: no CUDA device")
    dev = torch.device("cuda", torch.cuda.current_device())
    wn = WindingNumberTreecode(points_tensor.to(dev), max_tree_depth=int(max_depth))
    try:
        arrays = [wn.node_parent_list, wn.node_children_list, wn.node_is_leaf_list,
                  wn.node_half_w_list, wn.num_points_in_node, wn.node2point_index,
                  wn.node2point_indexstart]
        return [a.cpu() for a in arrays]
    finally:
        wn.close()


def _no_host_treecode(*args, **kwargs):
    raise RuntimeError("the host treecode of the reference's _cpu module has no counterpart in "
                       "cagr_b200, which evaluates on the GPU: pass CUDA tensors")


scatter_point_attrs_to_nodes = _no_host_treecode
multiply_by_A = _no_host_treecode
multiply_by_AT = _no_host_treecode
multiply_by_G = _no_host_treecode
