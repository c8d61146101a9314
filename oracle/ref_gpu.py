"""The reference's own CUDA kernels on the GPU (oracle/_ref/libwnref_gpu.so).

TEST AND BASELINE INFRASTRUCTURE ONLY: used by tests/ (GPU-to-GPU parity)
and by oracle/ref_gpu_bench.py (the reference GPU baseline rows).  Mirrors
one ``WindingNumberTreecode.forward_*`` call of the reference
(CUDA-based/ext/wn_treecode/wn_treecode_func.py:122-158): torch computes the
|value| weights, then the reference scatter and multiply kernels run on the
current stream.  Tree arrays are the reference layout (bit-identical to the
reference's CPU build_tree; here exported from the GPU build).
"""
from __future__ import annotations

import ctypes
import os

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libwnref_gpu.so")
OPS = {"A": 0, "AT": 1, "A3": 2, "A21": 3, "A22": 4, "A23": 5, "A2T1": 6, "A2T2": 7,
       "A2T3": 8, "G": 9}
OUT_DIM = {"A": 1, "AT": 3, "A3": 1, "A21": 1, "A22": 1, "A23": 1, "A2T1": 3, "A2T2": 3,
           "A2T3": 3, "G": 3}

_p = ctypes.c_void_p
_l = ctypes.c_long


class RefGPU:
    def __init__(self, path: str = LIB):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref-gpu`")
        L = ctypes.CDLL(path)
        L.wnref_gpu_scatter.restype = ctypes.c_int
        L.wnref_gpu_scatter.argtypes = [ctypes.c_int, _l] + [_p] * 5 + [_l] + [_p] * 4 + [_l] + [_p] * 6
        L.wnref_gpu_multiply.restype = ctypes.c_int
        L.wnref_gpu_multiply.argtypes = [ctypes.c_int, ctypes.c_int, _p, _p, _l] + [_p] * 11 + [ctypes.c_int, _p]
        L.wnref_gpu_last_error.restype = ctypes.c_char_p
        self.L = L

    @staticmethod
    def _ptr(t):
        return None if t is None else _p(t.data_ptr())

    def tree_from(self, wn) -> dict:
        """Reference-layout tree tensors of a cagr_b200 WindingNumberTreecode."""
        return dict(parent=wn.node_parent_list, children=wn.node_children_list,
                    is_leaf=wn.node_is_leaf_list, half_w=wn.node_half_w_list,
                    npts=wn.num_points_in_node, n2p=wn.node2point_index,
                    n2p_start=wn.node2point_indexstart, points=wn.points, depth=wn.tree_depth)

    def forward(self, op: str, tree: dict, values: torch.Tensor, widths: torch.Tensor,
                queries: torch.Tensor | None = None, continuous: bool = False) -> torch.Tensor:
        P = self._ptr
        pts = tree["points"]
        f64 = int(pts.dtype == torch.float64)
        M = tree["parent"].shape[0]
        dim = values.shape[1]
        weights = (values ** 2).sum(-1).sqrt()             # wn_treecode_func.py:131
        node_attrs = torch.empty(M, dim, dtype=pts.dtype, device=pts.device)
        rep = torch.empty(M, 3, dtype=pts.dtype, device=pts.device)
        node_w = torch.empty(M, dtype=pts.dtype, device=pts.device)
        masks = torch.empty(2, M, dtype=torch.bool, device=pts.device)
        stream = _p(torch.cuda.current_stream().cuda_stream)
        rc = self.L.wnref_gpu_scatter(
            f64, M, P(tree["parent"]), P(tree["children"]), P(pts), P(weights), P(values), dim,
            P(tree["n2p"]), P(tree["n2p_start"]), P(tree["npts"]), P(tree["is_leaf"]),
            tree["depth"], P(node_attrs), P(rep), P(node_w), P(masks[0]), P(masks[1]), stream)
        if rc:
            raise RuntimeError(f"reference scatter failed: {self.L.wnref_gpu_last_error().decode()}")
        q = pts if queries is None else queries
        out = torch.zeros(q.shape[0], OUT_DIM[op], dtype=pts.dtype, device=pts.device)
        rc = self.L.wnref_gpu_multiply(
            f64, OPS[op], P(q), P(widths), q.shape[0], P(pts), P(values), P(tree["n2p"]),
            P(tree["n2p_start"]), P(tree["children"]), P(node_attrs), P(tree["is_leaf"]),
            P(tree["half_w"]), P(rep), P(tree["npts"]), P(out), int(continuous), stream)
        if rc:
            raise RuntimeError(f"reference {op} launch failed: "
                               f"{self.L.wnref_gpu_last_error().decode()}")
        return out
