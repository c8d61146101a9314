"""CPU restatement of the CAGR normal solve.  TEST INFRASTRUCTURE ONLY.

Follows mayueji/CAGR CUDA-based/main_CAGR.py:40-174 line by line in float32
numpy (the reference's torch float32 arithmetic), with every operator call
composed as wn_treecode_func.py composes it (|value| weights, node moments,
traversal) on either oracle back end.  Used to pin the GPU solve and to check
the reference's published bunny output.
"""
from __future__ import annotations

import numpy as np

from .oracle import Oracle, point_weights

PRESET_WIDTHS = {"l0": (0.002, 0.016), "l1": (0.01, 0.04), "l2": (0.02, 0.08),
                 "l3": (0.03, 0.12), "l4": (0.04, 0.16), "l5": (0.05, 0.2)}


def normalize(points: np.ndarray) -> np.ndarray:
    p = np.asarray(points, np.float64)
    center = (p.min(0) + p.max(0)) / 2.0
    length = (p.max(0) - p.min(0)).max()
    return ((p - center) * (2.0 / (length * 1.1))).astype(np.float32)


class _Ops:
    def __init__(self, impl, points, max_depth: int = 15, leaf_size: int = 1):
        self.impl = impl
        self.p = points
        self.tree = impl.build_tree(points, max_depth, leaf_size)
        self.calls = 0

    def fwd(self, op, values, w):
        self.calls += 1
        values = np.ascontiguousarray(values, np.float32)
        mom = self.impl.moments(self.tree, self.p, point_weights(values), values)
        return self.impl.multiply(op, self.p, w, self.p, values, self.tree, mom)


def solve(points: np.ndarray, wsmin: float, wsmax: float, impl=None, iters: int = 40,
          n_sd: int = 30, lambda0: float = 0.0, wnnc_steps: int = 8,
          base_widths: np.ndarray | None = None, max_depth: int = 15,
          leaf_size: int = 1) -> np.ndarray:
    """points: normalised float32 [N, 3].  Returns mu [N, 3] float32.
    base_widths: per-point widths the schedule scales (main_CAGR.py:61 uses ones)."""
    impl = impl or Oracle()
    f32 = np.float32
    o = _Ops(impl, points, max_depth, leaf_size)
    n = points.shape[0]
    ones = np.ones(n, f32) if base_widths is None else np.ascontiguousarray(base_widths, f32)
    normals = np.zeros((n, 3), f32)
    b = np.full((n, 1), 0.5, f32)

    def A2T(v1, v2, v3, w):
        return o.fwd("A2T1", v1, w) + o.fwd("A2T2", v2, w) + o.fwd("A2T3", v3, w)

    width_scale = wsmin + 0.5 * (wsmax - wsmin)
    w = ones * f32(width_scale)
    rk1 = A2T(b, b, b, w)
    pk = rk1
    r = rk1
    for i in range(iters):
        width_scale = wsmin + ((iters - 1 - i) / (iters - 1)) * (wsmax - wsmin)
        w = ones * f32(width_scale)
        if i <= n_sd:
            A1, A2_, A3_ = (-o.fwd(op, normals, w) for op in ("A21", "A22", "A23"))
            AT_A_mu = A2T(A1, A2_, A3_, w)
            r = A2T(b, b, b, w) - AT_A_mu - f32(lambda0) * normals
            A_r = -(o.fwd("A21", r, w) + o.fwd("A22", r, w) + o.fwd("A23", r, w))
            alpha = f32((r * r).sum(dtype=f32) / (A_r * A_r).sum(dtype=f32))
            normals = normals + alpha * r
            if i == n_sd:
                A1, A2_, A3_ = (-o.fwd(op, normals, w) for op in ("A21", "A22", "A23"))
                AT_A_mu = A2T(A1, A2_, A3_, w)
                rk1 = A2T(b, b, b, w) - AT_A_mu - f32(lambda0) * normals
                pk = rk1
        else:
            P1, P2, P3 = (-o.fwd(op, pk, w) for op in ("A21", "A22", "A23"))
            T1, T2, T3 = o.fwd("A2T1", P1, w), o.fwd("A2T2", P2, w), o.fwd("A2T3", P3, w)
            den = ((T3 * pk) + (T2 * pk) + (T1 * pk)).sum(dtype=f32) + f32(lambda0) * (pk * pk).sum(dtype=f32)
            alpha = f32((rk1 * rk1).sum(dtype=f32) / den)
            normals = normals + alpha * pk
            rk20 = rk1 - alpha * T1 - alpha * T2 - alpha * T3 - alpha * f32(lambda0) * pk
            beta = f32((rk20 * rk20).sum(dtype=f32) / (rk1 * rk1).sum(dtype=f32))
            pk = rk20 + beta * pk
            rk1 = rk20
    for _ in range(wnnc_steps):
        g = o.fwd("G", normals, w)
        g = g / np.maximum(np.linalg.norm(g, axis=-1, keepdims=True), f32(1e-12))
        length = np.linalg.norm(normals, axis=-1, keepdims=True)
        normals = (g * length).astype(f32)
    return normals


def sign_agreement(mu_a: np.ndarray, mu_b: np.ndarray) -> float:
    """Fraction of points whose two normals point the same way (dot > 0)."""
    return float(((mu_a * mu_b).sum(1) > 0).mean())


def solve_torch(points, wsmin: float, wsmax: float, fwd, iters: int = 40, n_sd: int = 30,
                lambda0: float = 0.0, wnnc_steps: int = 8):
    """The reference solve in torch float32 on the points' device, line for
    line as main_CAGR.py:93-174 writes it (its sums, its step lengths, its
    float32 arithmetic), with every operator call made through
    ``fwd(op, values, widths) -> tensor`` -- one ``forward_*`` call of the
    reference (wn_treecode_func.py:122-158), e.g. ``RefGPU.forward`` for the
    reference's own CUDA kernels.  widths = ones (main_CAGR.py:61)."""
    import torch
    import torch.nn.functional as F
    n = points.shape[0]
    dev = points.device
    normals = torch.zeros(n, 3, device=dev)
    b = torch.ones(n, 1, device=dev) * 0.5
    widths = torch.ones(n, device=dev)

    def A2T(v1, v2, v3, w):
        return fwd("A2T1", v1, w) + fwd("A2T2", v2, w) + fwd("A2T3", v3, w)

    width_scale = wsmin + 0.5 * (wsmax - wsmin)
    rk1 = A2T(b, b, b, widths * width_scale)
    pk = rk1
    for i in range(iters):
        width_scale = wsmin + ((iters - 1 - i) / (iters - 1)) * (wsmax - wsmin)
        w = widths * width_scale
        if i <= n_sd:
            A1, A2_, A3_ = (-fwd(op, normals, w) for op in ("A21", "A22", "A23"))
            AT_A_mu = A2T(A1, A2_, A3_, w)
            r = A2T(b, b, b, w) - AT_A_mu - lambda0 * normals
            A_r = -(fwd("A21", r, w) + fwd("A22", r, w) + fwd("A23", r, w))
            alpha = (r * r).sum() / (A_r * A_r).sum()
            normals = normals + alpha * r
            if i == n_sd:
                A1, A2_, A3_ = (-fwd(op, normals, w) for op in ("A21", "A22", "A23"))
                AT_A_mu = A2T(A1, A2_, A3_, w)
                rk1 = A2T(b, b, b, w) - AT_A_mu - lambda0 * normals
                pk = rk1
        else:
            P1, P2, P3 = (-fwd(op, pk, w) for op in ("A21", "A22", "A23"))
            T1, T2, T3 = fwd("A2T1", P1, w), fwd("A2T2", P2, w), fwd("A2T3", P3, w)
            alpha = (rk1 * rk1).sum() / (((T3 * pk) + (T2 * pk) + (T1 * pk)).sum()
                                         + lambda0 * (pk * pk).sum())
            normals = normals + alpha * pk
            rk20 = rk1 - alpha * T1 - alpha * T2 - alpha * T3 - alpha * lambda0 * pk
            beta = (rk20 * rk20).sum() / (rk1 * rk1).sum()
            pk = rk20 + beta * pk
            rk1 = rk20
    for _ in range(wnnc_steps):
        g = F.normalize(fwd("G", normals, w), dim=-1).contiguous()
        normals = g * torch.linalg.norm(normals, dim=-1, keepdim=True)
    return normals
