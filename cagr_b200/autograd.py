"""Differentiable fused convection operator: torch.autograd.Function over the
treecode, with the hand-written adjoint treecode kernel as its backward.

    out = convection_gauss(tree, mu, widths, continuous=False)      # [N, 3]

computes (A21 mu, A22 mu, A23 mu) at the tree's own points -- the operator the
CAGR solve applies (main_CAGR.py:107,115,131) -- and is differentiable with
respect to mu and to the widths:

* d/d mu: `cagr_adjoint`, the exact adjoint of the forward treecode.  The
  forward's centroids are weighted by |mu| (wn_treecode_func.py:131) and
  decide which node terms each query takes; the derivative holds those weights
  fixed (as given by `weights`, by default |mu| detached), so for fixed
  weights the operator is linear in mu and the backward is its transpose: the
  same traversal recomputed, each pair term's derivative added into the node
  or point it used, then pushed from every node to its points.
* d/d widths: only the continuous kernel depends smoothly on a query's width
  (the pair terms inside the width, e^w (d.m/w^3 + m_k/(2w)) per direction,
  wn_treecode_cuda_kernels.cu:141-145); the width indicator itself is a step,
  whose derivative is zero wherever no pair sits exactly at r = w.  The
  backward recomputes the per-query inside sums D = sum d.m and M_k = sum m_k
  (CAGR_OP_A2_INSIDE) and applies
      d out_k / d w = e^w (D/w^3 + M_k/(2w) - 3 D/w^4 - M_k/(2 w^2)).
  For the discontinuous kernel the width gradient is zero.

The reference's own "transpose" operators A2T1..A2T3 (used by main_CAGR.py in
its normal equations) are a different operator (wn_treecode_cuda_kernels.cu
:263-379): this module's backward is the true adjoint of the forward.
"""
from __future__ import annotations

import torch

from .wn_treecode import WindingNumberTreecode


def _point_weights(mu: torch.Tensor) -> torch.Tensor:
    """|mu| per point as the reference computes it ((mu**2).sum(-1).sqrt())."""
    return (mu * mu).sum(-1).sqrt()


class ConvectionGaussA2(torch.autograd.Function):
    """forward(tree, mu [N,3], widths [N] or float, continuous, weights [N] or None)
    -> [N,3]; see the module docstring."""

    @staticmethod
    def forward(ctx, tree: WindingNumberTreecode, mu, widths, continuous: bool, weights):
        mu_d = mu.detach().contiguous()
        w_pts = _point_weights(mu_d) if weights is None else weights.detach().contiguous()
        per_point = torch.is_tensor(widths) and widths.dim() == 1
        wid = widths.detach().contiguous() if per_point else float(widths)
        tree.scatter(mu_d, weights=w_pts)
        out = tree.multiply("A2_FUSED", wid, continuous=continuous)
        ctx.tree, ctx.continuous, ctx.wid = tree, continuous, wid
        ctx.save_for_backward(mu_d, w_pts)
        return out

    @staticmethod
    def backward(ctx, grad_out):
        tree, cont, wid = ctx.tree, ctx.continuous, ctx.wid
        mu_d, w_pts = ctx.saved_tensors
        g = grad_out.contiguous().to(tree.dtype)
        # the forward's moments again (the slot may have been reused since)
        tree.scatter(mu_d, weights=w_pts)
        grad_mu = None
        if ctx.needs_input_grad[1]:
            grad_mu = tree.adjoint_A2(g, wid, continuous=cont)
        grad_w = None
        if ctx.needs_input_grad[2]:
            if cont:
                ins = tree.multiply("A2_INSIDE", wid, continuous=True)        # [N, 4]
                w = wid if torch.is_tensor(wid) else torch.full_like(ins[:, 0], wid)
                D, Mk = ins[:, 0:1], ins[:, 1:4]
                w1 = w.unsqueeze(1)
                dv = torch.exp(w1) * (D / w1 ** 3 + Mk / (2 * w1) - 3 * D / w1 ** 4
                                      - Mk / (2 * w1 * w1))                  # [N, 3]
                grad_w = (g * dv).sum(1)
            else:
                grad_w = torch.zeros(g.shape[0], dtype=g.dtype, device=g.device)
            if not torch.is_tensor(wid):
                grad_w = grad_w.sum()
        return None, grad_mu, grad_w, None, None


def convection_gauss(tree: WindingNumberTreecode, mu: torch.Tensor, widths,
                     continuous: bool = False, weights: torch.Tensor | None = None):
    """(A21 mu, A22 mu, A23 mu) at the tree's points, differentiable in mu and widths.
    weights: the per-point weights of the node centroids (default |mu|, held fixed
    under differentiation)."""
    return ConvectionGaussA2.apply(tree, mu, widths, continuous, weights)
