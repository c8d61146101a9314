"""Device-resident CAGR normal solve (the caller of the treecode hot path).

Restates main_CAGR.py (mayueji/CAGR, CUDA-based/main_CAGR.py:40-187):
normalise the cloud into the [-1/1.1, 1/1.1]^3 box, then 40 iterations with a
width schedule that shrinks linearly from wsmax to wsmin (:103) -- 31
steepest-descent-type steps (:105-118), a residual restart at i == 30
(:119-125), 9 CG-type steps (:126-144) -- and 8 WNNC G steps (:167-174).
Every operator application goes through the C ABI (A2k fused into one
traversal; the three A2Tk of a step fused into one, and in the
steepest-descent steps fused with the three of the right-hand side b, whose
moments are computed once).  The iteration stays on the
GPU: step lengths are device tensors, nothing is copied to the host until the
caller asks for the result.

Precision: operators in FP32 (the reference's dtype); the Krylov dot
products and norms accumulate in FP64 (the reference uses FP32 torch sums),
and so does the WNNC renormalisation.  This changes results only at rounding
level; parity with the reference is stated as normal-sign agreement.
"""
from __future__ import annotations

import dataclasses
import time

import numpy as np
import torch

from ._lib import CAGR_ERR_ALLOC, CagrError
from .wn_treecode import WindingNumberTreecode

# b's window table (cagr_b_window_table) takes at most this many widths
MAX_TABLE_WIDTHS = 64

# main_CAGR.py:74-82
PRESET_WIDTHS = {
    "l0": (0.002, 0.016),
    "l1": (0.01, 0.04),
    "l2": (0.02, 0.08),
    "l3": (0.03, 0.12),
    "l4": (0.04, 0.16),
    "l5": (0.05, 0.2),
}


def normalize_points(points_unnormalized: np.ndarray, bbox_scale: float = 1.1) -> np.ndarray:
    """main_CAGR.py:42-45 (float64), then cast to float32 as :47 does."""
    p = np.asarray(points_unnormalized, np.float64)
    center = (p.min(0) + p.max(0)) / 2.0
    length = (p.max(0) - p.min(0)).max()
    return ((p - center) * (2.0 / (length * bbox_scale))).astype(np.float32)


@dataclasses.dataclass
class SolveResult:
    normals: torch.Tensor          # [N, 3] in the points' dtype, the solved mu (area-weighted normals)
    residual_norm: float           # |r| after the steepest-descent phase (main_CAGR.py:165)
    rk_norm: float                 # |rk1| after the CG phase (main_CAGR.py:166)
    time_tree_s: float
    time_main_s: float
    operator_calls: int


def _dot(a: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
    return (a.double() * b.double()).sum()


def cagr_solve(points: torch.Tensor, wsmin: float, wsmax: float, iters: int = 40,
               n_sd: int = 30, lambda0: float = 0.0, wnnc_steps: int = 8,
               widths: torch.Tensor | None = None, max_tree_depth: int = 15,
               tree: WindingNumberTreecode | None = None, far_field: str = "reference",
               degree: int = 5, theta: float = 0.5) -> SolveResult:
    """Solve for mu on normalised float32 CUDA points [N, 3].

    widths: per-point base widths (main_CAGR.py:61 uses ones); each iteration
    uses widths * width_scale.  far_field / degree / theta: the tree's far-field
    mode when the tree is built here ("interp": the interpolated far field)."""
    dev = points.device
    n = points.shape[0]
    t0 = time.perf_counter()
    wn = tree if tree is not None else WindingNumberTreecode(
        points, max_tree_depth, far_field=far_field, degree=degree, theta=theta)
    torch.cuda.synchronize(dev)
    t1 = time.perf_counter()
    dt = points.dtype   # float32 as the reference runs it; float64 works alike
    base = torch.ones(n, device=dev, dtype=dt) if widths is None else widths
    normals = torch.zeros(n, 3, device=dev, dtype=dt)
    b = torch.full((n, 1), 0.5, device=dev, dtype=dt)   # main_CAGR.py:50
    calls = 0

    def A2(x, w):   # [A21 | A22 | A23](x)
        nonlocal calls
        calls += 3
        return wn.forward_A2(x, w)

    def A2T(v3, w):  # A2T1(v1) + A2T2(v2) + A2T3(v3)
        nonlocal calls
        calls += 3
        return wn.forward_A2T_sum(v3, w)

    def scale(i):
        return wsmin + ((iters - 1 - i) / (iters - 1)) * (wsmax - wsmin)

    # b is constant and the acceptance decisions do not depend on the width, so
    # A2Tb at every steepest-descent width comes from two walks per solve: b's
    # terms at r >= the largest of those widths (b_hi), and a table of b's terms
    # below it, bucketed by the step widths they pass (b_window_table); the
    # initial right-hand side, at the middle width, comes from the table too.
    # These widths are base * s with s rounded to the points' dtype, as the
    # table's kernel forms them.
    sd_steps = range(min(n_sd, iters - 1) + 1)
    s_of = {i: float(torch.tensor(scale(i), dtype=dt)) for i in sd_steps}
    s_mid = float(torch.tensor(wsmin + 0.5 * (wsmax - wsmin), dtype=dt))
    sd_scales = sorted(set(s_of.values()) | {s_mid})
    sc_t = torch.tensor(sd_scales, dtype=dt, device=dev)
    slot_of = {i: sd_scales.index(s_of[i]) for i in sd_steps}
    b_hi = b_table = None

    # more widths than the table takes: each step's four-slot walk adds b's
    # terms below the largest width itself
    use_table = len(sd_scales) <= MAX_TABLE_WIDTHS
    w_hi = base * sc_t[-1]
    # the interpolated far field has no per-query decisions to share between
    # widths: there each step evaluates A2Tb at its width
    interp = wn.far_field == "interp"

    def RHS(a_mu, i, w):  # A2Tb(w) - A2T(a_mu)
        nonlocal calls
        calls += 6
        if interp:
            return wn.forward_A2T_shared(b, w) - wn.forward_A2T_sum(a_mu, w)
        if use_table:
            return (b_hi + b_table[slot_of[i]]) - wn.forward_A2T_sum(a_mu, w)
        return wn.forward_A2T_rhs_window(a_mu, w, b_hi, w_hi)

    calls += 3   # the reference's A2T1..3(b) at the middle width (main_CAGR.py:98)
    if interp:
        rk1 = wn.forward_A2T_shared(b, base * sc_t[sd_scales.index(s_mid)])
    else:
        b_hi = wn.forward_A2T_shared(b, w_hi)
        wn.scatter(b, slot=1)   # b is constant: its moments serve every step
        if use_table:
            # an [S, N, 3] table: where the device has no room for it, each step
            # adds b's window itself (the four-slot walk, no table)
            try:
                b_table = wn.b_window_table(base, sc_t)
            except (torch.cuda.OutOfMemoryError, CagrError) as e:
                if isinstance(e, CagrError) and e.code != CAGR_ERR_ALLOC:
                    raise
                use_table, b_table = False, None
        if use_table:
            rk1 = b_hi + b_table[sd_scales.index(s_mid)]   # overwritten at i == n_sd
        else:
            rk1 = wn.forward_A2T_shared(b, base * sc_t[sd_scales.index(s_mid)])
    pk = rk1
    r = rk1
    for i in range(iters):
        w = base * sc_t[slot_of[i]] if i in slot_of else base * scale(i)
        if i <= n_sd:
            A_mu = -A2(normals, w)
            r = RHS(A_mu.contiguous(), i, w) - lambda0 * normals   # A2Tb(w) - A2T(A_mu)
            A_r = -A2(r.contiguous(), w).sum(1, keepdim=True)
            alpha = (_dot(r, r) / _dot(A_r, A_r)).to(dt)
            normals = normals + alpha * r
            if i == n_sd:
                A_mu = -A2(normals, w)
                rk1 = RHS(A_mu.contiguous(), i, w) - lambda0 * normals
                pk = rk1
        else:
            A_pk = -A2(pk.contiguous(), w)
            AT_A_pk = A2T(A_pk.contiguous(), w)
            den = _dot(AT_A_pk, pk) + lambda0 * _dot(pk, pk)
            alpha = (_dot(rk1, rk1) / den).to(dt)
            normals = normals + alpha * pk
            rk20 = rk1 - alpha * AT_A_pk - alpha * lambda0 * pk
            beta = (_dot(rk20, rk20) / _dot(rk1, rk1)).to(dt)
            pk = rk20 + beta * pk
            rk1 = rk20
    r_norm = torch.linalg.norm(r.double())
    rk_norm = torch.linalg.norm(rk1.double())
    # WNNC refinement at the last width (main_CAGR.py:167-174)
    for _ in range(wnnc_steps):
        calls += 1
        g = wn.forward_G(normals.contiguous(), w).double()
        g = g / torch.clamp(torch.linalg.norm(g, dim=-1, keepdim=True), min=1e-12)
        length = torch.linalg.norm(normals.double(), dim=-1, keepdim=True)
        normals = (g * length).to(dt).contiguous()
    torch.cuda.synchronize(dev)
    t2 = time.perf_counter()
    return SolveResult(normals, float(r_norm), float(rk_norm), t1 - t0, t2 - t1, calls)


def cagr_solve_autograd(points: torch.Tensor, wsmin: float, wsmax: float, iters: int = 40,
                        n_sd: int = 30, wnnc_steps: int = 8, widths: torch.Tensor | None = None,
                        max_tree_depth: int = 15,
                        tree: WindingNumberTreecode | None = None) -> SolveResult:
    """The CAGR solve driven through the differentiable operator
    (cagr_b200.autograd.convection_gauss) and its true adjoint.

    Objective per iteration, at main_CAGR.py's width of that iteration (:103):
        L(mu) = 1/2 sum_k || -A2k(mu) - b ||^2,   b = 1/2   (main_CAGR.py:50,107-110)
    -- the reference's three-block system, with J = -A2 (the fused A21/A22/A23),
    whose gradient the reference forms with its A2T operators; here
    grad L = J^T (J mu - b) comes from autograd, i.e. from the adjoint treecode
    kernel.  Steps: steepest descent with exact
    line search for i <= n_sd (:105-118), then CG on the normal equations
    J^T J mu = J^T b (:126-144; symmetric with the true adjoint), then the
    WNNC G steps (:167-174).  Dots and norms in FP64 as in cagr_solve."""
    from .autograd import convection_gauss
    dev = points.device
    n = points.shape[0]
    t0 = time.perf_counter()
    wn = tree if tree is not None else WindingNumberTreecode(points, max_tree_depth)
    torch.cuda.synchronize(dev)
    t1 = time.perf_counter()
    base = torch.ones(n, device=dev, dtype=points.dtype) if widths is None else widths
    b = torch.full((n, 1), 0.5, device=dev, dtype=points.dtype)
    calls = 0

    def J(x, w):                       # [N,3] -> [N,3]: the operator -A2 (no graph)
        nonlocal calls
        calls += 3
        with torch.no_grad():
            return -convection_gauss(wn, x, w)

    def JT(x, w, v):                   # J^T v at the moments of x (the adjoint kernel)
        nonlocal calls
        calls += 3
        xr = x.detach().requires_grad_(True)
        out = -convection_gauss(wn, xr, w)
        (g,) = torch.autograd.grad(out, xr, grad_outputs=v)
        return g

    def scale(i):
        return wsmin + ((iters - 1 - i) / (iters - 1)) * (wsmax - wsmin)

    normals = torch.zeros(n, 3, device=dev, dtype=points.dtype)
    r = rk = pk = None
    w = base * scale(0)
    for i in range(iters):
        w = base * scale(i)
        if i <= n_sd:
            res = b - J(normals, w)                       # b - J mu, [N,3]
            r = JT(normals, w, res)                       # -grad L
            Jr = J(r, w)
            alpha = (_dot(r, r) / _dot(Jr, Jr)).to(normals.dtype)
            normals = normals + alpha * r
            if i == n_sd:
                rk = JT(normals, w, b - J(normals, w))
                pk = rk
        else:
            Jp = J(pk, w)
            alpha = (_dot(rk, rk) / _dot(Jp, Jp)).to(normals.dtype)
            normals = normals + alpha * pk
            rk2 = rk - alpha * JT(pk, w, Jp)
            beta = (_dot(rk2, rk2) / _dot(rk, rk)).to(normals.dtype)
            pk = rk2 + beta * pk
            rk = rk2
    r_norm = torch.linalg.norm(r.double()) if r is not None else torch.zeros(())
    rk_norm = torch.linalg.norm(rk.double()) if rk is not None else torch.zeros(())
    for _ in range(wnnc_steps):
        calls += 1
        g = wn.forward_G(normals.contiguous(), w).double()
        g = g / torch.clamp(torch.linalg.norm(g, dim=-1, keepdim=True), min=1e-12)
        length = torch.linalg.norm(normals.double(), dim=-1, keepdim=True)
        normals = (g * length).to(points.dtype).contiguous()
    torch.cuda.synchronize(dev)
    t2 = time.perf_counter()
    return SolveResult(normals, float(r_norm), float(rk_norm), t1 - t0, t2 - t1, calls)


def orient_file(path_in: str, width_config: str = "l0", wsmin: float | None = None,
                wsmax: float | None = None, device: str = "cuda",
                iters: int = 40) -> tuple[np.ndarray, SolveResult]:
    """main_CAGR.py end to end for an .xyz/.npy file: returns [xyz, mu] rows as the
    reference writes them (:185-186)."""
    if path_in.endswith(".npy"):
        raw = np.load(path_in)[:, :3]
    else:
        raw = np.loadtxt(path_in)[:, :3]
    if width_config == "custom":
        lo, hi = wsmin, wsmax
    else:
        lo, hi = PRESET_WIDTHS[width_config]
    pts = torch.from_numpy(normalize_points(raw)).to(device)
    res = cagr_solve(pts, lo, hi, iters=iters)
    out = np.concatenate([raw, res.normals.cpu().numpy().astype(np.float64)], 1)
    return out, res
