"""GPU: the differentiable fused convection operator (cagr_b200.autograd) and
its backward, the adjoint treecode kernel (cagr_adjoint, CAGR_OP_A2_INSIDE).

* the adjoint equals the transpose of the forward's matrix, built column by
  column from the forward on unit vectors (FP64, both kernels, per-point
  widths) -- with the centroid weights held fixed the forward is linear;
* gradients w.r.t. mu and widths equal FP64 central finite differences
  (h = 1e-6) on 64 random directions each (error / (|grad| |direction|) below
  1e-8; the difference quotients carry rounding of that order, shrinking as
  1/h: 2e-8 at h = 1e-6, 1e-11 at h = 1e-3), on the 200,000-point thin-structure
  workload (closed 1 x 1 x 0.01 box + hollow cylinder of wall 0.005, 1 %
  uniform outliers) with per-point widths 1.5 x the mean 10-NN distance;
  width directions move only queries none of whose pair terms lies within
  1e-5 of its width (there the width indicator is a step and the derivative
  is the continuous kernel's);
* with the exact gradient every steepest-descent step with exact line search
  lowers the CAGR least-squares objective; the CAGR schedule runs through the
  autograd operator.
"""
import numpy as np
import pytest

from tests._cases import edge_cloud, sphere_cloud

pytestmark = pytest.mark.gpu


def _knn_widths(p, k=10, scale=1.5):
    from scipy.spatial import cKDTree
    d, _ = cKDTree(p).query(p, k=k + 1, workers=-1)
    return scale * d[:, 1:].mean(1)


@pytest.mark.parametrize("cloud", ["sphere", "edge"])
@pytest.mark.parametrize("continuous", [False, True])
def test_adjoint_equals_the_transpose_of_the_forward(cuda_lib, continuous, cloud):
    """(the edge cloud has duplicate points, hence multi-point leaves at the
    maximum depth, points on split planes and outside the unit box)"""
    import torch
    from cagr_b200 import WindingNumberTreecode
    n = 192
    pts = (sphere_cloud(n, seed=70, dtype=np.float64) if cloud == "sphere"
           else edge_cloud(n, seed=74, dtype=np.float64))
    rng = np.random.default_rng(71)
    mu0 = torch.from_numpy(rng.normal(size=(n, 3)) / n).cuda()
    wt = torch.from_numpy(np.abs(rng.normal(size=n)) + 0.1).cuda()   # fixed centroid weights
    # (coincident points: a positive floor keeps r = 0 pairs inside the width)
    widths = torch.from_numpy(_knn_widths(pts, k=4) + 0.01).cuda()
    tree = WindingNumberTreecode(torch.from_numpy(pts).cuda())
    cols = []
    for j in range(n):
        for c in range(3):
            e = torch.zeros(n, 3, dtype=torch.float64, device="cuda")
            e[j, c] = 1.0
            tree.scatter(e, weights=wt)
            cols.append(tree.multiply("A2_FUSED", widths, continuous=continuous).reshape(-1))
    Jm = torch.stack(cols, 1)                          # d out / d mu, [3n, 3n]
    g = torch.from_numpy(rng.normal(size=(n, 3))).cuda()
    tree.scatter(mu0, weights=wt)
    got = tree.adjoint_A2(g, widths, continuous=continuous).reshape(-1)
    ref = Jm.T @ g.reshape(-1)
    err = (torch.linalg.norm(got - ref) / torch.linalg.norm(ref)).item()
    assert err < 1e-12, err
    # the forward itself is the same matrix
    out = tree.multiply("A2_FUSED", widths, continuous=continuous).reshape(-1)
    assert torch.allclose(out, Jm @ mu0.reshape(-1), rtol=1e-12, atol=1e-18)


@pytest.fixture(scope="module")
def thin_case():
    import torch
    from cagr_b200 import WindingNumberTreecode
    from cagr_b200 import synthetic as S
    p = S.normalize(S.make("thin")).astype(np.float64)
    n = len(p)
    widths = torch.from_numpy(_knn_widths(p)).cuda()
    rng = np.random.default_rng(72)
    c = p - p.mean(0)
    mu0 = c / np.linalg.norm(c, axis=1, keepdims=True) * (4.0 / n) + rng.normal(size=(n, 3)) / (4 * n)
    g = rng.normal(size=(n, 3))
    tree = WindingNumberTreecode(torch.from_numpy(p).cuda())
    return tree, torch.from_numpy(mu0).cuda(), widths, torch.from_numpy(g).cuda(), rng


@pytest.mark.parametrize("continuous", [False, True])
def test_mu_gradient_matches_fp64_central_differences(cuda_lib, thin_case, continuous):
    import torch
    from cagr_b200.autograd import convection_gauss
    tree, mu0, widths, g, rng = thin_case
    wt = (mu0 * mu0).sum(1).sqrt()

    def loss(mu):
        with torch.no_grad():
            return (g * convection_gauss(tree, mu, widths, continuous, wt)).sum().item()

    mu = mu0.clone().requires_grad_(True)
    (g * convection_gauss(tree, mu, widths, continuous, wt)).sum().backward()
    grad = mu.grad
    h = 1e-6
    worst = 0.0
    for _ in range(64):
        v = torch.from_numpy(rng.normal(size=mu0.shape)).cuda() * (4.0 / len(mu0))
        fd = (loss(mu0 + h * v) - loss(mu0 - h * v)) / (2 * h)
        ad = (grad * v).sum().item()
        # error on the scale of the directional derivative, |grad| |v| (a plain
        # relative error blows up for directions nearly orthogonal to grad)
        worst = max(worst, abs(fd - ad) / (torch.linalg.norm(grad) * torch.linalg.norm(v)).item())
    assert worst < 1e-8, worst


def test_width_gradient_matches_fp64_central_differences(cuda_lib, thin_case):
    import torch
    from cagr_b200.autograd import convection_gauss
    tree, mu0, widths, g, rng = thin_case
    wt = (mu0 * mu0).sum(1).sqrt()
    # queries with no pair term within 1e-5 of their width: same inside set at w -+ 1e-5
    tree.scatter(mu0, weights=wt)
    ins_lo = tree.multiply("A2_INSIDE", widths - 1e-5, continuous=True)
    ins_hi = tree.multiply("A2_INSIDE", widths + 1e-5, continuous=True)
    safe = (ins_lo == ins_hi).all(1)
    assert safe.float().mean().item() > 0.9
    inside_any = (ins_hi[:, 1:] != 0).any(1) & safe
    assert inside_any.sum().item() > 1000   # the continuous branch is exercised

    def loss(w):
        with torch.no_grad():
            return (g * convection_gauss(tree, mu0, w, True, wt)).sum().item()

    w = widths.clone().requires_grad_(True)
    (g * convection_gauss(tree, mu0, w, True, wt)).sum().backward()
    grad = w.grad
    h = 1e-6
    worst = 0.0
    for _ in range(64):
        v = torch.from_numpy(np.clip(rng.normal(size=len(widths)), -4, 4)).cuda() * safe
        fd = (loss(widths + h * v) - loss(widths - h * v)) / (2 * h)
        ad = (grad * v).sum().item()
        worst = max(worst, abs(fd - ad) / (torch.linalg.norm(grad * safe) * torch.linalg.norm(v)).item())
    assert worst < 1e-8, worst
    # the discontinuous kernel has no width derivative
    w2 = widths.clone().requires_grad_(True)
    (g * convection_gauss(tree, mu0, w2, False, wt)).sum().backward()
    assert torch.count_nonzero(w2.grad).item() == 0


def test_exact_gradient_steps_descend(cuda_lib):
    """With the true adjoint, the steepest-descent step with exact line search
    lowers L(mu) = 1/2 sum_k ||-A2k mu - b||^2 at a fixed width every time (the
    centroid weights |mu| move with mu, so the check is of the method, not of
    an identity)."""
    import torch
    from cagr_b200 import WindingNumberTreecode
    from cagr_b200.autograd import convection_gauss
    pts = torch.from_numpy(sphere_cloud(20000, seed=73)).cuda()
    wn = WindingNumberTreecode(pts)
    w, b = 0.01, torch.full((len(pts), 1), 0.5, device="cuda")

    def J(x):
        with torch.no_grad():
            return -convection_gauss(wn, x, w)

    mu = torch.zeros_like(pts)
    for _ in range(6):
        res = J(mu) - b
        L0 = 0.5 * (res.double() ** 2).sum().item()
        x = mu.clone().requires_grad_(True)
        (g,) = torch.autograd.grad(-convection_gauss(wn, x, w), x, grad_outputs=-res)
        r = g                                           # -grad L = J^T (b - J mu)
        Jr = J(r)
        alpha = ((r.double() ** 2).sum() / (Jr.double() ** 2).sum()).float()
        mu = mu + alpha * r
        L1 = 0.5 * ((J(mu) - b).double() ** 2).sum().item()
        assert L1 < L0, (L0, L1)


def test_autograd_solve_runs_the_schedule(cuda_lib):
    """The CAGR schedule driven through the autograd operator (measured
    orientation agreement on this sphere: 0.883 at preset l1; the reference's
    own iteration, which uses its A2T operators instead of the adjoint, reaches
    more: see the design notes)."""
    import torch
    from cagr_b200.solver import PRESET_WIDTHS, cagr_solve_autograd
    pts = sphere_cloud(20000, seed=73)
    P = torch.from_numpy(pts).cuda()
    res = cagr_solve_autograd(P, *PRESET_WIDTHS["l1"])
    assert torch.isfinite(res.normals).all()
    agree = ((res.normals * P).sum(1) > 0).float().mean().item()
    assert agree >= 0.85, agree


@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_backward_is_bitwise_repeatable(cuda_lib, dtype):
    """The adjoint accumulates in 64-bit fixed point (integer atomics, whose sum
    does not depend on the order the warps arrive in): the same inputs give the
    same gradient bits on every run, on 200,000 points with per-point widths."""
    import torch
    from cagr_b200 import WindingNumberTreecode
    from cagr_b200 import synthetic as S
    dt = getattr(torch, dtype)
    p = S.normalize(S.make("thin")).astype(np.float64)
    n = len(p)
    rng = np.random.default_rng(75)
    widths = torch.from_numpy(_knn_widths(p)).to("cuda", dt)
    mu = torch.from_numpy(rng.normal(size=(n, 3)) / n).to("cuda", dt)
    g = torch.from_numpy(rng.normal(size=(n, 3))).to("cuda", dt)
    tree = WindingNumberTreecode(torch.from_numpy(p).to("cuda", dt))
    tree.scatter(mu, weights=(mu * mu).sum(1).sqrt())
    for continuous in (False, True):
        runs = [tree.adjoint_A2(g, widths, continuous=continuous) for _ in range(3)]
        assert torch.isfinite(runs[0]).all()
        assert torch.count_nonzero(runs[0]).item() > 0
        for r in runs[1:]:
            assert torch.equal(r, runs[0])
