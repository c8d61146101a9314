"""GPU: the interpolated far-field mode (CAGR_FAR_INTERP).

The same operators as the reference mode with the far field interpolated on
Chebyshev proxy grids (degree p per axis) and one acceptance test per warp of
32 queries.  Checked against:
  * the FP64 direct sum (the exact operator): the torus workload (100k
    points, leaf 32, theta 0.5, 20,000 random queries in [-1.5, 1.5]^3,
    width 0.01): max |A - direct| and max |A3 - direct| <= 1e-4 in float32
    (the reference algorithm's own error there is ~0.4);
  * the oracle's FP64 restatement of the same algorithm (same tree, same query
    groups): every operator, float32 within rounding, float64 to ~1e-12;
  * itself: bit-identical on repeated calls; the reference mode unchanged
    after switching back.
"""
import numpy as np
import pytest

from tests._cases import edge_cloud, random_values, rel_errors, smooth_normals, sphere_cloud

pytestmark = pytest.mark.gpu

OPS_VEC = ["A", "A3", "A21", "A22", "A23", "G", "A2_FUSED"]
OPS_SCALAR = ["AT", "A2T1", "A2T2", "A2T3", "A2T_SUM_SHARED"]


def _torus():
    from cagr_b200 import synthetic as S
    raw = S.make("torus")
    p64 = S.normalize(raw)
    scale = np.linalg.norm(p64[1] - p64[0]) / np.linalg.norm(raw[1] - raw[0])
    area = 4 * np.pi ** 2 * 1.0 * 0.3 * scale ** 2
    phi = np.arctan2(raw[:, 1], raw[:, 0])
    core = np.stack([np.cos(phi), np.sin(phi), np.zeros_like(phi)], 1)
    n = raw - core
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    return p64.astype(np.float32), (n * (area / len(raw))).astype(np.float32)


@pytest.mark.parametrize("degree", [5, 6])
def test_torus_field_within_1e_4_of_the_fp64_direct_sum(cuda_lib, oracle, degree):
    import torch
    from cagr_b200 import WindingNumberTreecode
    from cagr_b200.wn_treecode import morton_order
    p, mu = _torus()
    rng = np.random.default_rng(81)
    q = rng.uniform(-1.5, 1.5, size=(20000, 3)).astype(np.float32)
    width = 0.01
    wq = np.full(len(q), width, np.float32)
    wn = WindingNumberTreecode(torch.from_numpy(p).cuda(), leaf_size=32, far_field="interp",
                               degree=degree, theta=0.5)
    Q = torch.from_numpy(q).cuda()
    order = morton_order(Q)
    wn.scatter(torch.from_numpy(mu).cuda())
    tr = oracle.build_tree(p, leaf_size=32)
    for op, cont in (("A", False), ("A3", True)):
        gpu = wn.multiply(op, width, queries=Q, query_order=order,
                          continuous=cont).cpu().numpy()[:, 0].astype(np.float64)
        direct = oracle.direct(op, q, wq, p, mu, continuous=cont)[:, 0]
        err = np.abs(gpu - direct).max()
        print(f"torus 100k, degree {degree}, {op}: max |gpu - direct| = {err:.3e}")
        assert err <= 1e-4, (op, degree, err)
        # the same algorithm in FP64 (same groups): float32 rounding only
        ref = oracle.interp(op, q, wq, p, mu, tr, degree=degree, order=order.cpu().numpy(),
                            continuous=cont)[:, 0]
        assert np.abs(gpu - ref).max() <= 2e-5, (op, np.abs(gpu - ref).max())


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_every_operator_against_the_fp64_restatement(cuda_lib, oracle, dtype):
    import torch
    from cagr_b200 import WindingNumberTreecode
    pts = sphere_cloud(20000, seed=50, dtype=dtype)
    P = torch.from_numpy(pts).cuda()
    wn = WindingNumberTreecode(P, far_field="interp", degree=4, theta=0.5, direct_max=32)
    order = wn.query_groups().cpu().numpy()
    tr = oracle.build_tree(pts)
    w = np.random.default_rng(51).uniform(0.005, 0.02, len(pts)).astype(dtype)
    W = torch.from_numpy(w).cuda()
    mu = smooth_normals(pts, seed=52)
    s = random_values(len(pts), 1, seed=53, dtype=dtype)
    s3 = random_values(len(pts), 3, seed=54, dtype=dtype)
    tol = 2e-5 if dtype == np.float32 else 1e-10
    cases = [(op, mu, False) for op in OPS_VEC] + [(op, s, False) for op in OPS_SCALAR]
    cases += [("A3", mu, True), ("A2_FUSED", mu, True), ("A", mu, True), ("A2T_SUM", s3, False)]
    for op, vals, cont in cases:
        V = torch.from_numpy(vals).cuda()
        if op == "A2T_SUM":
            got = wn.forward_A2T_sum(V, W)
        else:
            wn.scatter(V)
            got = wn.multiply(op, W, continuous=cont)
        want = oracle.interp(op, pts, w, pts, vals, tr, degree=4, direct_max=32, order=order,
                             continuous=cont)
        l2, mx = rel_errors(got.cpu().numpy(), want)
        assert l2 <= tol and mx <= 20 * tol, (op, cont, l2, mx)
    # pair terms per query: the same interactions (groups and decisions)
    wn.scatter(torch.from_numpy(mu).cuda())
    cnt = wn.multiply("COUNT", W).cpu().numpy()[:, 0].astype(np.int64)
    _, terms = oracle.interp("COUNT", pts, w, pts, mu, tr, degree=4, direct_max=32, order=order,
                             counts=True)
    assert (cnt == terms).mean() >= 0.999, (cnt != terms).sum()


def test_repeatable_bits_and_switching_back(cuda_lib):
    import torch
    from cagr_b200 import WindingNumberTreecode
    pts = sphere_cloud(30000, seed=60)
    P = torch.from_numpy(pts).cuda()
    mu = torch.from_numpy(smooth_normals(pts, seed=61)).cuda()
    W = torch.full((len(pts),), 0.01, device="cuda")
    ref_tree = WindingNumberTreecode(P)
    want = ref_tree.forward_A2(mu, W)
    wn = WindingNumberTreecode(P)
    wn.set_far_field("interp", degree=5)
    assert wn.far_field_info()["mode"] == "interp"
    assert wn.far_field_info()["proxy_grids"] > 0
    a = wn.forward_A2(mu, W)
    b = wn.forward_A2(mu, W)
    assert torch.equal(a, b)
    # closer to the exact sum than the reference's algorithm, same scale
    assert torch.linalg.norm(a - want) <= 0.2 * torch.linalg.norm(want)
    wn.set_far_field("reference")
    assert torch.equal(wn.forward_A2(mu, W), want)


def test_edge_cloud_grid_and_empty_queries(cuda_lib, oracle):
    import torch
    from cagr_b200 import WindingNumberTreecode
    from cagr_b200.mesh import field_grid
    pts = edge_cloud(3000)
    P = torch.from_numpy(pts).cuda()
    wn = WindingNumberTreecode(P, far_field="interp", degree=3, direct_max=8)
    mu = smooth_normals(pts, seed=70)
    wn.scatter(torch.from_numpy(mu).cuda())
    w = np.full(len(pts), 0.01, np.float32)
    got = wn.multiply("A3", 0.01, continuous=True).cpu().numpy()
    assert np.isfinite(got).all()
    tr = oracle.build_tree(pts)
    want = oracle.interp("A3", pts, w, pts, mu, tr, degree=3, direct_max=8,
                         order=wn.query_groups().cpu().numpy(), continuous=True)
    l2, _ = rel_errors(got, want)
    assert l2 <= 2e-5, l2
    # grid queries (Morton groups of the grid) against explicit queries at the
    # same nodes, and against the direct sum
    g = 24
    field = field_grid(wn, (g, g, g), (-1.1, -1.1, -1.1), 2.2 / (g - 1), 0.01).cpu().numpy()
    idx = np.stack(np.meshgrid(np.arange(g), np.arange(g), np.arange(g), indexing="ij"), -1)
    q = (idx.reshape(-1, 3).astype(np.float64) * np.float64(np.float32(2.2 / (g - 1)))
         + np.float64(np.float32(-1.1))).astype(np.float32)
    direct = oracle.direct("A3", q, np.full(len(q), 0.01), pts, mu, continuous=True)[:, 0]
    gv = field[idx[..., 2].ravel(), idx[..., 1].ravel(), idx[..., 0].ravel()]
    assert np.abs(gv - direct).max() <= 1e-3 * max(1.0, np.abs(direct).max())
    empty = wn.multiply("A3", 0.01, queries=torch.empty(0, 3, device="cuda"), continuous=True)
    assert empty.shape == (0, 1)


def test_interp_solve_orients_the_bunny(cuda_lib):
    """The CAGR schedule with the interpolated operators: normal signs of the
    reference's published bunny output (stable 10-step l0 schedule)."""
    import os
    import torch
    from cagr_b200.solver import PRESET_WIDTHS, cagr_solve, normalize_points
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "bunny.npz"))
    pts = torch.from_numpy(normalize_points(g["points"])).cuda()
    res = cagr_solve(pts, *PRESET_WIDTHS["l0"], iters=10, far_field="interp", degree=5)
    mu = res.normals.cpu().numpy()
    assert np.isfinite(mu).all()
    agree = float(((mu * g["mu_reference"]).sum(1) > 0).mean())
    assert agree >= 0.995, agree


def test_interp_rejects_reference_only_calls(cuda_lib):
    import torch
    from cagr_b200 import WindingNumberTreecode
    from cagr_b200._lib import CagrError
    pts = sphere_cloud(5000, seed=80)
    wn = WindingNumberTreecode(torch.from_numpy(pts).cuda(), far_field="interp")
    mu = torch.from_numpy(smooth_normals(pts, seed=81)).cuda()
    wn.scatter(mu)
    with pytest.raises(CagrError):
        wn.adjoint_A2(mu, 0.01)
    with pytest.raises(CagrError):
        wn.scatter_export()
    with pytest.raises(CagrError):
        wn.set_far_field("interp", degree=9)
    with pytest.raises(CagrError):
        wn.set_far_field("interp", theta=1.5)


def test_an_abandoned_staging_wait_is_reported(cuda_lib):
    """Every wait of the walk for its staged records is bounded.  With the
    bound set to zero every walk abandons its first wait: it must report it
    (cagr_tree_far_field returns CAGR_ERR_CUDA), land its copies in flight and
    stop, leaving the context usable."""
    import torch
    from cagr_b200 import WindingNumberTreecode, _lib
    from cagr_b200._lib import CagrError
    pts = sphere_cloud(20000, seed=90)
    P = torch.from_numpy(pts).cuda()
    mu = torch.from_numpy(smooth_normals(pts, seed=91)).cuda()
    wn = WindingNumberTreecode(P, far_field="interp")
    _lib.check(_lib.lib().cagr_debug_interp_wait_limit(wn.handle, 0), "wait limit")
    wn.forward_A2(mu, 0.01)
    with pytest.raises(CagrError, match="staging wait"):
        wn.far_field_info()
    # the device and a fresh tree still work, with the same results as before
    ok = WindingNumberTreecode(P, far_field="interp")
    a = ok.forward_A2(mu, 0.01)
    b = WindingNumberTreecode(P, far_field="interp").forward_A2(mu, 0.01)
    assert torch.equal(a, b)
    assert ok.far_field_info()["mode"] == "interp"
