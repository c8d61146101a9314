"""GPU: the workload configurations other than the 1M-point benchmark.

* 5,000 points on the unit sphere, octree leaf 16 / depth 8, per-point width
  1.5 x the mean 10-NN distance: tree bit-exact and operators within the FP32
  tolerance against the reference's own kernels compiled for the host; the
  full solve (repo-default 40 iterations + 8 G steps) agrees in normal sign
  with the same solve on the host reference, at those widths and at 1/4 of
  them; the 128^3 reconstruction is a closed outward sphere.
* 100,000 points on a torus, leaf 32: the FP32 treecode field at 20,000
  random queries in [-1.5, 1.5]^3 equals the reference algorithm in FP32
  (same decisions) within FP32 rounding, and its error against the FP64 direct
  sum is the reference algorithm's own (the theta = 1/2 monopole rule, as its
  FP64 treecode shows); the 256^3 field runs.
* 4,000,000 points on a level set of 32 Gaussian blobs: the full pipeline
  (solve, 512^3 field, marching cubes) in FP32, and the 512^3 field at 20,000
  seeded grid nodes against the reference's kernels built for the host with
  the same normals (and against the FP64 form of the field).
"""
import numpy as np
import pytest

from tests._cases import rel_errors

pytestmark = pytest.mark.gpu


def _knn_widths(p, k=10, scale=1.5):
    from scipy.spatial import cKDTree
    d, _ = cKDTree(p).query(p, k=k + 1, workers=-1)
    return (scale * d[:, 1:].mean(1)).astype(p.dtype)


def test_sphere_5k_leaf16_depth8_against_the_reference(cuda_lib):
    import torch
    from cagr_b200 import WindingNumberTreecode
    from cagr_b200 import synthetic as S
    from cagr_b200.mesh import reconstruct
    from cagr_b200.solver import cagr_solve
    from oracle.oracle import RefOracle
    from oracle.solve import sign_agreement
    from oracle.solve import solve as host_solve
    ref = RefOracle()
    p = S.normalize(S.make("sphere")).astype(np.float32)
    w = _knn_widths(p)
    P, W = torch.from_numpy(p).cuda(), torch.from_numpy(w).cuda()
    wn = WindingNumberTreecode(P, max_tree_depth=8, leaf_size=16)
    tr = ref.build_tree(p, 8, 16)
    got = [t.cpu().numpy() for t in (wn.node_parent_list, wn.node_children_list,
                                       wn.node_is_leaf_list, wn.node_half_w_list,
                                       wn.num_points_in_node, wn.node2point_index,
                                       wn.node2point_indexstart)]
    for a, b in zip(got, tr.as_tuple()):
        assert np.array_equal(a, b)
    # operators against the reference kernels (host build)
    rng = np.random.default_rng(80)
    c = p - p.mean(0)
    mu = (c / np.linalg.norm(c, axis=1, keepdims=True) * (4.0 / len(p))).astype(np.float32)
    s = (rng.normal(size=(len(p), 3)) * 1e-3).astype(np.float32)
    out = wn.forward_A2(torch.from_numpy(mu).cuda(), W).cpu().numpy()
    want = np.concatenate([ref.forward(op, tr, p, mu, w) for op in ("A21", "A22", "A23")], 1)
    l2, mx = rel_errors(out, want)
    assert l2 <= 2e-5 and mx <= 2e-4, (l2, mx)
    out = wn.forward_A2T_sum(torch.from_numpy(s).cuda(), W).cpu().numpy()
    want = sum(ref.forward(op, tr, p, np.ascontiguousarray(s[:, k:k + 1]), w)
               for k, op in enumerate(("A2T1", "A2T2", "A2T3")))
    l2, mx = rel_errors(out, want)
    assert l2 <= 2e-5 and mx <= 2e-4, (l2, mx)
    # the solve at the configuration's widths as written (scale 1: 1.5 x mean
    # 10-NN).  The reference algorithm itself orients this cloud only partly
    # there (pairs within ~10 neighbours are dropped by the discontinuous
    # kernel), so the check is agreement with the host reference's own solve
    res1 = cagr_solve(P, 1.0, 1.0, widths=W, tree=wn)
    host1 = host_solve(p, 1.0, 1.0, impl=ref, base_widths=w, max_depth=8, leaf_size=16)
    mu1 = res1.normals.cpu().numpy()
    agree1 = sign_agreement(mu1, host1)
    print(f"sphere 5k at 1.5 x mean 10-NN: agreement with the host reference {agree1:.4f}, "
          f"outward: ours {sign_agreement(mu1, p):.4f}, reference {sign_agreement(host1, p):.4f}")
    assert agree1 >= 0.995, agree1
    # and at the widths scaled by 1/4, where the algorithm orients it fully
    res = cagr_solve(P, 0.25, 0.25, widths=W, tree=wn)
    host = host_solve(p, 0.25, 0.25, impl=ref, base_widths=w, max_depth=8, leaf_size=16)
    mu_gpu = res.normals.cpu().numpy()
    assert sign_agreement(mu_gpu, host) >= 0.995
    outward = sign_agreement(mu_gpu, p)
    assert outward >= 0.995, outward
    rec = reconstruct(P, res.normals, grid=128, tree=wn)
    v = rec.vertices.cpu().numpy()
    f = rec.faces.cpu().numpy()
    r = np.linalg.norm(v, axis=1)
    assert abs(np.median(r) - np.median(np.linalg.norm(p, axis=1))) < 0.03   # ~1.5 cells
    a, b, c3 = (v[f[:, k]].astype(np.float64) for k in range(3))
    assert np.einsum("ij,ij->i", a, np.cross(b, c3)).sum() / 6 > 0


def _torus_normals(raw, R=1.0):
    phi = np.arctan2(raw[:, 1], raw[:, 0])
    core = np.stack([R * np.cos(phi), R * np.sin(phi), np.zeros_like(phi)], 1)
    n = raw - core
    return n / np.linalg.norm(n, axis=1, keepdims=True)


def test_torus_100k_field_error_against_the_fp64_direct_sum(cuda_lib, oracle):
    import torch
    from cagr_b200 import WindingNumberTreecode
    from cagr_b200 import synthetic as S
    from cagr_b200.mesh import field_grid
    raw = S.make("torus")
    p64 = S.normalize(raw)
    scale = np.linalg.norm(p64[1] - p64[0]) / np.linalg.norm(raw[1] - raw[0])
    area = 4 * np.pi ** 2 * 1.0 * 0.3 * scale ** 2
    mu64 = _torus_normals(raw) * (area / len(raw))
    p, mu = p64.astype(np.float32), mu64.astype(np.float32)
    rng = np.random.default_rng(81)
    q = rng.uniform(-1.5, 1.5, size=(20000, 3)).astype(np.float32)
    width = 0.01
    wq = np.full(len(q), width, np.float32)
    wn = WindingNumberTreecode(torch.from_numpy(p).cuda(), leaf_size=32)
    wn.scatter(torch.from_numpy(mu).cuda())
    tr32 = oracle.build_tree(p, leaf_size=32)
    tr64 = oracle.build_tree(p.astype(np.float64), leaf_size=32)
    p_, mu_, wq_, q_ = (x.astype(np.float64) for x in (p, mu, wq, q))
    for op, cont in (("A", False), ("A3", True)):
        gpu = wn.multiply(op, width, queries=torch.from_numpy(q).cuda(),
                          continuous=cont).cpu().numpy()[:, 0]
        # the same algorithm and decisions (FP32 oracle): rounding only
        tree32 = oracle.forward(op, tr32, p, mu, wq, queries=q, continuous=cont)[:, 0]
        l2, mx = rel_errors(gpu, tree32)
        assert l2 <= 2e-5 and mx <= 2e-4, (op, l2, mx)
        # against the FP64 direct sum: the reference algorithm's own error, not more
        tree64 = oracle.forward(op, tr64, p_, mu_, wq_, queries=q_, continuous=cont)[:, 0]
        direct = oracle.direct(op, q_, wq_, p_, mu_, continuous=cont)[:, 0]
        e_gpu, e_ref = np.abs(gpu - direct).max(), np.abs(tree64 - direct).max()
        assert e_gpu <= 1.1 * e_ref + 1e-4, (op, e_gpu, e_ref)
    field = field_grid(wn, (256, 256, 256), (-1.2, -1.2, -1.2), 2.4 / 255, width, op="A3")
    assert torch.isfinite(field).all()


def test_blobs_4m_pipeline_and_fp32_field_against_fp64(cuda_lib):
    import torch
    from cagr_b200 import WindingNumberTreecode
    from cagr_b200 import synthetic as S
    from cagr_b200.mesh import field_grid, reconstruct
    from cagr_b200.solver import PRESET_WIDTHS, cagr_solve
    p = S.normalize(S.make("blobs")).astype(np.float32)
    P = torch.from_numpy(p).cuda()
    wn = WindingNumberTreecode(P)
    res = cagr_solve(P, *PRESET_WIDTHS["l0"], tree=wn)
    assert torch.isfinite(res.normals).all()
    rec = reconstruct(P, res.normals, grid=512, tree=wn)
    assert rec.faces.shape[0] > 100_000
    # the 512^3 field at 20,000 seeded grid nodes against the reference's own
    # kernels (host build) with the same normals: grid node (i, j, k) at
    # origin + (i, j, k) * spacing rounded once to float32, as the GPU forms it
    from oracle.oracle import RefOracle
    ref = RefOracle()
    mu = res.normals.cpu().numpy()
    G = 512
    h, o = np.float32(2.4 / 511), np.float32(-1.2)
    idx = np.random.default_rng(90).integers(0, G, size=(20000, 3))
    q = (idx.astype(np.float64) * np.float64(h) + np.float64(o)).astype(np.float32)
    tr = ref.build_tree(p)
    want = -ref.forward("A3", tr, p, mu, np.full(len(q), 0.01, np.float32), queries=q,
                        continuous=True)[:, 0]
    got = rec.field.cpu().numpy()[idx[:, 2], idx[:, 1], idx[:, 0]]
    l2, _ = rel_errors(got, want)
    # pairs lying exactly on the kernel's steps (the width test r >= w, whose
    # branches differ, and the acceptance test) may be decided differently by
    # two float32 builds with different libm rounding: a few nodes at most
    frac = float((np.abs(got - want) > 1e-4).mean())
    assert l2 <= 2e-5, l2
    assert frac <= 1e-3, frac
    # and the FP64 form of the same field (the plain FP64 pipeline) at the same nodes
    wn64 = WindingNumberTreecode(P.double())
    wn64.scatter(res.normals.double())
    f64 = field_grid(wn64, (G, G, G), (-1.2, -1.2, -1.2), 2.4 / 511, 0.01).neg_()
    got64 = f64.cpu().numpy()[idx[:, 2], idx[:, 1], idx[:, 0]]
    assert float((np.abs(got - got64) > 1e-4).mean()) <= 1e-3
