"""GPU: failure reporting and properties of the operators.

* Allocation failures (injected on the host with
  cagr_debug_fail_allocations_after: the n+1-th library allocation and every
  later one fail): at every point of a build / forward / adjoint / three-slot
  / autograd / marching-cubes sequence the failure surfaces as CAGR_ERR_ALLOC
  in a CagrError, nothing stays in use in the memory pool, and the library
  works (with identical results) afterwards.  No GPU fault is involved: the
  allocator refuses before anything is launched on the memory.
* Permuting the input points permutes the outputs (the tree, hence the pair
  terms, is the same up to the order of equal keys; sums differ by rounding).
* With max_tree_depth 0 the root is the only (leaf) node and every pair is
  summed directly: the treecode is the FP64 direct sum.
"""
import numpy as np
import pytest

from tests._cases import rel_errors, smooth_normals, sphere_cloud

pytestmark = pytest.mark.gpu


def _sequence(P, MU, S, W):
    """One pass of the library's allocating entry points; returns its outputs."""
    import torch
    from cagr_b200 import WindingNumberTreecode
    from cagr_b200.autograd import convection_gauss
    from cagr_b200.mesh import field_grid, marching_cubes
    wn = WindingNumberTreecode(P)
    try:
        a2 = wn.forward_A2(MU, W)
        at = wn.forward_A2T_sum(S, W)
        wn.scatter(MU)
        adj = wn.adjoint_A2(torch.ones_like(MU), W)
        mu = MU.clone().requires_grad_(True)
        (convection_gauss(wn, mu, W).sum()).backward()
        wn.scatter(MU)
        field = field_grid(wn, (40, 40, 40), (-1.1, -1.1, -1.1), 2.2 / 39, 0.02)
        v, f = marching_cubes(field.float(), (-1.1, -1.1, -1.1), 2.2 / 39,
                              float(field.median()))
        return [a2, at, adj, mu.grad, field, v, f]
    finally:
        wn.close()


def test_allocation_failures_are_reported_and_leak_nothing(cuda_lib):
    import torch
    from cagr_b200 import _lib
    from cagr_b200._lib import CagrError
    from cagr_b200.wn_treecode import pool_reserved
    pts = sphere_cloud(4000, seed=100)
    P = torch.from_numpy(pts).cuda()
    MU = torch.from_numpy(smooth_normals(pts, seed=101)).cuda()
    S = torch.from_numpy(np.random.default_rng(102).normal(size=(len(pts), 3)).astype(np.float32) * 1e-3).cuda()
    W = 0.02
    L = _lib.lib()
    ref = _sequence(P, MU, S, W)
    torch.cuda.synchronize()
    assert pool_reserved()[1] == 0
    failed = 0
    for n in range(0, 60):
        L.cagr_debug_fail_allocations_after(n)
        try:
            _sequence(P, MU, S, W)
        except CagrError as e:
            failed += 1
            assert "allocation" in str(e), str(e)
        finally:
            L.cagr_debug_fail_allocations_after(-1)
        torch.cuda.synchronize()
        assert pool_reserved()[1] == 0, n        # nothing left allocated
    assert failed > 10                            # the sweep reached many allocation sites
    again = _sequence(P, MU, S, W)
    for i, (a, b) in enumerate(zip(ref, again)):
        if i in (2, 3):   # the adjoint's atomic sums: order, hence rounding, varies
            assert torch.allclose(a, b, rtol=1e-5, atol=1e-6 * b.abs().max().item())
        else:
            assert torch.equal(a, b)


def test_permuting_the_points_permutes_the_outputs(cuda_lib):
    import torch
    from cagr_b200 import WindingNumberTreecode
    pts = sphere_cloud(5000, seed=103)
    mu = smooth_normals(pts, seed=104)
    s = np.random.default_rng(105).normal(size=(len(pts), 3)).astype(np.float32) * 1e-3
    perm = np.random.default_rng(106).permutation(len(pts))
    outs = []
    for idx in (np.arange(len(pts)), perm):
        wn = WindingNumberTreecode(torch.from_numpy(pts[idx]).cuda())
        a2 = wn.forward_A2(torch.from_numpy(mu[idx]).cuda(), 0.01).cpu().numpy()
        at = wn.forward_A2T_sum(torch.from_numpy(s[idx]).cuda(), 0.01).cpu().numpy()
        outs.append((a2, at))
    inv = np.argsort(perm)
    for k in range(2):
        l2, mx = rel_errors(outs[1][k][inv], outs[0][k])
        assert l2 <= 2e-5 and mx <= 2e-4, (k, l2, mx)


@pytest.mark.parametrize("op", ["A", "A3", "A21", "AT", "A2T2", "G"])
def test_depth_zero_tree_is_the_direct_sum(cuda_lib, oracle, op):
    import torch
    from cagr_b200 import WindingNumberTreecode
    from cagr_b200._lib import ATTR_DIM
    pts = sphere_cloud(1500, seed=107)
    rng = np.random.default_rng(108)
    vals = (smooth_normals(pts, seed=109) if ATTR_DIM[op] == 3
            else rng.normal(size=(len(pts), 1)).astype(np.float32) * 1e-3)
    w = np.full(len(pts), 0.02, np.float32)
    wn = WindingNumberTreecode(torch.from_numpy(pts).cuda(), max_tree_depth=0)
    assert wn.num_nodes == 1
    wn.scatter(torch.from_numpy(vals).cuda())
    got = wn.multiply(op, torch.from_numpy(w).cuda()).cpu().numpy()
    want = oracle.direct(op, pts.astype(np.float64), w.astype(np.float64),
                         pts.astype(np.float64), vals.astype(np.float64))
    l2, mx = rel_errors(got, want)
    assert l2 <= 2e-5 and mx <= 2e-4, (l2, mx)
