"""GPU parity: the CUDA path through the C ABI against the CPU oracle.

Integer/index work (the octree) must be bit-exact; node moments are computed
in the reference's operation order and must be bit-exact too; operator
values are floating point and must agree within the stated tolerances
(FP32: relative L2 <= 2e-5 and max error <= 2e-4 of max |ref|, set by
rsqrt/exp rounding and a different summation order over identical pair
sets; FP64: 1e-12 / 1e-11).
"""
import numpy as np
import pytest

from tests._cases import edge_cloud, random_values, rel_errors, smooth_normals, sphere_cloud

pytestmark = pytest.mark.gpu

TOL = {np.float32: (2e-5, 2e-4), np.float64: (1e-12, 1e-11)}
VALUE_OPS = ["AT", "A2T1", "A2T2", "A2T3"]
NORMAL_OPS = ["A", "A3", "A21", "A22", "A23", "G"]


def _torch():
    import torch
    return torch


def _tree(points, max_depth=15, leaf_size=1):
    torch = _torch()
    from cagr_b200 import WindingNumberTreecode
    return WindingNumberTreecode(torch.from_numpy(points).cuda(), max_tree_depth=max_depth,
                                 leaf_size=leaf_size)


TREE_CASES = [
    ("sphere3000", lambda: sphere_cloud(3000), 15, 1),
    ("edge", lambda: edge_cloud(), 15, 1),
    ("sphere_f64", lambda: sphere_cloud(2500, seed=5, dtype=np.float64), 15, 1),
    ("leaf16_depth8", lambda: sphere_cloud(5000, seed=6), 8, 16),
    ("leaf4_depth6_edge", lambda: edge_cloud(seed=7), 6, 4),
    ("depth0", lambda: sphere_cloud(50, seed=8), 0, 1),
    ("one_point", lambda: sphere_cloud(1, seed=9), 15, 1),
    ("all_duplicates", lambda: np.repeat(sphere_cloud(3, seed=10), 40, axis=0), 15, 1),
    ("depth21", lambda: edge_cloud(seed=11), 21, 1),
]


@pytest.mark.parametrize("name,make,max_depth,leaf_size", TREE_CASES, ids=[c[0] for c in TREE_CASES])
def test_tree_bit_exact(cuda_lib, oracle, name, make, max_depth, leaf_size):
    pts = make()
    tr = oracle.build_tree(pts, max_depth=max_depth, leaf_size=leaf_size)
    wn = _tree(pts, max_depth, leaf_size)
    got = [t.cpu().numpy() for t in (wn.node_parent_list, wn.node_children_list,
                                     wn.node_is_leaf_list, wn.node_half_w_list,
                                     wn.num_points_in_node, wn.node2point_index,
                                     wn.node2point_indexstart)]
    names = ["parent", "children", "is_leaf", "half_w", "npts", "n2p", "n2p_start"]
    for g, r, nm in zip(got, tr.as_tuple(), names):
        assert g.shape == r.shape, (nm, g.shape, r.shape)
        assert g.dtype == r.dtype, (nm, g.dtype, r.dtype)
        assert np.array_equal(g, r), nm
    assert wn.depth == tr.depth
    assert wn.num_leaves == tr.num_leaves


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("dim", [3, 1])
def test_moments_bit_exact(cuda_lib, oracle, dtype, dim):
    torch = _torch()
    from oracle.oracle import point_weights
    pts = edge_cloud(dtype=dtype)
    wn = _tree(pts)
    tr = oracle.build_tree(pts)
    vals = smooth_normals(pts, zero_frac=0.2) if dim == 3 else random_values(len(pts), 1, dtype=dtype)
    if dim == 1:
        vals[::7] = 0
    mom = oracle.moments(tr, pts, point_weights(vals), vals)
    wn.scatter(torch.from_numpy(vals).cuda())
    a, r, w = (t.cpu().numpy() for t in wn.scatter_export(0, dim))
    assert np.array_equal(w, mom.weights)
    assert np.array_equal(r, mom.rep)
    assert np.array_equal(a, mom.attrs)


def _ref_op(oracle, op, pts, vals, widths, queries=None, cont=False):
    tr = oracle.build_tree(pts)
    return oracle.forward(op, tr, pts, vals, widths, queries=queries, continuous=cont)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("op", NORMAL_OPS + VALUE_OPS)
def test_operator_parity(cuda_lib, oracle, op, dtype):
    torch = _torch()
    pts = sphere_cloud(4000, seed=12, dtype=dtype)
    rng = np.random.default_rng(13)
    widths = rng.uniform(0.005, 0.03, size=len(pts)).astype(dtype)
    if op in VALUE_OPS:
        vals = random_values(len(pts), 1, seed=14, dtype=dtype)
    else:
        vals = smooth_normals(pts, seed=15)
    ref = _ref_op(oracle, op, pts, vals, widths)
    wn = _tree(pts)
    fn = getattr(wn, f"forward_{op}")
    got = fn(torch.from_numpy(vals).cuda(), torch.from_numpy(widths).cuda()).cpu().numpy()
    assert got.shape == ref.shape
    l2, mx = rel_errors(got, ref)
    tl2, tmx = TOL[dtype]
    assert l2 <= tl2 and mx <= tmx, (op, l2, mx)


@pytest.mark.parametrize("op", ["A", "A3", "A21", "A22", "A23"])
def test_continuous_kernel_at_queries(cuda_lib, oracle, op):
    """Continuous kernel at external query points (the GaussRecon field
    evaluation shape: grid corners + the samples themselves)."""
    torch = _torch()
    pts = sphere_cloud(3000, seed=16)
    vals = smooth_normals(pts, seed=17)
    rng = np.random.default_rng(18)
    q = np.concatenate([rng.uniform(-1.0, 1.0, size=(3000, 3)), pts[:500]]).astype(np.float32)
    w = np.full(len(q), 0.02, np.float32)
    ref = _ref_op(oracle, op, pts, vals, w, queries=q, cont=True)
    wn = _tree(pts)
    wn.scatter(torch.from_numpy(vals).cuda())
    got = wn.multiply(op, torch.from_numpy(w).cuda(), queries=torch.from_numpy(q).cuda(),
                      continuous=True).cpu().numpy()
    l2, mx = rel_errors(got, ref)
    assert l2 <= 2e-5 and mx <= 2e-4, (op, l2, mx)


def test_fused_forward_matches_single_direction(cuda_lib):
    torch = _torch()
    pts = sphere_cloud(5000, seed=19)
    vals = torch.from_numpy(smooth_normals(pts, seed=20)).cuda()
    wn = _tree(pts)
    fused = wn.forward_A2(vals, 0.01)
    for k, op in enumerate(("A21", "A22", "A23")):
        single = getattr(wn, f"forward_{op}")(vals, 0.01)
        assert torch.equal(fused[:, k:k + 1], single), op


def test_scalar_width_equals_width_tensor(cuda_lib):
    torch = _torch()
    pts = sphere_cloud(3000, seed=21)
    vals = torch.from_numpy(smooth_normals(pts, seed=22)).cuda()
    wn = _tree(pts)
    a = wn.forward_A21(vals, 0.015)
    b = wn.forward_A21(vals, torch.full((len(pts),), 0.015, device="cuda"))
    assert torch.equal(a, b)


def test_a2t_sum_matches_reference_composition(cuda_lib, oracle):
    torch = _torch()
    pts = sphere_cloud(3000, seed=23)
    s = random_values(len(pts), 3, seed=24)
    w = np.full(len(pts), 0.01, np.float32)
    tr = oracle.build_tree(pts)
    ref = sum(oracle.forward(op, tr, pts, s[:, k:k + 1], w)
              for k, op in enumerate(("A2T1", "A2T2", "A2T3")))
    wn = _tree(pts)
    got = wn.forward_A2T_sum(torch.from_numpy(s).cuda(), 0.01).cpu().numpy()
    l2, mx = rel_errors(got, ref)
    assert l2 <= 2e-5 and mx <= 2e-4, (l2, mx)


def test_a2t_shared_matches_reference_composition(cuda_lib, oracle):
    """A2T1(b) + A2T2(b) + A2T3(b) with one input (the solve's right-hand side)."""
    torch = _torch()
    pts = sphere_cloud(3000, seed=25)
    b = random_values(len(pts), 1, seed=26)
    w = np.full(len(pts), 0.01, np.float32)
    tr = oracle.build_tree(pts)
    ref = sum(oracle.forward(op, tr, pts, b, w) for op in ("A2T1", "A2T2", "A2T3"))
    wn = _tree(pts)
    got = wn.forward_A2T_shared(torch.from_numpy(b).cuda(), 0.01).cpu().numpy()
    l2, mx = rel_errors(got, ref)
    assert l2 <= 2e-5 and mx <= 2e-4, (l2, mx)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_three_slot_moments_bit_exact(cuda_lib, oracle, dtype):
    torch = _torch()
    from oracle.oracle import point_weights
    pts = edge_cloud(dtype=dtype)
    wn = _tree(pts)
    tr = oracle.build_tree(pts)
    s = random_values(len(pts), 3, seed=27, dtype=dtype)
    s[::5, 1] = 0
    wn.scatter3(torch.from_numpy(s).cuda())
    for k in range(3):
        col = np.ascontiguousarray(s[:, k:k + 1])
        mom = oracle.moments(tr, pts, point_weights(col), col)
        a, r, w = (t.cpu().numpy() for t in wn.scatter_export(k, 1))
        assert np.array_equal(w, mom.weights) and np.array_equal(r, mom.rep)
        assert np.array_equal(a, mom.attrs)


def test_pair_term_counts_match_oracle(cuda_lib, oracle):
    """COUNT reproduces the reference traversal's term count per query."""
    torch = _torch()
    from oracle.oracle import point_weights
    pts = sphere_cloud(4000, seed=28)
    mu = smooth_normals(pts, seed=29)
    w = np.full(len(pts), 0.01, np.float32)
    tr = oracle.build_tree(pts)
    mom = oracle.moments(tr, pts, point_weights(mu), mu)
    _, terms, _ = oracle.multiply("A21", pts, w, pts, mu, tr, mom, counts=True)
    wn = _tree(pts)
    wn.scatter(torch.from_numpy(mu).cuda())
    got = wn.multiply("COUNT", 0.01).cpu().numpy()[:, 0]
    assert np.array_equal(got.astype(np.int64), terms)


def test_errors_are_raised(cuda_lib):
    torch = _torch()
    from cagr_b200 import WindingNumberTreecode
    from cagr_b200._lib import CagrError
    with pytest.raises(RuntimeError):
        WindingNumberTreecode(torch.zeros(10, 3))  # CPU tensor: no CPU path
    with pytest.raises(CagrError):
        WindingNumberTreecode(torch.zeros(10, 3, device="cuda"), max_tree_depth=40)
    wn = _tree(sphere_cloud(100))
    with pytest.raises(CagrError):
        wn.multiply("A21", 0.01)  # no moments computed yet
    with pytest.raises(AssertionError):
        wn.forward_A21(torch.zeros(99, 3, device="cuda"), 0.01)


def test_memory_pool_reuses_freed_trees(cuda_lib):
    """Trees and records come from the library's pool: a destroyed tree's memory
    stays reserved and serves the next tree of the same size, with nothing in
    use afterwards; trimming returns it to the CUDA driver."""
    torch = _torch()
    from cagr_b200 import WindingNumberTreecode
    from cagr_b200.wn_treecode import pool_reserved, pool_trim
    cloud = sphere_cloud(20000, seed=60)
    pts = torch.from_numpy(cloud).cuda()
    mu = torch.from_numpy(smooth_normals(cloud, seed=61)).cuda()
    for _ in range(2):
        wn = WindingNumberTreecode(pts)
        wn.forward_A2(mu, 0.01)
        wn.close()
    reserved, used = pool_reserved()
    assert used == 0 and reserved > 0
    wn = WindingNumberTreecode(pts)
    wn.forward_A2(mu, 0.01)
    wn.close()
    assert pool_reserved() == (reserved, 0)
    pool_trim(0)
    assert pool_reserved()[0] < reserved


def test_three_slot_scatter_and_slots_are_independent(cuda_lib, oracle):
    """scatter3 fills the packed adjoint records only: the record slots keep the
    last single-slot scatter (single-slot operators are unaffected), and a
    later single-slot scatter leaves the adjoint records (and the export of
    the other columns) intact."""
    torch = _torch()
    from oracle.oracle import point_weights
    pts = sphere_cloud(3000, seed=62)
    s = random_values(len(pts), 3, seed=63)
    b = random_values(len(pts), 1, seed=64)
    wn = _tree(pts)
    tr = oracle.build_tree(pts)
    S = torch.from_numpy(s).cuda()
    wn.scatter(torch.from_numpy(b).cuda())           # slot 0 holds b
    before = wn.multiply("A2T1", 0.01).clone()
    wn.scatter3(S)
    assert torch.equal(wn.multiply("A2T1", 0.01), before)   # slot 0 untouched
    first = wn.multiply("A2T_SUM", 0.01).clone()
    wn.scatter(torch.from_numpy(b).cuda())           # slot 0 = b again
    assert torch.equal(wn.multiply("A2T_SUM", 0.01), first)
    a0, _, _ = (t.cpu().numpy() for t in wn.scatter_export(0, 1))
    assert np.array_equal(a0, oracle.moments(tr, pts, point_weights(b), b).attrs)
    col = np.ascontiguousarray(s[:, 1:2])
    a1, r1, w1 = (t.cpu().numpy() for t in wn.scatter_export(1, 1))
    mom = oracle.moments(tr, pts, point_weights(col), col)
    assert np.array_equal(a1, mom.attrs) and np.array_equal(r1, mom.rep)
    assert np.array_equal(w1, mom.weights)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_a2t_rhs_equals_the_separate_calls(cuda_lib, dtype):
    """sum_k A2Tk(b) - sum_k A2Tk(s_k) in one walk (b in slot 1, each input with
    its own moments and decisions) equals the two reference-style calls."""
    torch = _torch()
    pts = sphere_cloud(3000, seed=90, dtype=dtype)
    s = torch.from_numpy(random_values(len(pts), 3, seed=91, dtype=dtype)).cuda()
    b = torch.from_numpy(random_values(len(pts), 1, seed=92, dtype=dtype)).cuda()
    w = torch.from_numpy(np.full(len(pts), 0.01, dtype)).cuda()
    wn = _tree(pts)
    sep = (wn.forward_A2T_shared(b, w) - wn.forward_A2T_sum(s, w)).cpu().numpy()
    wn.scatter(b, slot=1)
    fused = wn.forward_A2T_rhs(s, w).cpu().numpy()
    l2, mx = rel_errors(fused, sep)
    tl2, tmx = TOL[dtype]
    assert l2 <= tl2 and mx <= tmx, (l2, mx)


@pytest.mark.parametrize("leaf_size", [1, 8])
def test_query_grouping_changes_no_bit(cuda_lib, leaf_size):
    """Each query's pair terms and their order are its own, whatever other
    queries share its warp: the tree's points as self-queries (grouped along a
    Hilbert curve) and the same points as explicit queries in their original,
    random order give the same bits, for every walk."""
    torch = _torch()
    pts = sphere_cloud(20000, seed=95)
    P = torch.from_numpy(pts).cuda()
    mu = torch.from_numpy(smooth_normals(pts, seed=96)).cuda()
    s = torch.from_numpy(random_values(len(pts), 3, seed=97)).cuda() * 1e-3
    b = torch.from_numpy(random_values(len(pts), 1, seed=98)).cuda()
    w = torch.from_numpy(np.random.default_rng(99).uniform(0.005, 0.02, len(pts))
                         .astype(np.float32)).cuda()
    wn = _tree(pts, leaf_size=leaf_size)
    pairs = []
    for op in ["A", "A3", "A2_FUSED", "G"]:
        wn.scatter(mu)
        pairs.append((op, wn.multiply(op, w), wn.multiply(op, w, queries=P)))
        if op == "A3":
            pairs.append(("A3 cont", wn.multiply(op, w, continuous=True),
                          wn.multiply(op, w, queries=P, continuous=True)))
    wn.scatter(b[:, 0:1] * 1e-3)
    pairs.append(("AT", wn.multiply("AT", w), wn.multiply("AT", w, queries=P)))
    pairs.append(("A2T_SUM_SHARED", wn.multiply("A2T_SUM_SHARED", w),
                  wn.multiply("A2T_SUM_SHARED", w, queries=P)))
    wn.scatter(b, slot=1)
    wn.scatter3(s)
    for op in ["A2T_SUM", "A2T_RHS"]:
        pairs.append((op, wn.multiply(op, w), wn.multiply(op, w, queries=P)))
    for op, a, c in pairs:
        assert torch.equal(a, c), op


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_a2t_rhs_window_equals_the_full_walk(cuda_lib, dtype):
    """b's terms split at the upper widths: sum_k A2Tk(b) at widths_hi plus the
    window walk (b's terms with t(w) <= r^2 < t(w_hi), minus the s_k terms)
    equals the full right-hand-side walk at w (same terms, other summation
    order), for widths below, equal to and well below widths_hi."""
    torch = _torch()
    pts = sphere_cloud(3000, seed=113, dtype=dtype)
    n = len(pts)
    rng = np.random.default_rng(114)
    s = torch.from_numpy(random_values(n, 3, seed=115, dtype=dtype)).cuda()
    b = torch.from_numpy(random_values(n, 1, seed=116, dtype=dtype)).cuda()
    base = torch.from_numpy(rng.uniform(0.5, 1.5, n).astype(dtype)).cuda()
    wn = _tree(pts)
    wn.scatter(b, slot=1)
    tl2, tmx = TOL[dtype]
    for lo, hi in [(0.01, 0.04), (0.04, 0.04), (0.004, 0.06)]:
        w, w_hi = base * lo, base * hi
        full = wn.forward_A2T_rhs(s, w).cpu().numpy()
        b_hi = wn.forward_A2T_shared(b, w_hi)
        win = wn.forward_A2T_rhs_window(s, w, b_hi, w_hi).cpu().numpy()
        l2, mx = rel_errors(win, full)
        assert l2 <= tl2 and mx <= tmx, (lo, hi, l2, mx)


@pytest.mark.parametrize("cloud", ["sphere", "edge"])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_b_window_table_equals_the_walks_at_each_width(cuda_lib, dtype, cloud):
    """One walk for a schedule of widths: sum_k A2Tk(b) at base * scales[-1]
    plus row i of the table equals the walk at base * scales[i] (same terms,
    other summation order); the last row is empty."""
    torch = _torch()
    pts = (sphere_cloud(3000, seed=118, dtype=dtype) if cloud == "sphere"
           else edge_cloud(seed=122, dtype=dtype))
    n = len(pts)
    b = torch.from_numpy(random_values(n, 1, seed=119, dtype=dtype)).cuda()
    base = torch.from_numpy(np.random.default_rng(121).uniform(0.5, 1.5, n).astype(dtype)).cuda()
    scales = torch.tensor([0.002, 0.005, 0.011, 0.016, 0.04, 0.09], device="cuda",
                          dtype=base.dtype)
    wn = _tree(pts)
    wn.scatter(b, slot=1)
    table = wn.b_window_table(base, scales)
    assert table.shape == (len(scales), n, 3)
    assert torch.equal(table[-1], torch.zeros_like(table[-1]))
    b_hi = wn.forward_A2T_shared(b, base * scales[-1])
    tl2, tmx = TOL[dtype]
    for i in range(len(scales)):
        want = wn.forward_A2T_shared(b, base * scales[i]).cpu().numpy()
        got = (b_hi + table[i]).cpu().numpy()
        l2, mx = rel_errors(got, want)
        assert l2 <= tl2 and mx <= tmx, (i, l2, mx)
