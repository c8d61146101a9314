"""CPU: the oracle restatement pinned against the reference's own outputs.

The golden fixtures (tests/golden/*.npz) were produced by the reference's own
tree builder and kernels compiled for the host (tests/golden/make_golden.py).
The oracle must reproduce the tree and node moments exactly and the operator
values to rounding (it restates the same float operations in a different
arrangement).
"""
import glob
import os

import numpy as np
import pytest

from tests._cases import rel_errors, smooth_normals, sphere_cloud

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz"))
               if not os.path.basename(p).startswith(("bunny", "mc_")))
OPS = ["A", "AT", "A3", "A21", "A22", "A23", "A2T1", "A2T2", "A2T3", "G"]
TREE_KEYS = ["parent", "children", "is_leaf", "half_w", "npts", "n2p", "n2p_start"]


def load(name):
    return dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))


def test_fixtures_present():
    assert len(CASES) >= 4
    assert os.path.exists(os.path.join(GOLDEN, "bunny.npz"))


@pytest.mark.parametrize("case", CASES)
def test_tree_matches_reference(oracle, case):
    g = load(case)
    tr = oracle.build_tree(g["points"], int(g["max_depth"]), int(g["leaf_size"]))
    for key, arr in zip(TREE_KEYS, tr.as_tuple()):
        assert arr.dtype == g[key].dtype, key
        assert np.array_equal(arr, g[key]), key
    assert tr.depth == int(g["depth"])
    assert tr.num_leaves == int(g["num_leaves"])


@pytest.mark.parametrize("case", CASES)
def test_moments_match_reference(oracle, case):
    from oracle.oracle import point_weights
    g = load(case)
    pts = g["points"]
    tr = oracle.build_tree(pts, int(g["max_depth"]), int(g["leaf_size"]))
    for vals, tag in ((g["mu"], "mom3"), (g["s"], "mom1")):
        m = oracle.moments(tr, pts, point_weights(vals), vals)
        assert np.array_equal(m.attrs, g[f"{tag}_attrs"]), tag
        assert np.array_equal(m.rep, g[f"{tag}_rep"]), tag
        assert np.array_equal(m.weights, g[f"{tag}_w"]), tag


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("op", OPS)
def test_operators_match_reference(oracle, case, op):
    g = load(case)
    pts = g["points"]
    tol = (1e-6, 1e-5) if pts.dtype == np.float32 else (1e-13, 1e-12)
    tr = oracle.build_tree(pts, int(g["max_depth"]), int(g["leaf_size"]))
    vals = g["s"] if op in ("AT", "A2T1", "A2T2", "A2T3") else g["mu"]
    got = oracle.forward(op, tr, pts, vals, g["widths"])
    l2, mx = rel_errors(got, g[f"out_{op}"])
    assert l2 <= tol[0] and mx <= tol[1], (l2, mx)
    if f"out_{op}_cont" in g:
        got = oracle.forward(op, tr, pts, vals, g["widths"], continuous=True)
        l2, mx = rel_errors(got, g[f"out_{op}_cont"])
        assert l2 <= tol[0] and mx <= tol[1], ("cont", l2, mx)


@pytest.mark.parametrize("case", CASES)
def test_field_at_queries_matches_reference(oracle, case):
    g = load(case)
    pts = g["points"]
    tr = oracle.build_tree(pts, int(g["max_depth"]), int(g["leaf_size"]))
    got = oracle.forward("A3", tr, pts, g["mu"], g["qwidths"], queries=g["queries"],
                         continuous=True)
    l2, mx = rel_errors(got, g["out_A3_cont_queries"])
    tol = 1e-6 if pts.dtype == np.float32 else 1e-13
    assert l2 <= tol and mx <= 10 * tol


def test_reference_build_reproduces_fixtures():
    """When the reference host build is present, it regenerates the fixtures exactly."""
    from oracle.oracle import REF_LIB_PATH, RefOracle
    if not os.path.exists(REF_LIB_PATH):
        pytest.skip("oracle/_ref not built")
    ref = RefOracle()
    g = load("edge_f32")
    tr = ref.build_tree(g["points"], int(g["max_depth"]), int(g["leaf_size"]))
    for key, arr in zip(TREE_KEYS, tr.as_tuple()):
        assert np.array_equal(arr, g[key]), key
    out = ref.forward("A21", tr, g["points"], g["mu"], g["widths"])
    assert np.array_equal(out, g["out_A21"])


def test_single_leaf_tree_is_the_direct_sum(oracle):
    """max_depth 0 makes the root the only (leaf) node: every pair is summed
    directly, so the FP64 treecode equals the FP64 direct sum."""
    pts = sphere_cloud(400, seed=30, dtype=np.float64)
    mu = smooth_normals(pts, seed=31)
    w = np.full(len(pts), 0.02)
    tr = oracle.build_tree(pts, max_depth=0)
    assert tr.num_nodes == 1
    for op in ("A21", "A3", "G"):
        tree = oracle.forward(op, tr, pts, mu, w)
        direct = oracle.direct(op, pts, w, pts, mu)
        assert rel_errors(tree, direct)[0] < 1e-12, op


def test_treecode_error_against_direct_sum(oracle):
    """The reference acceptance rule (theta = 1/2, monopole) has a bounded
    error against the FP64 direct sum for smooth normals."""
    pts = sphere_cloud(3000, seed=32, dtype=np.float64)
    mu = smooth_normals(pts, seed=33)
    w = np.full(len(pts), 0.02)
    tr = oracle.build_tree(pts)
    tree = oracle.forward("A3", tr, pts, mu, w)
    direct = oracle.direct("A3", pts, w, pts, mu)
    l2, _ = rel_errors(tree, direct)
    assert l2 < 0.05


def test_positive_scaling_is_exact_up_to_rounding(oracle):
    """Scaling mu by c > 0 scales every node weight by c and leaves centroids
    (hence every acceptance decision) unchanged: the operator scales by c."""
    pts = sphere_cloud(2000, seed=34)
    mu = smooth_normals(pts, seed=35)
    w = np.full(len(pts), 0.02, np.float32)
    tr = oracle.build_tree(pts)
    a = oracle.forward("A21", tr, pts, mu, w)
    b = oracle.forward("A21", tr, pts, (mu * np.float32(4.0)), w)
    assert np.array_equal(b, a * np.float32(4.0))


def test_point_permutation_permutes_outputs(oracle):
    """Relabelling the points relabels the outputs (same cells, same pairs)."""
    pts = sphere_cloud(2000, seed=36, dtype=np.float64)
    mu = smooth_normals(pts, seed=37)
    w = np.full(len(pts), 0.02)
    perm = np.random.default_rng(38).permutation(len(pts))
    a = oracle.forward("A3", oracle.build_tree(pts), pts, mu, w)
    b = oracle.forward("A3", oracle.build_tree(pts[perm]), pts[perm], mu[perm], w)
    assert rel_errors(b, a[perm])[0] < 1e-12


def test_bunny_fixture_is_the_reference_output():
    g = np.load(os.path.join(GOLDEN, "bunny.npz"))
    assert g["points"].shape == (5000, 3) and g["mu_reference"].shape == (5000, 3)
    nrm = np.linalg.norm(g["mu_reference"], axis=1)
    assert nrm.min() > 0 and nrm.max() < 1e-3


def test_oracle_solve_reproduces_published_bunny_signs(oracle):
    """A stable schedule of the reference solve (10 steepest-descent steps at
    preset l0) orients every bunny normal as the reference's published output."""
    from oracle.solve import PRESET_WIDTHS, normalize, sign_agreement, solve
    g = np.load(os.path.join(GOLDEN, "bunny.npz"))
    mu = solve(normalize(g["points"]), *PRESET_WIDTHS["l0"], impl=oracle, iters=10)
    assert sign_agreement(mu, g["mu_reference"]) >= 0.995


def test_oracle_solve_matches_reference_kernels_solve(oracle):
    """The restated solve with the restated kernels against the fixture made
    with the reference's own kernels (l1, the full 40-iteration schedule)."""
    from oracle.solve import PRESET_WIDTHS, normalize, sign_agreement, solve
    g = np.load(os.path.join(GOLDEN, "bunny.npz"))
    s = np.load(os.path.join(GOLDEN, "bunny_solve.npz"))
    mu = solve(normalize(g["points"]), *PRESET_WIDTHS["l1"], impl=oracle)
    assert sign_agreement(mu, s["mu_l1_40"]) >= 0.995
