"""GPU: the device-resident CAGR solve against the reference.

Parity for the solve is normal-sign agreement (the iteration amplifies
rounding differences; the FP64 Krylov scalars differ from the reference's
FP32 ones by design):
  * against the reference's published bunny output (CUDA-based/results/
    bunny.xyz) with a stable schedule (10 steepest-descent steps, preset l0);
  * against the reference algorithm run with the reference's own kernels on
    the host (tests/golden/bunny_solve.npz), full 40-iteration schedule, l1.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _bunny():
    import torch
    from cagr_b200.solver import normalize_points
    g = np.load(os.path.join(GOLDEN, "bunny.npz"))
    return g, torch.from_numpy(normalize_points(g["points"])).cuda()


def _agree(a, b):
    return float(((a * b).sum(1) > 0).mean())


def test_bunny_published_output_signs(cuda_lib):
    from cagr_b200.solver import PRESET_WIDTHS, cagr_solve
    g, pts = _bunny()
    res = cagr_solve(pts, *PRESET_WIDTHS["l0"], iters=10)
    mu = res.normals.cpu().numpy()
    assert _agree(mu, g["mu_reference"]) >= 0.995


def test_bunny_reference_algorithm_full_schedule(cuda_lib):
    from cagr_b200.solver import PRESET_WIDTHS, cagr_solve
    g, pts = _bunny()
    s = np.load(os.path.join(GOLDEN, "bunny_solve.npz"))
    res = cagr_solve(pts, *PRESET_WIDTHS["l1"])
    mu = res.normals.cpu().numpy()
    assert np.isfinite(mu).all()
    assert _agree(mu, s["mu_l1_40"]) >= 0.995
    rel = np.linalg.norm(mu - s["mu_l1_40"], axis=1) / np.linalg.norm(s["mu_l1_40"], axis=1)
    assert np.median(rel) < 0.05
    assert res.operator_calls == 3 + 31 * 12 + 9 + 9 * 6 + 8


def test_solve_accepts_per_point_widths(cuda_lib):
    import torch
    from cagr_b200.solver import cagr_solve
    _, pts = _bunny()
    a = cagr_solve(pts, 0.01, 0.04, iters=4)
    b = cagr_solve(pts, 0.01, 0.04, iters=4, widths=torch.ones(pts.shape[0], device="cuda"))
    assert torch.equal(a.normals, b.normals)


def test_float64_solve_reproduces_the_published_signs(cuda_lib):
    """The same solve in float64 (points, widths, moments and sums): the
    published output's signs as in float32."""
    import torch
    from cagr_b200.solver import PRESET_WIDTHS, cagr_solve
    g, pts = _bunny()
    res = cagr_solve(pts.double(), *PRESET_WIDTHS["l0"], iters=10)
    assert res.normals.dtype == torch.float64
    mu = res.normals.cpu().numpy()
    assert np.isfinite(mu).all()
    assert _agree(mu, g["mu_reference"]) >= 0.995


def test_width_table_and_its_fallback_give_the_same_solve(cuda_lib, monkeypatch):
    """b's window table (one walk for all steepest-descent widths) and the
    fallback for schedules with more widths than the table takes (each step's
    four-slot walk adds b's window itself) sum the same terms: the same solve
    up to rounding."""
    from cagr_b200 import solver
    _, pts = _bunny()
    a = solver.cagr_solve(pts, 0.01, 0.04, iters=8, n_sd=5, wnnc_steps=0)
    monkeypatch.setattr(solver, "MAX_TABLE_WIDTHS", 0)
    b = solver.cagr_solve(pts, 0.01, 0.04, iters=8, n_sd=5, wnnc_steps=0)
    mu_a, mu_b = a.normals.cpu().numpy(), b.normals.cpu().numpy()
    assert a.operator_calls == b.operator_calls
    assert _agree(mu_a, mu_b) >= 0.999
    assert np.linalg.norm(mu_a - mu_b) <= 1e-3 * np.linalg.norm(mu_a)


def test_window_table_alloc_failure_falls_back(cuda_lib, monkeypatch):
    """When the device has no room for b's window table (its allocation fails
    with CAGR_ERR_ALLOC), the solve uses the table-free per-step walk and
    gives the same result as the fallback chosen up front."""
    from cagr_b200 import _lib, solver
    from cagr_b200.wn_treecode import WindingNumberTreecode
    _, pts = _bunny()
    real = WindingNumberTreecode.b_window_table

    def no_room(self, base, scales):
        raise _lib.CagrError("cagr_b_window_table: device allocation failed", _lib.CAGR_ERR_ALLOC)

    monkeypatch.setattr(WindingNumberTreecode, "b_window_table", no_room)
    a = solver.cagr_solve(pts, 0.01, 0.04, iters=8, n_sd=5, wnnc_steps=0)
    monkeypatch.setattr(WindingNumberTreecode, "b_window_table", real)
    monkeypatch.setattr(solver, "MAX_TABLE_WIDTHS", 0)
    b = solver.cagr_solve(pts, 0.01, 0.04, iters=8, n_sd=5, wnnc_steps=0)
    assert a.operator_calls == b.operator_calls
    assert np.array_equal(a.normals.cpu().numpy(), b.normals.cpu().numpy())

    def broken(self, base, scales):
        raise _lib.CagrError("cagr_b_window_table: invalid", 1)

    monkeypatch.setattr(WindingNumberTreecode, "b_window_table", broken)
    monkeypatch.setattr(solver, "MAX_TABLE_WIDTHS", 64)
    with pytest.raises(_lib.CagrError):
        solver.cagr_solve(pts, 0.01, 0.04, iters=8, n_sd=5, wnnc_steps=0)
