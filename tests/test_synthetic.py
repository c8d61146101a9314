"""CPU: the seeded synthetic workloads."""
import numpy as np
import pytest

from cagr_b200 import synthetic as S


@pytest.mark.parametrize("name", S.WORKLOADS)
def test_generators_are_seeded_and_shaped(name):
    a = S.make(name, 2000)
    b = S.make(name, 2000)
    assert a.shape == (2000, 3)
    assert np.array_equal(a, b)
    assert np.isfinite(a).all()


def test_normalize_matches_main_cagr():
    p = np.random.default_rng(0).normal(size=(500, 3)) * 7 + 3
    q = S.normalize(p)
    lo, hi = q.min(0), q.max(0)
    assert np.isclose((hi - lo).max(), 2 / 1.1)
    assert np.allclose((hi + lo) / 2, 0, atol=1e-12)


def test_sphere_is_on_the_unit_sphere():
    p = S.sphere(5000)
    r = np.linalg.norm(p, axis=1)
    assert abs(r.mean() - 1) < 1e-3 and r.std() < 3e-3


def test_torus_density_follows_the_tube_angle():
    p = S.torus(50_000)
    rho = np.hypot(p[:, 0], p[:, 1])
    outer = (rho > 1.0).mean()   # cos(phi) > 0 half of the tube
    assert outer > 0.6           # density 1 + 0.8 cos(phi) weights the outer half


def test_blobs_lie_on_the_level_set():
    p = S.blobs(3000)
    assert p.shape == (3000, 3)
