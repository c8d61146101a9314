"""GPU: the double-precision reciprocal square root of the FP64 traversals (the
hardware approximation rsqrt.approx.f64 refined by one third-order step)
against CUDA's rsqrt(double) (torch.rsqrt on the same device) and against
1/sqrt in numpy: within 2 ulp over 1e-300..1e300 and over the squared
distances the traversals meet (1e-12..20); negative and NaN arguments give
NaN, as CUDA's does.  0 and +inf give NaN where CUDA gives inf and 0: the
traversals call it only for squared distances at or above a positive width
threshold, finite.  Subnormal arguments (below 2.2e-308) are flushed to
zero; they are not tested."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _probe(x):
    import torch
    from cagr_b200 import _lib
    out = torch.empty_like(x)
    _lib.check(_lib.lib().cagr_probe_rsqrt64(
        ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()), x.numel(),
        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)), "cagr_probe_rsqrt64")
    torch.cuda.synchronize()
    return out


def test_rsqrt64_within_2_ulp(cuda_lib):
    import torch
    rng = np.random.default_rng(120)
    x = np.concatenate([10.0 ** rng.uniform(-300, 300, 200_000),
                        10.0 ** rng.uniform(-12, 1.3, 200_000),
                        np.array([1.0, 4.0, 0.25, 2.0, 3.0, 1e-300, 1e300])])
    X = torch.from_numpy(x).cuda()
    got = _probe(X).cpu().numpy()
    cuda = torch.rsqrt(X).cpu().numpy()
    ref = 1.0 / np.sqrt(x)
    for want in (cuda, ref):
        ulps = np.abs(got - want) / np.spacing(np.abs(want))
        assert ulps.max() <= 2.0, ulps.max()


def test_rsqrt64_nan_arguments(cuda_lib):
    import torch
    x = torch.tensor([-1.0, float("nan"), -float("inf"), -1e-300],
                     dtype=torch.float64, device="cuda")
    got = _probe(x).cpu().numpy()
    assert np.isnan(got).all()
    assert np.isnan(torch.rsqrt(x).cpu().numpy()).all()
