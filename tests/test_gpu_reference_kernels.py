"""GPU: cagr_b200 against the reference's own CUDA kernels run on the same GPU.

oracle/_ref/libwnref_gpu.so is the reference's wn_treecode_cuda_kernels.cu
compiled for sm_100a with launchers replaying its torch interface.  On the
same tree (reference layout) and inputs, every operator must agree within the
FP32 / FP64 tolerances of the oracle tests.
"""
import os

import numpy as np
import pytest

from tests._cases import random_values, rel_errors, smooth_normals, sphere_cloud

pytestmark = pytest.mark.gpu

LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                   "libwnref_gpu.so")
OPS = ["A", "AT", "A3", "A21", "A22", "A23", "A2T1", "A2T2", "A2T3", "G"]


@pytest.mark.skipif(not os.path.exists(LIB), reason="reference GPU build absent")
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_all_operators_match_reference_cuda(cuda_lib, dtype):
    import torch
    from cagr_b200 import WindingNumberTreecode
    from oracle.ref_gpu import RefGPU
    ref = RefGPU()
    pts = sphere_cloud(20000, seed=40, dtype=dtype)
    wn = WindingNumberTreecode(torch.from_numpy(pts).cuda())
    tree = ref.tree_from(wn)
    w = torch.from_numpy(np.random.default_rng(41).uniform(0.005, 0.02, len(pts)).astype(dtype)).cuda()
    mu = torch.from_numpy(smooth_normals(pts, seed=42)).cuda()
    s = torch.from_numpy(random_values(len(pts), 1, seed=43, dtype=dtype)).cuda()
    tol = (2e-5, 2e-4) if dtype == np.float32 else (1e-12, 1e-11)
    for op in OPS:
        vals = s if op in ("AT", "A2T1", "A2T2", "A2T3") else mu
        r = ref.forward(op, tree, vals, w)
        o = getattr(wn, f"forward_{op}")(vals, w)
        l2, mx = rel_errors(o.cpu().numpy(), r.cpu().numpy())
        assert l2 <= tol[0] and mx <= tol[1], (op, l2, mx)
