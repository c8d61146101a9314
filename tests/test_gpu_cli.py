"""GPU: the command line, run as the reference's programs are run.

* `python -m cagr_b200 orient bunny.xyz --width_config l0 --iters 10` writes
  results/bunny.xyz as main_CAGR.py does (CUDA-based/main_CAGR.py:185-186): the
  input points unchanged, then normals whose signs agree with the reference's
  published output (CUDA-based/results/bunny.xyz) on >= 99.5 % of the points;
* `python -m cagr_b200 recon -i results/bunny.xyz -o mesh --grid 96` writes
  mesh.ply: a closed, consistently oriented surface inside the input's box.
"""
import os
import subprocess
import sys
from collections import Counter

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def _run(args, cwd):
    env = dict(os.environ, PYTHONPATH=ROOT + os.pathsep + os.environ.get("PYTHONPATH", ""))
    r = subprocess.run([sys.executable, "-m", "cagr_b200", *args], cwd=cwd, env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout


def test_orient_then_recon_on_the_bunny(cuda_lib, tmp_path):
    from cagr_b200.mesh import read_ply
    g = np.load(os.path.join(GOLDEN, "bunny.npz"))
    pts = np.asarray(g["points"], np.float64)
    np.savetxt(tmp_path / "bunny.xyz", pts)
    out = _run(["orient", "bunny.xyz", "--width_config", "l0", "--iters", "10",
                "--out_dir", "results"], tmp_path)
    assert "[LOG] time_main:" in out
    oriented = np.loadtxt(tmp_path / "results" / "bunny.xyz")
    assert oriented.shape == (len(pts), 6)
    assert np.array_equal(oriented[:, :3], pts)
    agree = float(((oriented[:, 3:] * g["mu_reference"]).sum(1) > 0).mean())
    assert agree >= 0.995, agree

    _run(["recon", "-i", "results/bunny.xyz", "-o", "mesh", "--grid", "96"], tmp_path)
    v, f = read_ply(str(tmp_path / "mesh.ply"))
    assert len(f) > 2000
    lo, hi = pts.min(0), pts.max(0)
    pad = 0.05 * (hi - lo).max()
    assert (v >= lo - pad).all() and (v <= hi + pad).all()
    edges = Counter()
    for a, b, c in f:
        edges.update([(a, b), (b, c), (c, a)])
    # every directed edge once and its reverse once: closed, consistently oriented
    assert max(edges.values()) == 1
    assert all((b, a) in edges for a, b in edges)
