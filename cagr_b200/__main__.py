"""Command line, mirroring the reference's two programs.

    python -m cagr_b200 orient INPUT --width_config l0 [--wsmin W --wsmax W]
                               [--iters 40] [--out_dir results]
        main_CAGR.py (CUDA-based/main_CAGR.py:14-23, 27-38, 185-186): reads an
        .xyz / .npy point cloud (first three columns), normalises it, runs the
        CAGR solve and writes OUT_DIR/<name>.xyz with the input points and the
        solved normals (six columns).

    python -m cagr_b200 recon -i ORIENTED.xyz -o OUT [-w 0.01] [--grid 256 | -d 8]
        main_GaussReconCUDA (ext/gaussrecon_src/main_GaussRecon_cuda.cu:236-245,
        266-301, 427-494): oriented points (six columns) -> normals rescaled to
        n / |n| * 1e-5, field A3 (continuous kernel, width -w) on a regular
        grid, iso-value = the median at the samples, marching cubes -> OUT.ply
        in the input's coordinates.  The reference evaluates on an adaptive
        octree of depth -d; here -d d means a regular grid of 2^d + 1 nodes per
        axis.

There is no CPU path: --cpu is rejected.
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np


def _load_points(path: str, columns: int) -> np.ndarray:
    ext = os.path.splitext(path)[-1]
    if ext == ".xyz":
        data = np.loadtxt(path, ndmin=2)
    elif ext == ".npy":
        data = np.load(path)
    else:
        raise SystemExit(f"input must have extension xyz/npy, got {path}")
    if data.shape[1] < columns:
        raise SystemExit(f"{path}: need at least {columns} columns, found {data.shape[1]}")
    return np.asarray(data[:, :columns], np.float64)


def _orient(args) -> int:
    from .solver import orient_file
    if args.cpu:
        raise SystemExit("cagr_b200 has no CPU path (a CUDA device is required)")
    if os.path.splitext(args.input)[-1] not in (".xyz", ".npy"):
        raise SystemExit(f"input must have extension xyz/npy, got {args.input}")
    out, res = orient_file(args.input, args.width_config, args.wsmin, args.wsmax,
                           iters=args.iters)
    os.makedirs(args.out_dir, exist_ok=True)
    name = os.path.basename(args.input)[:-4] + ".xyz"
    np.savetxt(os.path.join(args.out_dir, name), out)
    print(f"[LOG] time_tree: {res.time_tree_s:.4f}")
    print(f"[LOG] time_main: {res.time_main_s:.4f}")
    return 0


def _recon(args) -> int:
    import torch
    from .mesh import reconstruct, write_ply
    data = _load_points(args.i, 6)
    raw, nrm = data[:, :3], data[:, 3:6]
    center = (raw.min(0) + raw.max(0)) / 2.0
    scale = 2.0 / ((raw.max(0) - raw.min(0)).max() * 1.1)       # as main_CAGR.py:42-45
    pts = torch.from_numpy(((raw - center) * scale).astype(np.float32)).cuda()
    mu = torch.from_numpy(nrm.astype(np.float32)).cuda()
    grid = args.grid if args.d is None else (1 << args.d) + 1
    rec = reconstruct(pts, mu, grid=grid, width=args.w, area=1e-5)
    v = rec.vertices.cpu().numpy().astype(np.float64) / scale + center
    write_ply(args.o + ".ply", v.astype(np.float32), rec.faces.cpu().numpy())
    print(f"[LOG] vertices {len(v)}, faces {rec.faces.shape[0]}, iso {rec.iso:.6g}")
    return 0


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m cagr_b200")
    sub = ap.add_subparsers(dest="cmd", required=True)
    o = sub.add_parser("orient", help="main_CAGR.py: solve for oriented normals")
    o.add_argument("input", type=str)
    o.add_argument("--width_config", type=str, required=True,
                   choices=["l0", "l1", "l2", "l3", "l4", "l5", "custom"])
    o.add_argument("--wsmax", type=float, default=0.01)   # the reference's defaults,
    o.add_argument("--wsmin", type=float, default=0.04)   # main_CAGR.py:17-18
    o.add_argument("--iters", type=int, default=40)
    o.add_argument("--out_dir", type=str, default="results")
    o.add_argument("--cpu", action="store_true")
    o.add_argument("--tqdm", action="store_true", help="accepted, no effect")
    r = sub.add_parser("recon", help="main_GaussReconCUDA: oriented points -> mesh")
    r.add_argument("-i", type=str, required=True, help="oriented points (.xyz, six columns)")
    r.add_argument("-o", type=str, required=True, help="output name without suffix")
    r.add_argument("-w", type=float, default=0.01, help="field width")
    r.add_argument("--grid", type=int, default=256, help="grid nodes per axis")
    r.add_argument("-d", type=int, default=None, help="depth: 2^d + 1 grid nodes per axis")
    r.add_argument("-m", type=int, default=None, help="accepted, no effect (regular grid)")
    args = ap.parse_args(argv)
    return _orient(args) if args.cmd == "orient" else _recon(args)


if __name__ == "__main__":
    sys.exit(main())
