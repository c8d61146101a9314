"""Reference GPU baseline: the reference's own CUDA kernels on this B200.

TEST AND BASELINE INFRASTRUCTURE ONLY.  Times one operator pair of the CAGR
solve as the reference composes it (main_CAGR.py:107-110: A21, A22, A23 on
mu and A2T1, A2T2, A2T3 on the three columns of w, each call with its own
|value| weights and node scatter), in float32 and float64, on the bench.py
workload, and checks the reference kernels' results against the cagr_b200
kernels on the same tree.  Prints one JSON line.

    make -C oracle ref-gpu && python oracle/ref_gpu_bench.py [--n 1000000]
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from bench import make_workload  # noqa: E402
from cagr_b200 import WindingNumberTreecode  # noqa: E402
from oracle.ref_gpu import RefGPU  # noqa: E402


def rel_l2(a, b):
    a, b = a.double(), b.double()
    return float(torch.linalg.norm(a - b) / torch.linalg.norm(b))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=1_000_000)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=2)
    args = ap.parse_args()
    dev = torch.device("cuda")
    p, widths, mu = make_workload("union8", args.n)
    ref = RefGPU()
    out = {"n": args.n}
    flush = torch.empty(64 << 20, device=dev)
    for dtype, tag in ((torch.float32, "fp32"), (torch.float64, "fp64")):
        P = torch.from_numpy(p).to(dev, dtype)
        W = torch.from_numpy(widths).to(dev, dtype)
        MU = torch.from_numpy(mu).to(dev, dtype)
        wn = WindingNumberTreecode(P)
        tree = ref.tree_from(wn)
        WV = (-wn.forward_A2(MU, W)).contiguous()
        cols = [WV[:, k:k + 1].contiguous() for k in range(3)]

        def ref_step():
            a = [ref.forward(op, tree, MU, W) for op in ("A21", "A22", "A23")]
            t = [ref.forward(op, tree, cols[k], W) for k, op in enumerate(("A2T1", "A2T2", "A2T3"))]
            return torch.cat(a, 1), t[0] + t[1] + t[2]

        def our_step():
            return wn.forward_A2(MU, W), wn.forward_A2T_sum(WV, W)

        for _ in range(args.warmup):
            ref_step()
            our_step()
        torch.cuda.synchronize()
        times = {"ref": [], "ours": []}
        for _ in range(args.steps):
            for name, fn in (("ref", ref_step), ("ours", our_step)):
                flush.fill_(1.0)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                fn()
                e1.record()
                torch.cuda.synchronize()
                times[name].append(e0.elapsed_time(e1))
        ra, rt = ref_step()
        oa, ot = our_step()
        torch.cuda.synchronize()
        out[f"reference_gpu_{tag}_ms_per_step"] = round(float(np.mean(times["ref"])), 3)
        out[f"cagr_b200_{tag}_ms_per_step"] = round(float(np.mean(times["ours"])), 3)
        out[f"{tag}_rel_l2_A2"] = rel_l2(oa, ra)
        out[f"{tag}_rel_l2_A2T_sum"] = rel_l2(ot, rt)
        if tag == "fp32":
            # both GPU results against the reference algorithm in IEEE host arithmetic
            # (the reference's kernels compiled for the host), on sampled queries
            from oracle.oracle import RefOracle, point_weights
            host = RefOracle()
            pn = p.astype(np.float32)
            tr = host.build_tree(pn)
            mun = mu.astype(np.float32)
            mom = host.moments(tr, pn, point_weights(mun), mun)
            sel = np.random.default_rng(9).choice(args.n, size=min(50_000, args.n), replace=False)
            h21 = host.multiply("A21", pn[sel], widths[sel], pn, mun, tr, mom)[:, 0]
            g_ref = ra[:, 0].cpu().numpy()[sel]
            g_our = oa[:, 0].cpu().numpy()[sel]
            nrm = np.linalg.norm(h21)
            out["A21_rel_l2_vs_host_reference"] = {
                "reference_gpu": float(np.linalg.norm(g_ref - h21) / nrm),
                "cagr_b200": float(np.linalg.norm(g_our - h21) / nrm),
                "queries": int(len(sel))}
        wn.close()
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
