#!/usr/bin/env python
"""Benchmark of the CAGR treecode hot path on B200.

One step = one convection-augmented Gauss operator pair at 1M points, as the
CAGR normal solve applies it (main_CAGR.py:107-116):
  A.mu   -- node moments of mu + A21/A22/A23 in one fused traversal
  A^T.w  -- sum_k A2Tk(w_k): for each k node moments of w_k + one traversal
            (the reference's three calls with their own node moments)
Workload: 1,000,000 points on the union of 8 seeded primitives (normalised as
main_CAGR.py does), octree leaf 1 / depth 15 (the reference defaults), per-point
width 1.5 x the mean distance to the 10 nearest neighbours.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  For N > 1 (torchrun) every rank runs an
independent replica (one GPU's worth of work does not need sharding) and
times are the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "treecode A·μ+Aᵀ·w ms and end-to-end s @1M pts, FP32/adjoint vs FP64 form"
UNIT = "ms"
# FP32 work per pair term, counted from the kernel source (cagr_b200/csrc/traverse.cu,
# pair_term; an FMA counts 2): d (3) + |d|^2 without contraction (5) + r^-3 (2)
# + d.mu (5) + d.mu r^-3 (1) + r^-1/2 (1), then per direction 2 FMA (4):
FLOPS_A2_FUSED = 29      # three directions
FLOPS_A2T = 22           # d (3) + |d|^2 (5) + r^-3 (2) + e s r^-3 (2) + 3 FMA (6) + e s r^-1/2 (3) + add (1)
# The interpolated A2T sum evaluates all three directions of a (query, source)
# pair at once (cagr_b200/csrc/interp.cu, pterm, A2T sum): d (3) + |d|^2 (5)
# + r^-3 (2) + g_k = exp(x_k/2) (exp(-y_k/2) s_k) (3) + sum g (2) + (sum g) r^-3 (1)
# + r/2 (1) + per direction d_k c + g_k r/2 as 2 FMA (12); rsqrt not counted,
# as in the counts above.  (Per-direction terms of the reference mode: 22 each.)
FLOPS_IA2T_SUM = 29
L2_FLUSH_BYTES = 256 << 20
# Counters of the two traversals on this workload from one ncu capture of the
# warm-up step's launches (ncu does not run inside the bench; these are
# constants of that capture, reported with the command that made it): DRAM
# bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum), MUFU (XU
# pipe) and issue-slot utilisation, FMA-pipe activity.
TRAFFIC_BYTES = {"A2T_SUM": 163_672_832 + 7_347_968, "A2_FUSED": 136_197_888 + 4_479_488}
KERNEL_COUNTERS = {
    "A2T_SUM": {"mufu_frac": 0.1493, "issue_active": 0.8898, "fma_pipe_active": 0.3858},
    "A2_FUSED": {"mufu_frac": 0.0962, "issue_active": 0.7988, "fma_pipe_active": 0.3437},
}
TRAFFIC_SOURCE = ("ncu --metrics smsp__issue_active.avg.pct_of_peak_sustained_active,"
                  "sm__inst_executed_pipe_xu.avg.pct_of_peak_sustained_active,"
                  "sm__pipe_fma_cycles_active.avg.pct_of_peak_sustained_active,"
                  "dram__bytes_read.sum,dram__bytes_write.sum,gpu__time_duration.sum "
                  "--clock-control none -k regex:k_traverse -s 5 -c 2 python bench.py --steps 1 "
                  "--warmup 1 --no-fp64 --no-cpu-baseline --no-interp (one capture, not measured "
                  "in this run)")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="union8")
    ap.add_argument("--n", type=int, default=1_000_000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-solve", action="store_true")
    ap.add_argument("--no-interp", action="store_true",
                    help="skip the interpolated far-field mode's leg")
    ap.add_argument("--interp-degree", type=int, default=5)
    ap.add_argument("--grid", type=int, default=512, help="field grid for the end-to-end run")
    return ap.parse_args()


# ---------------------------------------------------------------- workload ----

def knn_widths(p: np.ndarray, k: int = 10, scale: float = 1.5) -> np.ndarray:
    from scipy.spatial import cKDTree
    d, _ = cKDTree(p).query(p, k=k + 1, workers=-1)
    return (scale * d[:, 1:].mean(1)).astype(p.dtype)


def make_workload(name: str, n: int, seed: int = 2):
    from cagr_b200 import synthetic as S
    raw = S.make(name, n, seed)
    p = S.normalize(raw).astype(np.float32)
    widths = knn_widths(p)
    # mu: area-weighted outward normals of the cloud (the magnitude CAGR's mu has)
    c = p.astype(np.float64) - p.mean(0)
    mu = (c / np.maximum(np.linalg.norm(c, axis=1, keepdims=True), 1e-12) * (4.0 / n))
    return p, widths, mu.astype(np.float32)


def workload_config(args, width_mean: float) -> dict:
    return {
        "workload": (f"{args.workload}: {args.n:,} points on the union of 8 seeded primitives "
                     "(seed 2, noise 1e-3), normalised as main_CAGR.py; octree leaf 1, depth 15; "
                     "per-point width 1.5x mean 10-NN distance"),
        "points": args.n,
        "step": ("A.mu (moments of mu + one A21/A22/A23 traversal) + A^T.w (moments of w_1, "
                 "w_2, w_3 + one traversal summing A2T1(w_1) + A2T2(w_2) + A2T3(w_3), each "
                 "direction with its own moments and acceptance decisions)"),
        "width_mean": round(width_mean, 6),
        "l2": "flushed between timed steps (256 MiB write)",
        "parallelism": "replicas" if args.gpus > 1 else "single",
    }


# ------------------------------------------------------------------ clocks ----

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "20"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "samples": len(sm), "reasons": sorted(reasons)}


# ------------------------------------------------------------- CPU legs -------

class CpuReference:
    """The reference's own CPU-side algorithm for the step: the reference CUDA
    kernels compiled for the host (oracle/_ref) when present, else the C
    restatement, on every host thread (OpenMP over queries).  The tree is built
    once, as the reference builds it once per solve."""

    def __init__(self, p):
        from oracle.oracle import Oracle, RefOracle
        try:
            self.impl, self.kind = RefOracle(), "reference"
        except (FileNotFoundError, OSError):
            self.impl, self.kind = Oracle(), "port"
        self.tree = self.impl.build_tree(p)

    def step_ms(self, p, widths, mu, wvals, threads: int):
        """One full step: per A21/A22/A23/A2T1/A2T2/A2T3 call |value| weights,
        node moments over the whole tree and the traversal of all queries.
        Returns (ms, description)."""
        ms = cpu_reference_step_ms(self.impl, self.tree, p, widths, mu, wvals)
        desc = (f"the whole step: all {p.shape[0]:,} queries per operator, node moments "
                f"over all {self.tree.num_nodes:,} nodes, 6 operator calls (A21, A22, A23, "
                f"A2T1, A2T2, A2T3) as main_CAGR.py makes them; {threads} OpenMP threads")
        return ms, desc


def cpu_reference_step_ms(impl, tree, p, widths, mu, wvals):
    from oracle.oracle import point_weights
    q, wq = p, widths
    t_scatter = t_trav = 0.0
    for op, vals in (("A21", mu), ("A22", mu), ("A23", mu), ("A2T1", wvals[:, 0:1]),
                     ("A2T2", wvals[:, 1:2]), ("A2T3", wvals[:, 2:3])):
        vals = np.ascontiguousarray(vals)
        t0 = time.perf_counter()
        mom = impl.moments(tree, p, point_weights(vals), vals)
        t1 = time.perf_counter()
        impl.multiply(op, q, wq, p, vals, tree, mom)
        t2 = time.perf_counter()
        t_scatter += t1 - t0
        t_trav += t2 - t1
    return (t_scatter + t_trav) * 1e3


def max_over_ranks(values, world: int, device):
    """Each rank runs one replica: the job's step time is the slowest rank's.
    A collective over the process group (NCCL on GPUs, gloo in the CPU tests)."""
    if world <= 1:
        return list(values)
    import torch
    import torch.distributed as dist
    t = torch.tensor(list(values), device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t]


def run_reference_arm(args, rank: int):
    if rank != 0:
        return
    import multiprocessing
    threads = multiprocessing.cpu_count()
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    p, widths, mu = make_workload(args.workload, args.n)
    rng = np.random.default_rng(5)
    wvals = rng.normal(size=(args.n, 3)).astype(np.float32) * 1e-3
    cpu = CpuReference(p)
    kind = cpu.kind
    times = []
    desc = None
    for i in range(args.warmup + args.steps):
        ms, desc = cpu.step_ms(p, widths, mu, wvals, threads)
        if i >= args.warmup:
            times.append(ms)
    v = float(np.mean(times))
    line = {
        "impl": "reference", "metric": METRIC, "value": round(v, 3), "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(v, 3), "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(args, float(widths.mean())),
        "cpu_baseline": {"value": round(v, 3), "unit": UNIT, "cores": threads, "kind": kind,
                         "sample": desc},
        "e2e": {"value": round(v, 3), "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ GPU arm ---

def field_error_sample(p, rng, n_grid=400, n_self=400, grid=512, lo=-1.2, hi=1.2):
    """Queries for the field error against the FP64 direct sum: random nodes of
    the reconstruction grid (A3, continuous kernel, width 0.01, as the field
    evaluation runs) and random input points (the solve's self-queries)."""
    h = np.float32((hi - lo) / (grid - 1))
    idx = rng.integers(0, grid, size=(n_grid, 3))
    qg = (idx.astype(np.float64) * np.float64(h) + np.float64(np.float32(lo))).astype(np.float32)
    sel = np.sort(rng.choice(p.shape[0], size=n_self, replace=False))
    return qg, sel


def interp_leg(args, P, W, MU, WV, p, widths, mu, dev, stream, flush, rank):
    import torch

    from cagr_b200 import WindingNumberTreecode
    from oracle.oracle import Oracle
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    wn = WindingNumberTreecode(P, far_field="interp", degree=args.interp_degree, theta=0.5)
    out_a = torch.empty(P.shape[0], 3, device=dev)
    out_t = torch.empty(P.shape[0], 3, device=dev)
    wn.scatter(MU)
    terms = float(wn.multiply("COUNT", W).sum().item())

    def step(marks):
        marks[0].record(stream)
        wn.scatter(MU)
        marks[1].record(stream)
        wn.multiply("A2_FUSED", W, out=out_a)
        marks[2].record(stream)
        wn.scatter3(WV)
        marks[3].record(stream)
        wn.multiply("A2T_SUM", W, out=out_t)
        marks[4].record(stream)

    for _ in range(max(1, args.warmup)):
        step([ev() for _ in range(5)])
    torch.cuda.synchronize(dev)
    st, a2, a2t = [], [], []
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    for _ in range(max(3, min(args.steps, 10))):
        flush.fill_(1.0)
        m = [ev() for _ in range(5)]
        step(m)
        torch.cuda.synchronize(dev)
        st.append(m[0].elapsed_time(m[4]))
        a2.append(m[1].elapsed_time(m[2]))
        a2t.append(m[3].elapsed_time(m[4]))
    leg_clocks = clocks.stop()
    leg = {"degree": args.interp_degree, "theta": 0.5, "clocks": leg_clocks,
           "proxy_grids": wn.far_field_info()["proxy_grids"],
           "step_ms": round(float(np.mean(st)), 3),
           "A2_FUSED_walk_ms": round(float(np.mean(a2)), 3),
           "A2T_SUM_walk_ms": round(float(np.mean(a2t)), 3),
           "pair_terms_A2": round(terms), "pair_terms_per_query": round(terms / P.shape[0])}
    if rank != 0 or args.n > 2_000_000:
        return leg
    # the A3 field (continuous kernel, width 0.01) of both modes against the FP64
    # direct sum, at random reconstruction-grid nodes and at random input points
    rng = np.random.default_rng(11)
    qg, sel = field_error_sample(p, rng)
    o = Oracle()
    ref_tree = WindingNumberTreecode(P)
    errs = {}
    for name, t in (("interp", wn), ("reference_mode", ref_tree)):
        t.scatter(MU)
        fg = t.multiply("A3", 0.01, queries=torch.from_numpy(qg).to(dev), continuous=True)
        fs = t.multiply("A3", 0.01, continuous=True)[torch.from_numpy(sel).to(dev)]
        errs[name] = (fg.cpu().numpy()[:, 0].astype(np.float64), fs.cpu().numpy()[:, 0].astype(np.float64))
    dg = o.direct("A3", qg, np.full(len(qg), 0.01), p, mu, continuous=True)[:, 0]
    ds = o.direct("A3", p[sel], np.full(len(sel), 0.01), p, mu, continuous=True)[:, 0]
    leg["field_error_vs_fp64_direct"] = {
        "queries": f"{len(qg)} random nodes of the 512^3 grid over [-1.2, 1.2]^3 and {len(sel)} "
                   "random input points; A3, continuous kernel, width 0.01",
        "field_range": [round(float(min(dg.min(), ds.min())), 4), round(float(max(dg.max(), ds.max())), 4)],
        **{f"max_abs_{k}": float(f"{max(np.abs(v[0] - dg).max(), np.abs(v[1] - ds).max()):.3e}")
           for k, v in errs.items()},
    }
    ref_tree.close()
    wn.close()
    return leg


def reference_reconstruction(points: np.ndarray, normals: np.ndarray, verts: np.ndarray,
                             faces: np.ndarray, like: tuple | None = None) -> dict:
    """The reference's CPU reconstructor (build_GR_cpu.sh's sources, built by
    `make -C oracle ref-gaussrecon`: its adaptive octree, host treecode with the
    plain Gauss operator, octree marching cubes) on the oriented cloud of this
    run's solve, timed as a whole program on the host cores (it sets 20 OpenMP
    threads itself), and the distance between its mesh and this run's 512^3
    reconstruction of the same oriented cloud (verts, faces), and `like`: a
    512^3 reconstruction with the reference driver's own operator and weights
    (A, unit normals times area 1e-5).  A CPU-baseline leg: the reference
    build is test infrastructure under oracle/."""
    exe = os.path.join(os.path.dirname(os.path.abspath(__file__)), "oracle", "_ref",
                       "main_GaussRecon_cpu")
    if not os.path.exists(exe):
        return {"unavailable": "the reference reconstructor is not built "
                               "(make -C oracle ref-gaussrecon needs the reference checkout)"}
    from oracle.mesh_distance import hausdorff, read_ply
    with tempfile.TemporaryDirectory() as d:
        xyz, ply = os.path.join(d, "oriented.xyz"), os.path.join(d, "ref.ply")
        np.hstack([points, normals]).astype(np.float32).tofile(xyz, sep=" ", format="%.7g")
        t0 = time.perf_counter()
        r = subprocess.run([exe, "-i", xyz, "-o", ply], cwd=d, capture_output=True, text=True,
                           timeout=1200)
        seconds = time.perf_counter() - t0
        if r.returncode != 0 or not os.path.exists(ply):
            return {"unavailable": f"the reference reconstructor failed (exit {r.returncode})"}
        rv, rf = read_ply(ply)
    diag = float(np.linalg.norm(rv.max(0) - rv.min(0)))
    H, mean = hausdorff((verts.astype(np.float64), faces), (rv, rf), n=100_000)
    out = {"value": round(seconds, 3), "unit": "s", "cores": os.cpu_count(), "threads": 20,
           "kind": "reference", "program": "main_GaussRecon_cpu (build_GR_cpu.sh sources)",
           "input": f"this run's {len(points):,} points with their solved normals",
           "mesh_vertices": int(rv.shape[0]), "mesh_faces": int(rf.shape[0]),
           "hausdorff_over_diagonal_vs_ours": round(H / diag, 5),
           "mean_distance_over_diagonal_vs_ours": round(mean / diag, 6),
           "ours": "end_to_end's mesh: A3, weights |mu|, 512^3 over [-1.2, 1.2]^3"}
    if like is not None:
        H2, mean2 = hausdorff((like[0].astype(np.float64), like[1]), (rv, rf), n=100_000)
        out["hausdorff_over_diagonal_vs_ours_same_operator"] = round(H2 / diag, 5)
        out["mean_distance_over_diagonal_vs_ours_same_operator"] = round(mean2 / diag, 6)
    return out


def run_ours(args, rank: int, world: int, local_rank: int):
    import ctypes

    import torch
    import torch.distributed as dist

    from cagr_b200 import WindingNumberTreecode, _lib

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)
    p, widths, mu = make_workload(args.workload, args.n)
    P = torch.from_numpy(p).to(dev)
    W = torch.from_numpy(widths).to(dev)
    MU = torch.from_numpy(mu).to(dev)
    wn = WindingNumberTreecode(P)
    # adjoint input: the forward result, as the solve feeds A2k(mu) back (main_CAGR.py:107-110)
    WV = (-wn.forward_A2(MU, W)).contiguous()
    out_a = torch.empty(args.n, 3, device=dev)
    out_t = torch.empty(args.n, 3, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, device=dev)
    wcols = [WV[:, k:k + 1].contiguous() for k in range(3)]

    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731

    def step(marks=None):
        # A.mu: moments of mu, then A21/A22/A23 in one traversal
        if marks is not None:
            marks[0].record(stream)
        wn.scatter(MU)
        if marks is not None:
            marks[1].record(stream)
        wn.multiply("A2_FUSED", W, out=out_a)
        if marks is not None:
            marks[2].record(stream)
        # A^T.w: moments of w_1, w_2, w_3 (one launch), then sum_k A2Tk(w_k) in one traversal
        wn.scatter3(WV)
        if marks is not None:
            marks[3].record(stream)
        wn.multiply("A2T_SUM", W, out=out_t)
        if marks is not None:
            marks[4].record(stream)

    launches_per_step = 4

    # pair-term counts of every traversal in a step (algorithmic work): each
    # direction of the adjoint counted with its own moments
    wn.scatter(MU)
    terms_a2 = float(wn.multiply("COUNT", W).sum().item())
    terms_t = []
    for k in range(3):
        wn.scatter(wcols[k])
        terms_t.append(float(wn.multiply("COUNT", W).sum().item()))

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()

    clocks = ClockSampler(local_rank)
    clocks.start()
    step_ms, a2_ms, a2t_ms, mom_ms = [], [], [], []
    for _ in range(args.steps):
        flush.fill_(1.0)
        marks = [ev() for _ in range(5)]
        step(marks)
        torch.cuda.synchronize(dev)
        step_ms.append(marks[0].elapsed_time(marks[4]))
        mom_ms.append(marks[0].elapsed_time(marks[1]) + marks[2].elapsed_time(marks[3]))
        a2_ms.append(marks[1].elapsed_time(marks[2]))
        a2t_ms.append(marks[3].elapsed_time(marks[4]))
    torch.cuda.synchronize(dev)
    clk = clocks.stop()

    # the autograd backward of A.mu (cagr_b200.autograd): moments of mu + the
    # adjoint traversal (exact transpose of the forward's) + push to the points
    G = torch.randn(args.n, 3, device=dev, generator=torch.Generator(dev).manual_seed(3))
    grad_mu = torch.empty_like(MU)
    adj_ms = []
    for it in range(args.warmup + 5):
        flush.fill_(1.0)
        a, b = ev(), ev()
        a.record(stream)
        wn.scatter(MU)
        wn.adjoint_A2(G, W, out=grad_mu)
        b.record(stream)
        torch.cuda.synchronize(dev)
        if it >= args.warmup:
            adj_ms.append(a.elapsed_time(b))

    # end to end through the public API with host buffers
    h_mu = torch.from_numpy(mu).pin_memory()
    h_w = WV.cpu().pin_memory()
    h_oa = torch.empty(args.n, 3).pin_memory()
    h_ot = torch.empty(args.n, 3).pin_memory()
    d_mu = torch.empty_like(MU)
    d_w = torch.empty_like(WV)

    # the copies the computation does not wait for run on a side stream: w
    # uploads while A.mu runs, A.mu's result downloads while A^T.w runs (all of
    # them inside the timed region: the step ends when the side stream is done)
    side = torch.cuda.Stream(device=dev)
    w_up, a_done, mu_up = torch.cuda.Event(), torch.cuda.Event(), torch.cuda.Event()

    def e2e_step():
        side.wait_stream(stream)                 # the previous step is done with d_w
        d_mu.copy_(h_mu, non_blocking=True)
        mu_up.record(stream)
        with torch.cuda.stream(side):
            # w follows mu over the bus: mu, which A.mu waits for, gets all of it
            side.wait_event(mu_up)
            d_w.copy_(h_w, non_blocking=True)
            w_up.record(side)
        oa = wn.forward_A2(d_mu, W)
        a_done.record(stream)
        with torch.cuda.stream(side):
            side.wait_event(a_done)
            oa.record_stream(side)
            h_oa.copy_(oa, non_blocking=True)
        stream.wait_event(w_up)                  # only the upload of w
        ot = wn.forward_A2T_sum(d_w, W)
        h_ot.copy_(ot, non_blocking=True)
        stream.wait_stream(side)                 # the step ends with A.mu's download too

    for _ in range(2):
        e2e_step()
    torch.cuda.synchronize(dev)
    e2e_ms = []
    for _ in range(max(3, args.steps // 2)):
        flush.fill_(1.0)
        a, b = ev(), ev()
        a.record(stream)
        e2e_step()
        b.record(stream)
        torch.cuda.synchronize(dev)
        e2e_ms.append(a.elapsed_time(b))

    # FP64 form of the same step (the plain FP64-accumulate comparison)
    fp64_ms = None
    if not args.no_fp64:
        wn64 = WindingNumberTreecode(P.double())
        W64, MU64, WV64 = W.double(), MU.double(), WV.double()
        for _ in range(2):
            wn64.forward_A2(MU64, W64)
            wn64.forward_A2T_sum(WV64, W64)
        torch.cuda.synchronize(dev)
        t = []
        for _ in range(3):
            flush.fill_(1.0)
            a, b = ev(), ev()
            a.record(stream)
            wn64.forward_A2(MU64, W64)
            wn64.forward_A2T_sum(WV64, W64)
            b.record(stream)
            torch.cuda.synchronize(dev)
            t.append(a.elapsed_time(b))
        fp64_ms = float(np.mean(t))
        wn64.close()

    # end to end: the whole CAGR normal solve on this cloud (tree build + 40
    # iterations + 8 G steps, main_CAGR.py's schedule, preset l0)
    solve = solve64 = our_mesh = our_mesh_like = None
    if not args.no_solve:
        from cagr_b200.mesh import reconstruct
        from cagr_b200.solver import PRESET_WIDTHS, cagr_solve

        def pipeline(pts):
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            res = cagr_solve(pts, *PRESET_WIDTHS["l0"])
            torch.cuda.synchronize(dev)
            t1 = time.perf_counter()
            rec = reconstruct(pts, res.normals, grid=args.grid)
            torch.cuda.synchronize(dev)
            return res, rec, t1 - t0, time.perf_counter() - t1

        def record(res, rec, t_solve, t_rec, first):
            return {"total_s": round(t_solve + t_rec, 4), "solve_s": round(t_solve, 4),
                    "tree_build_s": round(res.time_tree_s, 4),
                    "iterations_s": round(res.time_main_s, 4),
                    "operator_calls": res.operator_calls, "preset": "l0",
                    "reconstruct_s": round(t_rec, 4), "grid": args.grid,
                    "field_s": round(rec.seconds["field"], 4),
                    "marching_cubes_s": round(rec.seconds["marching_cubes"], 4),
                    "vertices": int(rec.vertices.shape[0]), "faces": int(rec.faces.shape[0]),
                    "first_call_total_s": round(first, 4)}

        # the first run pays one-off costs (module loading of the kernels and torch
        # ops it touches, growth of the memory pools to this size): reported apart,
        # the second run is the number
        _, rec, c_solve, c_rec = pipeline(P)
        del rec
        res, rec, t_solve, t_rec = pipeline(P)
        solve = record(res, rec, t_solve, t_rec, c_solve + c_rec)
        our_mesh = (rec.vertices.cpu().numpy(), rec.faces.cpu().numpy(),
                    res.normals.float().cpu().numpy())
        del rec
        # the same normals through the reference CPU driver's operator and weights
        # (A, n / |n| * 1e-5), for the like-for-like mesh distance
        rec = reconstruct(P, res.normals.float(), grid=args.grid, area=1e-5, op="A")
        our_mesh_like = (rec.vertices.cpu().numpy(), rec.faces.cpu().numpy())
        del rec
        if not args.no_fp64:
            # the same pipeline in float64 throughout (points, widths, moments, pair
            # sums, Krylov scalars, field; marching cubes on the field rounded to
            # float32): the FP64 form the mixed-precision pipeline is compared with
            P64 = P.double()
            _, rec, c_solve, c_rec = pipeline(P64)
            del rec
            res, rec, t_solve, t_rec = pipeline(P64)
            solve64 = record(res, rec, t_solve, t_rec, c_solve + c_rec)
            solve64["form"] = ("float64 throughout; 1/sqrt as rsqrt.approx.f64 refined by one "
                               "third-order step (within 2 ulp of CUDA's rsqrt(double))")
            del rec

    # the interpolated far-field mode: the same step with the far field
    # interpolated on Chebyshev proxy grids (degree --interp-degree, theta 0.5),
    # and the field error of both modes against the FP64 direct sum
    interp = None
    if not args.no_interp:
        interp = interp_leg(args, P, W, MU, WV, p, widths, mu, dev, stream, flush, rank)

    # measured FP32 FMA peak (roofline denominator)
    gf = ctypes.c_double()
    _lib.check(_lib.lib().cagr_probe_fp32_peak(20000, ctypes.byref(gf),
                                               ctypes.c_void_p(stream.cuda_stream)),
               "cagr_probe_fp32_peak")
    peak_tflops = gf.value / 1e3

    if interp is not None:
        # FP32 work of the interpolated walks per (query, source) pair term, a proxy
        # term counting as a point term: A2_FUSED as in the reference mode, the A2T
        # sum with its three directions together
        ta = interp["pair_terms_A2"] * FLOPS_A2_FUSED / (interp["A2_FUSED_walk_ms"] * 1e-3) / 1e12
        tt = interp["pair_terms_A2"] * FLOPS_IA2T_SUM / (interp["A2T_SUM_walk_ms"] * 1e-3) / 1e12
        interp["flops_per_pair_term"] = {"A2_FUSED": FLOPS_A2_FUSED, "A2T_SUM": FLOPS_IA2T_SUM}
        interp["A2_FUSED_tflops"], interp["A2_FUSED_fp32_frac"] = round(ta, 3), round(ta / peak_tflops, 4)
        interp["A2T_SUM_tflops"], interp["A2T_SUM_fp32_frac"] = round(tt, 3), round(tt / peak_tflops, 4)
    T, E = max_over_ranks([float(np.mean(step_ms)), float(np.mean(e2e_ms))], world, dev)
    if rank != 0:
        return

    # dominant kernel: the traversal with the most time per step
    a2_avg = float(np.mean(a2_ms))
    a2t_avg = float(np.mean(a2t_ms))
    if a2t_avg >= a2_avg:
        dom, dur, key = "k_traverse_a2t3 (A2T_SUM)", a2t_avg, "A2T_SUM"
        terms_dom, fpt = float(sum(terms_t)), FLOPS_A2T
    else:
        dom, dur, key = "k_traverse<A2_FUSED>", a2_avg, "A2_FUSED"
        terms_dom, fpt = terms_a2, FLOPS_A2_FUSED
    traffic = TRAFFIC_BYTES[key] if args.n == 1_000_000 and args.workload == "union8" else None
    achieved = terms_dom * fpt / (dur * 1e-3) / 1e12
    cpu = recon_ref = None
    if not args.no_cpu_baseline and our_mesh is not None:
        recon_ref = reference_reconstruction(p, our_mesh[2], our_mesh[0], our_mesh[1],
                                             our_mesh_like)
    if not args.no_cpu_baseline:
        import multiprocessing
        threads = multiprocessing.cpu_count()
        wv_host = WV.cpu().numpy()
        ref_cpu = CpuReference(p)
        ms, desc = ref_cpu.step_ms(p, widths, mu, wv_host, threads)
        cpu = {"value": round(ms, 3), "unit": UNIT, "cores": threads, "kind": ref_cpu.kind,
               "sample": desc}
    bi = (MU.numel() + WV.numel()) * 4
    bo = (out_a.numel() + out_t.numel()) * 4
    line = {
        "metric": METRIC, "value": round(T / world, 4), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(T, 4),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": workload_config(args, float(widths.mean())),
        "e2e": {"value": round(E / world, 4), "unit": UNIT, "h2d_bytes_per_step": bi,
                "d2h_bytes_per_step": bo},
        "gpu_launches": launches_per_step * args.steps,
        "roofline": {"bound": "fp32", "kernel": dom, "achieved": round(achieved, 3),
                     "peak": round(peak_tflops, 3), "unit": "TFLOP/s",
                     "frac": round(achieved / peak_tflops, 4), "traffic": traffic,
                     "traffic_unit": "bytes per launch",
                     "traffic_source": TRAFFIC_SOURCE if traffic is not None else None,
                     "counters": (dict(KERNEL_COUNTERS[key], source=TRAFFIC_SOURCE)
                                  if traffic is not None else None),
                     "peak_source": "measured FP32 FMA probe (cagr_probe_fp32_peak)",
                     "pair_terms_per_launch": round(terms_dom), "flops_per_term": fpt},
        "kernels_ms": {"moments_per_step": round(float(np.mean(mom_ms)), 4),
                       "A2_FUSED": round(a2_avg, 4), "A2T_SUM": round(a2t_avg, 4),
                       "A2_FUSED_backward": round(float(np.mean(adj_ms)), 4)},
        "pair_terms": {"A2_FUSED": round(terms_a2), "A2T1": round(terms_t[0]),
                       "A2T2": round(terms_t[1]), "A2T3": round(terms_t[2])},
        "fp64_ms_per_step": None if fp64_ms is None else round(fp64_ms, 3),
        "interp": interp,
        "end_to_end": solve,
        "end_to_end_fp64": solve64,
        "end_to_end_fp64_over_fp32": (round(solve64["total_s"] / solve["total_s"], 3)
                                      if solve and solve64 else None),
        "clocks": clk,
    }
    if cpu is not None:
        line["cpu_baseline"] = cpu
    if recon_ref is not None:
        line["cpu_baseline_reconstruction"] = recon_ref
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference_arm(args, rank)
        return
    import datetime

    import torch
    import torch.distributed as dist
    if world > 1:
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
