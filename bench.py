"""Benchmark of the batched ImmutableKdTree query engine on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload c2_knn16|c2_approx|c1_nn1]

Default workload (the headline config): ImmutableKdTree<f32, 3>, 16,000,000
points of a Gaussian mixture (1,024 centres uniform in [0,1)^3, sigma 0.005,
Dirichlet(1) weights) of which 20% are a uniform background; 16,000,000
queries drawn from the same mixture; nearest_n(16) sorted, SquaredEuclidean.
One step = the whole query batch through one engine call.  Inputs are seeded
synthetic arrays (no dataset); the tree (256 MB arena) and the queries
(192 MB) are both larger than the 126 MB L2, so no flush is needed between
steps.

Under torchrun each rank owns one GPU, holds its own replica of the tree and
answers its own 16M queries (weak scaling, no data-path collective); timing is
the max over ranks of the CUDA-event time.  `--impl reference` times the CPU
restatement of the reference path (the oracle; the Rust reference cannot be
built here) on all host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import threading
import time

import numpy as np

METRIC = "bit-exact kNN queries/s on 1 B200: batched vs per-tree launch; Chamfer fwd+bwd/s"
ROOT = os.path.dirname(os.path.abspath(__file__))

WORKLOADS = {
    # name: (dtype, n_points, n_queries, family, k)
    "c2_knn16": ("f32", 16_000_000, 16_000_000, "nearest_n", 16),
    "c2_approx": ("f32", 16_000_000, 16_000_000, "approx", 1),
    "c1_nn1": ("f64", 100_000, 1_000_000, "nearest_one", 1),
}


def gaussian_mixture(n, rng, centres, dtype, sigma=0.005, background=0.2):
    """1,024 centres uniform in [0,1)^3, isotropic sigma, Dirichlet(1)
    weights, plus a uniform background fraction (the C2 distribution)."""
    nb = int(round(n * background))
    nm = n - nb
    w = rng.dirichlet(np.ones(len(centres)))
    lab = rng.choice(len(centres), size=nm, p=w)
    pts = np.empty((n, 3), dtype=dtype)
    pts[:nm] = centres[lab] + rng.normal(0.0, sigma, size=(nm, 3))
    pts[nm:] = rng.random((nb, 3))
    return pts[rng.permutation(n)]


def make_data(workload, rank, n=None, nq=None):
    dt, n0, nq0, fam, k = WORKLOADS[workload]
    n = n or n0
    nq = nq or nq0
    dtype = np.float32 if dt == "f32" else np.float64
    if workload == "c1_nn1":
        P = np.random.default_rng(0).random((n, 3)).astype(dtype)
        Q = np.random.default_rng(1 + 1000 * rank).random((nq, 3)).astype(dtype)
        return P, Q
    centres = np.random.default_rng(12345).random((1024, 3))
    P = gaussian_mixture(n, np.random.default_rng(0), centres, dtype)
    Q = gaussian_mixture(nq, np.random.default_rng(1 + 1000 * rank), centres, dtype)
    return P, Q


def builder_for(tree, Q, workload):
    import kiddo_b200 as kb
    _, _, _, fam, k = WORKLOADS[workload]
    b = tree.query(Q)
    if fam == "nearest_n":
        return b.nearest_n(kb.SquaredEuclidean, k)
    b = b.nearest_one(kb.SquaredEuclidean)
    if fam == "approx":
        b = b.approx()
    return b


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    QUERY = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(
                    ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.QUERY}",
                     "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                if out.returncode == 0 and out.stdout.strip():
                    self.samples.append([x.strip() for x in out.stdout.strip().split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for nm, v in zip(names, s[4:8]):
                if v.strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.samples)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic(workload):
    """dram bytes per launch from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", f"traffic_{workload}.json")
    try:
        with open(path) as f:
            return json.load(f)
    except Exception:
        return None


def cpu_baseline(tree, Q, workload, target_seconds=12.0, threads=0):
    """The CPU restatement of the reference path on the host cores, on a
    bounded sample of the same queries (test infrastructure: the oracle)."""
    import oracle
    lay = oracle.Layout(tree.dtype, tree.dims, tree.stems(), tree.leaf_bytes(),
                        tree.leaf_extents(), tree.max_stem_level(), tree.size(),
                        tree.max_leaf_len())
    ot = oracle.OracleTree.from_layout(lay)
    nthreads = threads if threads > 0 else (os.cpu_count() or 1)
    _, _, _, fam, k = WORKLOADS[workload]
    famcode = {"nearest_n": oracle.FAM_NEAREST_N, "approx": oracle.FAM_APPROX,
               "nearest_one": oracle.FAM_NEAREST_ONE}[fam]

    def run(m):
        t0 = time.perf_counter()
        ot.query_fixed(famcode, Q[:m], k=k, threads=nthreads)
        return time.perf_counter() - t0

    m = min(len(Q), 20000)
    dt = run(m)
    m2 = int(min(len(Q), max(m, m * target_seconds / max(dt, 1e-6))))
    if m2 > m:
        dt = run(m2)
        m = m2
    return {"value": m / dt, "unit": "queries/s", "cores": nthreads, "kind": "port",
            "sample": f"{m} of the {len(Q)} queries, {fam}(k={k}), {nthreads} threads, "
                      f"{dt:.1f} s, oracle (C++ restatement of the reference scalar path)"}


def bytes_per_query(stats, nq, dtype_size, k):
    """Algorithmic bytes of one query: the query, every
    stem visited, every point scanned (K coords + u32 item), and the output."""
    stems, leaves, pts = (float(x) / nq for x in stats)
    out = k * (dtype_size + 4) + (4 if k > 1 else 0)
    return 3 * dtype_size + stems * dtype_size + pts * (3 * dtype_size + 4) + out


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    P, Q = make_data(args.workload, 0)
    import kiddo_b200 as kb
    tree = kb.ImmutableKdTree.new_from_slice(P)
    _, _, _, fam, k = WORKLOADS[args.workload]
    times = []
    base = None
    for s in range(args.warmup + args.steps):
        cb = cpu_baseline(tree, Q, args.workload, target_seconds=8.0)
        if s >= args.warmup:
            times.append(cb["value"])
            base = cb
    val = statistics.median(times)
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": "queries/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": args.workload, "points": len(P), "queries": len(Q),
                       "family": fam, "k": k},
            "cpu_baseline": {"value": val, "unit": "queries/s", "cores": base["cores"],
                             "kind": "port", "sample": base["sample"]},
            "e2e": {"value": val, "unit": "queries/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c2_knn16", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--spatial-order", action="store_true")
    ap.add_argument("--engine", default=None, choices=["warp", "thread"],
                    help="force the kernel variant (default: the library chooses)")
    ap.add_argument("--points", type=int, default=0, help="override the tree size (profiling)")
    ap.add_argument("--queries", type=int, default=0, help="override the batch size (profiling)")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch
    import torch.distributed as dist
    import kiddo_b200 as kb
    from kiddo_b200 import multi

    torch.cuda.set_device(local)
    if world > 1:
        multi.init_process_group("nccl")
    dev = torch.device("cuda", local)
    dtype_name, n, nq, fam, k = WORKLOADS[args.workload]
    n = args.points or n
    nq = args.queries or nq
    P, Q = make_data(args.workload, rank, n, nq)
    tree = kb.ImmutableKdTree.new_from_slice(P)
    gtree = tree.to_gpu()
    stream = torch.cuda.current_stream(dev)
    dq = torch.from_numpy(Q).to(dev)

    def step():
        b = builder_for(gtree, dq, args.workload).with_engine(args.engine)
        if args.spatial_order:
            b = b.with_spatial_order()
        return b.execute_gpu()

    # algorithmic bytes per query from the engine's own traversal counters
    sub = Q[: min(nq, 2_000_000)]
    stats = builder_for(gtree, sub, args.workload).traversal_stats()
    bpq = bytes_per_query(stats, len(sub), Q.itemsize, k)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    multi.barrier()
    with ClockSampler(local) as clk:
        l0 = kb.launch_count()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
        torch.cuda.synchronize()
        ev[0].record(stream)
        for s in range(args.steps):
            step()
            ev[s + 1].record(stream)
        torch.cuda.synchronize()
        launches = kb.launch_count() - l0
    step_ms = [ev[i].elapsed_time(ev[i + 1]) for i in range(args.steps)]
    total_ms = sum(step_ms)
    total_ms_max = multi.max_over_ranks(total_ms)
    multi.barrier()

    # end to end through the C ABI with pinned host buffers
    hq = torch.from_numpy(Q).pin_memory().numpy()
    for _ in range(max(1, args.warmup // 2)):
        builder_for(gtree, hq, args.workload).execute_gpu()
    torch.cuda.synchronize()
    multi.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e2e_steps = max(1, min(args.steps, 3))
    e0.record(stream)
    for _ in range(e2e_steps):
        builder_for(gtree, hq, args.workload).execute_gpu()
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = multi.max_over_ranks(e0.elapsed_time(e1))

    w = 1 if fam != "nearest_n" else k
    h2d = nq * 3 * Q.itemsize
    d2h = nq * w * (Q.itemsize + 4) + (nq * 4)
    value = world * nq * args.steps / (total_ms_max / 1e3)
    e2e_val = world * nq * e2e_steps / (e2e_ms / 1e3)
    kern_ms = total_ms / args.steps
    achieved = bpq * nq / (kern_ms / 1e3) / 1e9
    peak, peak_kind = measured_peaks()
    traffic = profile_traffic(args.workload)
    line = {
        "metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if dtype_name == "f32" else "f64", "data": "synthetic",
        "config": {"workload": args.workload, "points": n, "queries_per_gpu": nq, "family": fam,
                   "k": k, "metric": "SquaredEuclidean", "parallelism": f"replicas{world}",
                   "l2": "inputs larger than L2 (tree 256 MB, queries 192 MB), no flush",
                   "spatial_order": bool(args.spatial_order),
                   "engine": args.engine or "auto"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "bytes_per_query": bpq,
                     "traffic": (traffic or {}).get("dram_bytes_per_launch"),
                     "kernel": "k_tfixed<nearest_n>" if args.engine != "warp" else "k_fixed<nearest_n>"},
        "e2e": {"value": e2e_val, "unit": "queries/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
        "traversal_per_query": {"stems": float(stats[0]) / len(sub),
                                "leaves": float(stats[1]) / len(sub),
                                "points": float(stats[2]) / len(sub)},
        "step_ms": step_ms,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(tree, Q, args.workload)
    if rank == 0:
        print(json.dumps(line), flush=True)
    multi.barrier()
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
