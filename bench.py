"""Benchmark of the batched ImmutableKdTree query engine on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload c2_knn16|c2_approx|c1_nn1|c3_forest|c4_chamfer|c5_periodic]

Default workload (the headline config): ImmutableKdTree<f32, 3>, 16,000,000
points of a Gaussian mixture (1,024 centres uniform in [0,1)^3, sigma 0.005,
Dirichlet(1) weights) of which 20% are a uniform background; 16,000,000
queries drawn from the same mixture; nearest_n(16) sorted, SquaredEuclidean.
One step = the whole query batch through one engine call.  Inputs are seeded
synthetic arrays (no dataset); the tree (256 MB arena) and the queries
(192 MB) are both larger than the 126 MB L2, so no flush is needed between
steps.

On one GPU the default run measures every term of the metric in the same
process after the headline: approx on the same tree, the f64 nearest_one and
periodic configurations, the 256-catalogue forest batched against one launch
per tree, and Chamfer forward + backward; each becomes a sub-object of the
headline line (``--headline-only`` skips them).  Every timed result is sampled
(100,000 rows) against the oracle inside the run (``parity_sample``).

Under torchrun each rank owns one GPU, holds its own replica of the tree and
answers its own 16M queries (weak scaling, no data-path collective); timing is
the max over ranks of the CUDA-event time.  `--impl reference` times the CPU
restatement of the reference path (the oracle; the Rust reference cannot be
built here), built -O3 -march=native on the host it runs on, on all host
threads; it loads nothing of the product package.
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
    # every particle of a periodic unit box queries its 32 nearest within r = 0.01
    "c5_periodic": ("f64", 16_000_000, 16_000_000, "periodic_nearest_n_within", 32),
    # batches over many trees and Chamfer run through their own functions below
    "c3_forest": ("f32", 120_000_000, 64_000_000, "mixed", 5),
    "c4_chamfer": ("f32", 0, 0, "chamfer", 8),
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


def periodic_particles(n, rng, dtype, clumps=4096, sigma=0.002, clumped=0.7):
    """70% of the particles from 4,096 isotropic Gaussian clumps (sigma 0.002,
    centres uniform) wrapped into the unit box, 30% uniform."""
    nc = int(round(n * clumped))
    centres = rng.random((clumps, 3))
    pts = np.empty((n, 3), dtype=np.float64)
    pts[:nc] = centres[rng.integers(0, clumps, nc)] + rng.normal(0.0, sigma, (nc, 3))
    pts[nc:] = rng.random((n - nc, 3))
    pts = np.mod(pts, 1.0)
    pts[pts >= 1.0] = 0.0  # np.mod can round up to the box edge
    return pts[rng.permutation(n)].astype(dtype)


# rows of each timed result compared with the oracle inside the run
SAMPLE_ROWS = 100_000

# radius argument of the periodic neighbour lists, in the metric's own units
# (SquaredEuclidean: 0.01 = a Euclidean radius of 0.1), as within(0.01) takes it
C5_RADIUS = 0.01


def make_data(workload, rank, n=None, nq=None):
    dt, n0, nq0, fam, k = WORKLOADS[workload]
    n = n or n0
    nq = nq or nq0
    dtype = np.float32 if dt == "f32" else np.float64
    if workload == "c1_nn1":
        P = np.random.default_rng(0).random((n, 3)).astype(dtype)
        Q = np.random.default_rng(1 + 1000 * rank).random((nq, 3)).astype(dtype)
        return P, Q
    if workload == "c5_periodic":
        P = periodic_particles(n, np.random.default_rng(5), dtype)
        if nq == n:
            return P, P
        return P, periodic_particles(nq, np.random.default_rng(6 + 1000 * rank), dtype)
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
    if fam == "periodic_nearest_n_within":
        return (b.periodic_boundary_condition(np.ones(3)).nearest_n(kb.SquaredEuclidean, k)
                .within(C5_RADIUS))
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

    def wait_first(self, timeout=15.0):
        """Block until the first sample is in, so that starting nvidia-smi does
        not land inside the timed region."""
        t0 = time.time()
        while not self.samples and time.time() - t0 < timeout and self._t.is_alive():
            time.sleep(0.05)

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


def cpu_info():
    import oracle
    model, logical, physical = oracle.host_cpu()
    return {"cpu_model": model, "logical_cpus": logical, "physical_cores": physical}


def oracle_family(workload):
    import oracle
    _, _, _, fam, k = WORKLOADS[workload]
    code = {"nearest_n": oracle.FAM_NEAREST_N, "approx": oracle.FAM_APPROX,
            "nearest_one": oracle.FAM_NEAREST_ONE,
            "periodic_nearest_n_within": oracle.FAM_PERIODIC_NEAREST_N}[fam]
    extra = {"radius": C5_RADIUS, "box": np.ones(3)} if fam == "periodic_nearest_n_within" else {}
    return code, k, extra


def time_cpu(ot, Q, workload, target_seconds, threads):
    """Queries/s of the oracle tree `ot` on a bounded sample of Q: a first
    pass of 20,000 queries sizes a sample of about `target_seconds`."""
    fam, k, extra = oracle_family(workload)

    def run(m):
        t0 = time.perf_counter()
        ot.query_fixed(fam, Q[:m], k=k, threads=threads, **extra)
        return time.perf_counter() - t0

    m = min(len(Q), 20000)
    dt = run(m)
    m2 = int(min(len(Q), max(m, m * target_seconds / max(dt, 1e-6))))
    if m2 > m:
        dt = run(m2)
        m = m2
    reps = 1
    if m == len(Q) and dt < 0.5 * target_seconds:
        # the whole batch is quick: repeat it for a sample of about target_seconds
        reps = int(min(1000, max(2, target_seconds / max(dt, 1e-6))))
        dt = sum(run(m) for _ in range(reps))
    return m, reps, dt


def timing_tree_from(tree):
    """The oracle's -O3 -march=native build (built on this host) over the
    product tree's layout, for the CPU baseline leg of our own arm."""
    import oracle
    lay = oracle.Layout(tree.dtype, tree.dims, tree.stems(), tree.leaf_bytes(),
                        tree.leaf_extents(), tree.max_stem_level(), tree.size(),
                        tree.max_leaf_len())
    return oracle.OracleTree.from_layout(lay, L=oracle.timing_lib())


def cpu_baseline(tree, Q, workload, target_seconds=12.0, threads=0):
    """The CPU restatement of the reference path on all host cores, on a
    bounded sample of the same queries (test infrastructure: the oracle)."""
    ot = timing_tree_from(tree)
    nthreads = threads if threads > 0 else (os.cpu_count() or 1)
    _, _, _, fam, k = WORKLOADS[workload]
    m, reps, dt = time_cpu(ot, Q, workload, target_seconds, nthreads)
    return dict({"value": m * reps / dt, "unit": "queries/s", "cores": nthreads, "kind": "port",
                 "sample": f"{m} of the {len(Q)} queries x {reps}, {fam}(k={k}), {nthreads} "
                           f"threads, {dt:.1f} s; the oracle (C++ restatement of the reference "
                           f"scalar path) built -O3 -march=native -ffp-contract=off on this host"},
                **cpu_info())


def parity_sample(tree, Q, res, workload, n=SAMPLE_ROWS, seed=0):
    """Compare `n` seeded sampled rows of a timed result with the oracle (the
    checker build) on the same tree layout, bit for bit."""
    import oracle
    fam, k, extra = oracle_family(workload)
    rows = np.sort(np.random.default_rng(seed).choice(len(Q), size=min(n, len(Q)),
                                                      replace=False))
    lay = oracle.Layout(tree.dtype, tree.dims, tree.stems(), tree.leaf_bytes(),
                        tree.leaf_extents(), tree.max_stem_level(), tree.size(),
                        tree.max_leaf_len())
    ot = oracle.OracleTree.from_layout(lay)
    od, oi, oc = ot.query_fixed(fam, Q[rows], k=k, **extra)
    idx = __import__("torch").from_numpy(rows).to(res.distances.device)
    gd = res.distances.index_select(0, idx).cpu().numpy().reshape(len(rows), -1)
    gi = res.items.index_select(0, idx).cpu().numpy().view(np.uint32).reshape(len(rows), -1)
    same = np.all((gd == od) | (np.isnan(gd) & np.isnan(od)), axis=1) & np.all(gi == oi, axis=1)
    if getattr(res, "counts", None) is not None:
        gc = res.counts.index_select(0, idx).cpu().numpy().astype(np.uint32)
        same &= gc == oc
    return {"n": int(len(rows)), "mismatches": int((~same).sum()),
            "rule": "bit-exact distances, items and counts against the oracle, seeded rows"}


def bytes_per_query(stats, nq, dtype_size, k):
    """Algorithmic bytes of one query: the query, every
    stem visited, every point scanned (K coords + u32 item), and the output."""
    stems, leaves, pts = (float(x) / nq for x in stats)
    out = k * (dtype_size + 4) + (4 if k > 1 else 0)
    return 3 * dtype_size + stems * dtype_size + pts * (3 * dtype_size + 4) + out


def l2_note(n, nq, itemsize):
    tree_mb = n * (3 * itemsize + 4) / 1e6
    q_mb = nq * 3 * itemsize / 1e6
    big = "inputs larger than L2" if tree_mb > 126 else "tree fits in L2"
    return f"{big} (tree {tree_mb:.0f} MB, queries {q_mb:.0f} MB), no flush"


def kernel_name(fam, engine):
    if fam.startswith("periodic"):
        # rows away from the box's faces: the plain cooperative pass; the rest
        # (a few percent) take the periodic walk
        return ("k_tnn_coop (plain pass) + k_tperiodic_nn (rows near the faces)"
                if engine != "warp" else "k_periodic_fixed<nearest_n>")
    if fam == "nearest_n" and engine == "coop":
        return "k_tnn_coop"
    f = {"nearest_n": "nearest_n", "approx": "approx", "nearest_one": "nearest_one"}[fam]
    return f"k_tfixed<{f}>" if engine != "warp" else f"k_fixed<{f}>"


def config_for(workload, n, nq, world):
    """The workload's description, identical in both arms' lines."""
    dt, _, _, fam, k = WORKLOADS[workload]
    cfg = {"workload": workload, "points": n, "queries_per_gpu": nq, "family": fam, "k": k,
           "metric": "SquaredEuclidean", "parallelism": f"replicas{world}",
           "l2": l2_note(n, nq, 4 if dt == "f32" else 8)}
    if fam == "periodic_nearest_n_within":
        cfg.update({"radius": C5_RADIUS, "periodic_box": [1.0, 1.0, 1.0]})
    return cfg


def run_reference(args, rank, world):
    """The reference arm: the oracle (a C++ restatement of the reference's
    scalar path; the Rust crate cannot be built here), built -O3
    -march=native on this host, timed on all host threads over the same
    workload and config.  It loads nothing of the product package."""
    if rank != 0:
        return 0
    import oracle
    dtype_name, n, nq, fam, k = WORKLOADS[args.workload]
    n = args.points or n
    nq = args.queries or nq
    P, Q = make_data(args.workload, 0, n, nq)
    ot = oracle.OracleTree.build(P, L=oracle.timing_lib())
    nthreads = os.cpu_count() or 1
    # one sample size for every step: about 3 s of CPU work
    m, _, dt0 = time_cpu(ot, Q, args.workload, 3.0, nthreads)
    code, kk, extra = oracle_family(args.workload)
    times = []
    for s in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        ot.query_fixed(code, Q[:m], k=kk, threads=nthreads, **extra)
        if s >= args.warmup:
            times.append(time.perf_counter() - t0)
    val = m / statistics.median(times)
    sample = (f"{m} of the {len(Q)} queries per step, {fam}(k={k}), {nthreads} threads, "
              f"median of {args.steps} steps; the oracle (C++ restatement of the reference "
              f"scalar path) built -O3 -march=native -ffp-contract=off on this host")
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": "queries/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * statistics.median(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": dtype_name, "data": "synthetic",
            "config": config_for(args.workload, n, nq, world),
            "cpu_baseline": dict({"value": val, "unit": "queries/s", "cores": nthreads,
                                  "kind": "port", "sample": sample}, **cpu_info()),
            "e2e": {"value": val, "unit": "queries/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_tree_workload(args, workload, rank, world, steps, warmup, points=0, queries=0,
                      with_cpu=True, parity_rows=SAMPLE_ROWS):
    """One single-tree workload (C1, C2, C5): the line's fields, measured
    with the queries resident in HBM (`value`) and through host buffers
    (`e2e`), with the roofline of the dominant kernel."""
    import torch
    import kiddo_b200 as kb
    from kiddo_b200 import multi

    local = torch.cuda.current_device()
    dev = torch.device("cuda", local)
    dtype_name, n, nq, fam, k = WORKLOADS[workload]
    n = points or n
    nq = queries or nq
    P, Q = make_data(workload, rank, n, nq)
    t_host = time.perf_counter()
    tree = kb.ImmutableKdTree.new_from_slice(P)
    host_build_s = time.perf_counter() - t_host
    gtree = tree.to_gpu()
    stream = torch.cuda.current_stream(dev)
    dq = torch.from_numpy(Q).to(dev)

    def step():
        b = builder_for(gtree, dq, workload).with_engine(args.engine)
        return b.with_spatial_order(args.spatial_order).execute_gpu()

    # algorithmic bytes per query from the engine's own traversal counters,
    # which the tests hold equal to the oracle's (the reference traversal)
    sub = Q[: min(nq, 2_000_000)]
    stats = builder_for(gtree, sub, workload).traversal_stats()
    bpq = bytes_per_query(stats, len(sub), Q.itemsize, k)
    walked_bpq = None
    if fam == "periodic_nearest_n_within":
        # the periodic rows away from the box's faces are answered by the plain
        # walk (same rows, bit for bit), which touches fewer bytes than the
        # reference's periodic walk that `bpq` counts
        plain = gtree.query(sub).nearest_n(kb.SquaredEuclidean, k).within(C5_RADIUS)
        walked_bpq = bytes_per_query(plain.traversal_stats(), len(sub), Q.itemsize, k)

    with ClockSampler(local) as clk:
        clk.wait_first()
        for _ in range(warmup):
            res = step()
        torch.cuda.synchronize()
        multi.barrier()
        l0 = kb.launch_count()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
        torch.cuda.synchronize()
        ev[0].record(stream)
        for s in range(steps):
            res = step()
            ev[s + 1].record(stream)
        torch.cuda.synchronize()
        launches = kb.launch_count() - l0
    step_ms = [ev[i].elapsed_time(ev[i + 1]) for i in range(steps)]
    total_ms = sum(step_ms)
    total_ms_max = multi.max_over_ranks(total_ms)
    multi.barrier()
    # the last timed step's own output, sampled against the oracle
    check = parity_sample(tree, Q, res, workload, parity_rows) if parity_rows else None
    del res

    # end to end through the C ABI with pinned host buffers
    hq = torch.from_numpy(Q).pin_memory().numpy()
    for _ in range(max(1, warmup // 2)):
        builder_for(gtree, hq, workload).execute_gpu()
    torch.cuda.synchronize()
    multi.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e2e_steps = max(1, min(steps, 3))
    e0.record(stream)
    for _ in range(e2e_steps):
        builder_for(gtree, hq, workload).execute_gpu()
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = multi.max_over_ranks(e0.elapsed_time(e1))
    del hq

    # the same tree built on the device from device points (same bytes); the
    # call synchronizes, so it is timed on the host clock: median of 3 after one
    dP = torch.from_numpy(P).to(dev)
    builds = []
    for _ in range(4):
        torch.cuda.synchronize()
        t_dev = time.perf_counter()
        g_dev = kb.GpuTree.build(dP, stream=stream)
        torch.cuda.synchronize()
        builds.append((time.perf_counter() - t_dev) * 1e3)
        del g_dev
    device_build_ms = float(np.median(builds[1:]))
    del dP, dq

    w = k if fam in ("nearest_n", "periodic_nearest_n_within") else 1
    h2d = nq * 3 * Q.itemsize
    # per-row counts cross the bus only where they vary (nearest_n without a
    # radius has min(k, size) in every row, written on the host)
    d2h = nq * w * (Q.itemsize + 4) + (nq * 4 if w > 1 and fam != "nearest_n" else 0)
    out_bytes = nq * w * (Q.itemsize + 4) + (nq * 4 if w > 1 else 0)  # written to HBM
    value = world * nq * steps / (total_ms_max / 1e3)
    e2e_val = world * nq * e2e_steps / (e2e_ms / 1e3)
    kern_ms = total_ms / steps
    achieved = bpq * nq / (kern_ms / 1e3) / 1e9
    peak, peak_kind = measured_peaks()
    traffic = profile_traffic(workload)
    # compulsory bytes: the whole tree once, the queries once, the results once
    tree_bytes = sum(a.nbytes for a in (tree.stems(), tree.leaf_bytes(), tree.leaf_extents()))
    compulsory = tree_bytes + h2d + out_bytes
    comp_gbs = compulsory / (kern_ms / 1e3) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": world,
        "steps": steps, "warmup": warmup, "ms_per_step": total_ms_max / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": dtype_name, "data": "synthetic",
        "config": config_for(workload, n, nq, world),
        "path": {"spatial_order": "auto" if args.spatial_order is None else args.spatial_order,
                 "engine": args.engine or "auto"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "bytes_per_query": bpq,
                     "traffic": (traffic or {}).get("dram_bytes_per_launch"),
                     "compulsory": {"bytes": int(compulsory), "achieved": comp_gbs,
                                    "frac": comp_gbs / peak},
                     "kernel": kernel_name(fam, args.engine)},
        "e2e": {"value": e2e_val, "unit": "queries/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
        "tree_build": {"host_s": host_build_s, "host_threads": os.cpu_count(),
                       "device_ms": device_build_ms},
        "traversal_per_query": {"stems": float(stats[0]) / len(sub),
                                "leaves": float(stats[1]) / len(sub),
                                "points": float(stats[2]) / len(sub)},
        "step_ms": step_ms,
    }
    if check is not None:
        line["parity_sample"] = check
    if walked_bpq is not None:
        walked = walked_bpq * nq / (kern_ms / 1e3) / 1e9
        line["roofline"]["walked"] = {
            "bytes_per_query": walked_bpq, "achieved": walked, "frac": walked / peak,
            "note": "bytes of the plain walk that answers the rows away from the box's faces "
                    "(the rest, a few percent, take the periodic walk); bytes_per_query above "
                    "counts the reference's periodic walk"}
    if rank == 0 and world == 1 and with_cpu:
        line["cpu_baseline"] = cpu_baseline(tree, Q, workload)
    del gtree, tree
    return line


# the other configurations, measured in the same run as the headline (one
# GPU): their own lines' main fields, as sub-objects of the headline line
SUB_KEYS = ("value", "unit", "ms_per_step", "steps", "warmup", "dtype", "config", "roofline",
            "e2e", "gpu_launches", "clocks", "parity_sample", "cpu_baseline",
            "traversal_per_query")


def _free_device():
    import gc
    import torch
    gc.collect()
    torch.cuda.synchronize()
    torch.cuda.empty_cache()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c2_knn16", choices=sorted(WORKLOADS))
    ap.add_argument("--scale", type=float, default=1.0,
                    help="scale the c3/c4 workloads (tests and profiling only)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--headline-only", action="store_true",
                    help="measure the chosen workload alone, without the other configurations")
    ap.add_argument("--no-parity-sample", action="store_true")
    ap.add_argument("--spatial-order", default=None, action="store_true",
                    help="force leaf-grouped processing (default: the library decides)")
    ap.add_argument("--no-spatial-order", dest="spatial_order", action="store_false")
    ap.add_argument("--engine", default=None, choices=["warp", "thread", "coop"],
                    help="force the kernel variant (default: the library chooses)")
    ap.add_argument("--points", type=int, default=0, help="override the tree size (profiling)")
    ap.add_argument("--queries", type=int, default=0, help="override the batch size (profiling)")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.workload == "c3_forest":
        return run_forest(args, rank, world)
    if args.workload == "c4_chamfer":
        return run_chamfer(args, rank, world)

    import torch
    import torch.distributed as dist
    from kiddo_b200 import multi

    torch.cuda.set_device(local)
    if world > 1:
        multi.init_process_group("nccl")
    parity_rows = 0 if args.no_parity_sample else SAMPLE_ROWS
    line = run_tree_workload(args, args.workload, rank, world, args.steps, args.warmup,
                             args.points, args.queries, not args.no_cpu_baseline, parity_rows)
    full = (args.workload == "c2_knn16" and world == 1 and not args.headline_only
            and not (args.points or args.queries))
    if full:
        # every term of the metric in the one run: approx and the f64
        # configurations on single trees, the batched-vs-per-tree forest, and
        # Chamfer forward + backward
        sub_steps, sub_warm = max(1, min(args.steps, 10)), max(3, min(args.warmup, 5))
        for wl in ("c2_approx", "c1_nn1", "c5_periodic"):
            _free_device()
            sub = run_tree_workload(args, wl, rank, world, sub_steps, sub_warm,
                                    with_cpu=not args.no_cpu_baseline, parity_rows=parity_rows)
            line[wl] = {k: sub[k] for k in SUB_KEYS if k in sub}
        _free_device()
        fa = argparse.Namespace(**vars(args))
        fa.steps, fa.warmup = sub_steps, sub_warm
        line["c3_batched_vs_per_tree"] = forest_measure(fa, rank, world, parity_rows)
        _free_device()
        line["c4_chamfer"] = chamfer_measure(fa, rank, world)
        line["gpu_launches_all_workloads"] = line["gpu_launches"] + sum(
            line[w].get("gpu_launches", 0) for w in ("c2_approx", "c1_nn1", "c5_periodic",
                                                     "c3_batched_vs_per_tree", "c4_chamfer"))
    if rank == 0:
        print(json.dumps(line), flush=True)
    multi.barrier()
    if world > 1:
        dist.destroy_process_group()
    return 0


# ---------------------------------------------------------------------------
# Batches over many trees: 256 catalogues of unit vectors, mixed radius queries
# ---------------------------------------------------------------------------
def sphere_catalogue(n, rng, clumps=32, kappa=1e5, clumped=0.3):
    """Unit vectors: uniform directions, 30% of them in von Mises-Fisher clumps
    (kappa = 1e5, drawn as tangent-plane Gaussians of sigma 1/sqrt(kappa))."""
    v = rng.normal(size=(n, 3))
    nc = int(n * clumped)
    if nc:
        mu = rng.normal(size=(clumps, 3))
        mu /= np.linalg.norm(mu, axis=1, keepdims=True)
        lab = rng.integers(0, clumps, nc)
        v[:nc] = mu[lab] + rng.normal(0, 1 / np.sqrt(kappa), (nc, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return v[rng.permutation(n)].astype(np.float32)


def pareto_ranks(n, rng):
    """u32 rank of a Pareto(alpha=1.5) weight (0 = heaviest); unique per tree."""
    w = rng.pareto(1.5, n)
    r = np.empty(n, dtype=np.uint32)
    r[np.argsort(-w, kind="stable")] = np.arange(n, dtype=np.uint32)
    return r


def forest_workload(scale, seed=3):
    rng = np.random.default_rng(seed)
    n_trees = 256
    sizes = np.exp(rng.uniform(np.log(1e4), np.log(4e6), n_trees))
    sizes = np.maximum((sizes * (120e6 * scale) / sizes.sum()).astype(np.int64), 32)
    n_q = int(64e6 * scale)
    share = rng.dirichlet(np.full(n_trees, 0.5))
    per_tree = np.floor(share * n_q).astype(np.int64)
    per_tree[0] += n_q - per_tree.sum()

    def one_tree(t):
        # every tree draws from its own seeded generator, so the threads give
        # the same arrays in any order
        trng = np.random.default_rng(seed * 1000 + t)
        p = sphere_catalogue(int(sizes[t]), trng)
        it = pareto_ranks(int(sizes[t]), trng)
        return p, it, sphere_catalogue(int(per_tree[t]), trng)

    import concurrent.futures as cf
    with cf.ThreadPoolExecutor(max_workers=min(16, os.cpu_count() or 1)) as ex:
        parts = list(ex.map(one_tree, range(n_trees)))
    pts = [p for p, _, _ in parts]
    items = [it for _, it, _ in parts]
    qs = [q for _, _, q in parts]
    tree_of = np.repeat(np.arange(n_trees, dtype=np.int32), per_tree)
    Q = np.concatenate(qs)
    chord = np.exp(rng.uniform(np.log(1e-4), np.log(1e-2), n_q))
    radii = (chord * chord).astype(np.float32)  # SquaredEuclidean radius
    family = rng.integers(0, 3, n_q)  # 0 within sorted, 1 within unsorted, 2 best_n_within(5)
    return pts, items, Q, tree_of, radii, family


def forest_parity_sample(trees, parts, results, n=SAMPLE_ROWS, seed=0):
    """Sampled rows of each family's batched result against the oracle tree
    of the query's catalogue (checker build, the same layouts), bit for bit."""
    import oracle
    import torch
    rng = np.random.default_rng(seed)
    mism, total = 0, 0
    ots = {}

    def ot(t):
        if t not in ots:
            tr = trees[t]
            ots[t] = oracle.OracleTree.from_layout(oracle.Layout(
                tr.dtype, tr.dims, tr.stems(), tr.leaf_bytes(), tr.leaf_extents(),
                tr.max_stem_level(), tr.size(), tr.max_leaf_len()))
        return ots[t]

    for fam, ((q, _, r, host_t), res) in enumerate(zip(parts, results)):
        nq = q.shape[0]
        if nq == 0:
            continue
        rows = np.sort(rng.choice(nq, size=min(n // 3, nq), replace=False))
        sel = torch.from_numpy(rows).to(q.device)
        qh = q.index_select(0, sel).cpu().numpy()
        rh = r.index_select(0, sel).cpu().numpy()
        idx = sel
        if fam < 2:
            # every sampled row's hits in one gather: row j at [goff[j], goff[j + 1])
            off = res.offsets.cpu().numpy().astype(np.int64)
            lens = off[rows + 1] - off[rows]
            goff = np.concatenate([[0], np.cumsum(lens)])
            hit = np.repeat(off[rows] - goff[:-1], lens) + np.arange(goff[-1])
            th = torch.from_numpy(hit).to(q.device)
            gd = res.distances.index_select(0, th).cpu().numpy()
            gi = res.items.index_select(0, th).cpu().numpy().view(np.uint32)
        else:
            gd = res.distances.index_select(0, idx).cpu().numpy()
            gi = res.items.index_select(0, idx).cpu().numpy().view(np.uint32)
            gc = res.counts.index_select(0, idx).cpu().numpy()
        tof = host_t[rows]
        for t in np.unique(tof):
            m = np.nonzero(tof == t)[0]
            if fam < 2:
                oo, od, oi = ot(int(t)).within(qh[m], rh[m], sorted=(fam == 0))
                for j, p in enumerate(m):
                    a, b = goff[p], goff[p + 1]
                    oa, ob = int(oo[j]), int(oo[j + 1])
                    ok = (b - a) == (ob - oa) and np.array_equal(gd[a:b], od[oa:ob]) and \
                        np.array_equal(gi[a:b], oi[oa:ob])
                    mism += int(not ok)
            else:
                od, oi, oc = ot(int(t)).best_n_within(qh[m], rh[m], 5)
                same = (np.all(gd[m] == od, axis=1) & np.all(gi[m] == oi, axis=1) &
                        (gc[m].astype(np.uint32) == oc))
                mism += int((~same).sum())
            total += len(m)
    return {"n": int(total), "mismatches": int(mism),
            "rule": "bit-exact CSR rows / best_n rows against the oracle, seeded rows per family"}


def forest_measure(args, rank, world, parity_rows=SAMPLE_ROWS):
    """One job of 256 catalogues and 64M queries, batched (one persistent
    launch per family) and per tree (one launch per tree and family).  With
    N > 1 GPUs every tree has one owner rank (multi.partition_trees on points x
    queries) that holds it and answers its queries (strong scaling: the job is
    fixed); the time is the max over ranks.  Returns the measured fields on
    rank 0 (None elsewhere)."""
    import torch
    import kiddo_b200 as kb
    from kiddo_b200 import multi
    pts, items, Q, tree_of, radii, family = forest_workload(args.scale)
    nq_total = len(Q)
    if world > 1:
        counts = np.bincount(tree_of, minlength=len(pts))
        owner = np.asarray(multi.partition_trees([len(p) * max(int(c), 1) for p, c in
                                                  zip(pts, counts)], world))
        mine = np.nonzero(owner == rank)[0]
        local = np.full(len(pts), -1, np.int64)
        local[mine] = np.arange(len(mine))
        keep = owner[tree_of] == rank
        Q, radii, family = Q[keep], radii[keep], family[keep]
        tree_of = local[tree_of[keep]].astype(np.int32)
        pts = [pts[i] for i in mine]
        items = [items[i] for i in mine]
    n_points = int(sum(len(p) for p in pts))
    trees = [kb.ImmutableKdTree.new_from_entries(it, p) for it, p in zip(items, pts)]
    del pts, items
    forest = kb.Forest(trees)
    stream = torch.cuda.Stream()
    parts = []
    for fam in range(3):
        sel = np.nonzero(family == fam)[0]  # queries stay grouped by tree
        parts.append((torch.from_numpy(Q[sel]).cuda(), torch.from_numpy(tree_of[sel]).cuda(),
                      torch.from_numpy(radii[sel]).cuda(), tree_of[sel]))
    del Q
    SE = kb.SquaredEuclidean

    def builders(q, t, r):
        return [forest.query(q, t, r).within(SE, 0.0).on_stream(stream),
                forest.query(q, t, r).within(SE, 0.0).unsorted().on_stream(stream),
                forest.query(q, t, r).best_n_within(SE, 0.0, 5).on_stream(stream)]

    def batched():
        out = []
        for fam, (q, t, r, _) in enumerate(parts):
            out.append(builders(q, t, r)[fam].execute_gpu())
        return out

    def per_tree():
        for fam, (q, t, r, host_t) in enumerate(parts):
            cuts = np.searchsorted(host_t, np.arange(len(trees) + 1))
            for a, b in zip(cuts[:-1], cuts[1:]):
                if b > a:
                    builders(q[a:b], t[a:b], r[a:b])[fam].execute_gpu()

    with torch.cuda.stream(stream):
        res = batched()
        torch.cuda.synchronize()
        hits = [int(x.offsets[-1].item()) for x in res[:2]]
        check = forest_parity_sample(trees, parts, res, parity_rows) if parity_rows else None
        del res

        def timed(fn, steps):
            for _ in range(args.warmup):
                fn()
            torch.cuda.synchronize()
            multi.barrier()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(steps):
                fn()
            e1.record(stream)
            torch.cuda.synchronize()
            return multi.max_over_ranks(e0.elapsed_time(e1) / steps)

        l0 = kb.launch_count()
        ms_batched = timed(batched, args.steps)
        launches = (kb.launch_count() - l0) // (args.warmup + args.steps)
        per_tree_steps = max(1, args.steps // 2)
        ms_per_tree = timed(per_tree, per_tree_steps)
    hits = [int(multi.fixed_order_sum(torch.tensor([h], dtype=torch.float64,
                                                   device="cuda"))[0].item()) for h in hits]
    del parts, forest, trees
    if rank != 0:
        return None
    out = {"value": nq_total / (ms_batched / 1e3), "unit": "queries/s",
           "ms_per_step": ms_batched, "steps": args.steps, "warmup": args.warmup,
           "config": {"workload": "c3_forest", "trees": 256, "points": n_points,
                      "queries": nq_total,
                      "families": "within sorted / within unsorted / best_n_within(5), thirds",
                      "radii": "chord log-uniform [1e-4, 1e-2], squared",
                      "hits": {"within_sorted": hits[0], "within_unsorted": hits[1]}},
           "per_tree_launch": {"ms_per_step": ms_per_tree, "steps": per_tree_steps,
                               "value": nq_total / (ms_per_tree / 1e3)},
           "batched_over_per_tree": ms_per_tree / ms_batched,
           "gpu_launches": int(launches)}
    if check is not None:
        out["parity_sample"] = check
    return out


def run_forest(args, rank, world):
    """The forest configuration as its own line (``--workload c3_forest``)."""
    import torch
    from kiddo_b200 import multi
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    if world > 1:
        multi.init_process_group("nccl")
    local = torch.cuda.current_device()
    with ClockSampler(local) as clk:
        clk.wait_first()
        m = forest_measure(args, rank, world,
                           0 if getattr(args, "no_parity_sample", False) else SAMPLE_ROWS)
    if rank == 0:
        line = {"metric": METRIC, "n_gpus": world, "higher_is_better": True,
                "scaling": "strong" if world > 1 else "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic"}
        line.update(m)
        line["clocks"] = clk.summary()
        if world > 1:
            line["config"]["parallelism"] = f"trees partitioned over {world} ranks"
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        multi.barrier()
        dist.destroy_process_group()
    return 0


# ---------------------------------------------------------------------------
# Chamfer forward + backward over a batch of 64 cloud pairs
# ---------------------------------------------------------------------------
def chamfer_workload(scale, seed=4):
    rng = np.random.default_rng(seed)
    pairs = []
    for p in range(64):
        n = int(np.exp(rng.uniform(np.log(1e4), np.log(1e6))) * scale) + 16
        kind = "plane" if p % 2 == 0 else "sphere"
        rot, _ = np.linalg.qr(rng.normal(size=(3, 3)))  # one orientation per pair

        def cloud(m):
            if kind == "plane":
                c = np.c_[rng.uniform(-0.5, 0.5, (m, 2)), np.zeros(m)]
            else:
                v = rng.normal(size=(m, 3))
                c = 0.5 * v / np.linalg.norm(v, axis=1, keepdims=True)
            return (c @ rot + rng.normal(0, 0.001, (m, 3))).astype(np.float32)
        pairs.append((cloud(n), cloud(4 * n)))
    return pairs


def chamfer_measure(args, rank, world):
    """Forward + backward over 64 cloud pairs at k = 8 and k = 1.  With N > 1
    GPUs every pair has one owner rank (multi.partition_trees on source x
    target sizes); a pair's gradients stay on its owner and the loss partials
    are added in rank order (multi.fixed_order_sum), so the job is fixed
    (strong scaling).  Returns the measured fields on rank 0 (None elsewhere)."""
    import torch
    import kiddo_b200 as kb
    from kiddo_b200 import multi
    from kiddo_b200.chamfer import chamfer_backward, chamfer_forward
    pairs = chamfer_workload(args.scale)
    n_src_total = sum(len(s) for s, _ in pairs)
    n_tgt_total = sum(len(t) for _, t in pairs)
    if world > 1:
        owner = multi.partition_trees([len(s) * 5.0 for s, _ in pairs], world)
        pairs = [pr for pr, o in zip(pairs, owner) if o == rank]
    trees = [kb.ImmutableKdTree.new_from_slice(t) for _, t in pairs]
    forest = kb.Forest(trees)
    src = torch.from_numpy(np.concatenate([s for s, _ in pairs])).cuda()
    tgt = torch.from_numpy(np.concatenate([t for _, t in pairs])).cuda()
    tree_of = torch.from_numpy(np.concatenate(
        [np.full(len(s), i, np.int32) for i, (s, _) in enumerate(pairs)])).cuda()
    base = torch.from_numpy(np.cumsum([0] + [len(t) for _, t in pairs[:-1]]).astype(np.int64)).cuda()
    out = {}
    for k in (8, 1):
        def step():
            loss, ctx = chamfer_forward(forest, src, tgt, k, 0.01, tree_of, base)
            grads = chamfer_backward(ctx)
            return multi.fixed_order_sum(loss), grads
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        multi.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        l0 = kb.launch_count()
        e0.record()
        for _ in range(args.steps):
            step()
        e1.record()
        torch.cuda.synchronize()
        ms = multi.max_over_ranks(e0.elapsed_time(e1) / args.steps)
        out[k] = (ms, (kb.launch_count() - l0) // args.steps)
    del forest, trees, src, tgt
    if rank != 0:
        return None
    ms8 = out[8][0]
    return {"value": 64 / (ms8 / 1e3), "unit": "cloud pairs/s (fwd+bwd)", "ms_per_step": ms8,
            "steps": args.steps, "warmup": args.warmup,
            "config": {"workload": "c4_chamfer", "pairs": 64, "k": 8, "sigma": 0.01,
                       "source_points": int(n_src_total), "target_points": int(n_tgt_total)},
            "k1": {"ms_per_step": out[1][0], "value": 64 / (out[1][0] / 1e3)},
            "gpu_launches": int(out[8][1])}


def run_chamfer(args, rank, world):
    """The Chamfer configuration as its own line (``--workload c4_chamfer``)."""
    import torch
    from kiddo_b200 import multi
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    if world > 1:
        multi.init_process_group("nccl")
    with ClockSampler(torch.cuda.current_device()) as clk:
        clk.wait_first()
        m = chamfer_measure(args, rank, world)
    if rank == 0:
        line = {"metric": METRIC, "n_gpus": world, "higher_is_better": True,
                "scaling": "strong" if world > 1 else "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic"}
        line.update(m)
        line["clocks"] = clk.summary()
        if world > 1:
            line["config"]["parallelism"] = f"cloud pairs partitioned over {world} ranks"
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        multi.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
