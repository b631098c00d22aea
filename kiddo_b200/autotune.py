"""Autotuner for the query kernels.

Every knob it turns leaves results bit-identical, so it only ever measures
time.  For a (GPU, dtype, dims, family, metric, k, tree-size, periodic) key it
times, on a sample of the caller's own batch, in three stages (each stage
keeps the best choice of the ones before it):

1. the engine and the processing order:
   * one warp per query (lanes scan a leaf side by side, per-level
     continuation records in lane registers), one thread per query
     (continuation slots and the k-list in shared memory), or, for sorted
     nearest_n up to 32 entries, per-thread walks whose leaves the whole warp
     scans (each leaf's rows loaded once, coalesced: the staged-leaf form);
   * the queries as given, or bucketed by their straight-descent leaf
     (KGPU_FLAG_SPATIAL_ORDER);
2. the lane refill threshold of the per-thread engines: how many of a warp's
   lanes must be idle before they take new queries (8, 16, 24, 32);
3. the queries handed to a warp at a time (32, 64, 128, 256).

The winner is cached in a JSON file (``KIDDO_B200_TUNE_CACHE`` or
``~/.cache/kiddo_b200/autotune.json``) and applied by
``QueryBuilder.autotuned()``.  The reference's own benchmark sweeps the
analogous knobs of its CPU path per dimensionality and query family
(benches/v6_codspeed_queries.rs:51-70).
"""
from __future__ import annotations

import json
import math
import os
import threading

_LOCK = threading.Lock()
REFILLS = (8, 16, 24, 32)
CHUNKS = (32, 64, 128, 256)


def cache_path() -> str:
    p = os.environ.get("KIDDO_B200_TUNE_CACHE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "kiddo_b200", "autotune.json")


def _load():
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except Exception:
        return {}


def _store(db):
    path = cache_path()
    os.makedirs(os.path.dirname(path), exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(db, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def key_for(builder) -> str:
    import torch
    tree = builder.tree
    dev = torch.cuda.get_device_name() if torch.cuda.is_available() else "cpu"
    size = tree.size() if hasattr(tree, "size") else 0
    size_bucket = int(math.log2(max(size, 1))) // 2 * 2
    k = builder.max_qty if builder.max_qty else 1
    return "|".join(str(x) for x in (dev, tree.dtype, tree.dims, builder.family, builder.metric,
                                     k, size_bucket, builder.box is not None))


def engines_for(builder):
    """The engines that serve this query (the cooperative scan for sorted
    nearest_n with k <= 32, Cartesian)."""
    from . import _capi as C
    out = ["thread", "warp"]
    if (builder.family in (C.NEAREST_N, C.NEAREST_N_WITHIN) and builder.sorted
            and builder.max_qty <= 32 and builder.box is None):
        out.append("coop")
    return out


def _time(builder, sub, repeats, engine, order, refill, chunk):
    import torch
    b = _clone(builder, sub).with_engine(engine).with_spatial_order(order)
    b.with_tuning(refill, chunk)
    b.execute_gpu()  # warm up (first launch, allocator)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(repeats):
        b.execute_gpu()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / repeats


def tune(builder, sample: int = 1 << 20, repeats: int = 3):
    """Time the candidates on up to `sample` queries of the batch, stage by
    stage; cache and return the best {engine, spatial_order, refill, chunk}."""
    q = builder.queries
    sub = q[: min(q.shape[0], sample)]
    timings = {}
    best = None
    for engine in engines_for(builder):
        for order in (True, False):
            ms = _time(builder, sub, repeats, engine, order, None, None)
            timings[f"{engine},{int(order)}"] = ms
            if best is None or ms < best[0]:
                best = (ms, engine, order, None, None)
    ms0, engine, order, _, _ = best
    refill = chunk = None
    if engine != "warp":  # the per-thread engines refill lanes
        for r in REFILLS:
            ms = _time(builder, sub, repeats, engine, order, r, None)
            timings[f"{engine},{int(order)},refill={r}"] = ms
            if ms < best[0]:
                best = (ms, engine, order, r, None)
        refill = best[3]
    for c in CHUNKS:
        ms = _time(builder, sub, repeats, engine, order, refill, c)
        timings[f"{engine},{int(order)},refill={refill},chunk={c}"] = ms
        if ms < best[0]:
            best = (ms, engine, order, refill, c)
    choice = {"engine": best[1], "spatial_order": bool(best[2]), "refill": best[3],
              "chunk": best[4]}
    with _LOCK:
        db = _load()
        db[key_for(builder)] = dict(choice, ms=timings, sample=int(sub.shape[0]))
        _store(db)
    return choice


def lookup(builder):
    entry = _load().get(key_for(builder))
    if entry is None or "engine" not in entry:
        return None
    return {"engine": entry["engine"], "spatial_order": bool(entry["spatial_order"]),
            "refill": entry.get("refill"), "chunk": entry.get("chunk")}


def _clone(builder, queries):
    b = type(builder).__new__(type(builder))
    b.__dict__.update(builder.__dict__)
    b.queries = queries
    return b
