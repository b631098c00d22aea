"""Autotuner for the query kernels.

Every knob it turns leaves results bit-identical, so it only ever measures
time.  For a (GPU, dtype, dims, family, metric, k, tree-size) key it times, on
a sample of the caller's own batch:

* the engine: one warp per query (lanes scan a leaf side by side, per-level
  continuation records in lane registers) or one thread per query
  (continuation slots and the k-list in shared memory);
* the processing order: as given, or bucketed by each query's straight-descent
  leaf (KGPU_FLAG_SPATIAL_ORDER).

The winner is cached in a JSON file (``KIDDO_B200_TUNE_CACHE`` or
``~/.cache/kiddo_b200/autotune.json``) and applied by
``QueryBuilder.autotuned()``.
"""
from __future__ import annotations

import json
import math
import os
import threading

_LOCK = threading.Lock()
CANDIDATES = [("thread", True), ("thread", False), ("warp", True), ("warp", False)]


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


def tune(builder, sample: int = 1 << 20, repeats: int = 3):
    """Time every candidate on up to `sample` queries of the batch; cache and
    return the best (engine, spatial_order)."""
    import torch
    q = builder.queries
    n = q.shape[0]
    sub = q[: min(n, sample)]
    best, best_ms = None, float("inf")
    timings = {}
    for engine, order in CANDIDATES:
        b = _clone(builder, sub).with_engine(engine).with_spatial_order(order)
        b.execute_gpu()  # warm up (first launch, allocator)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(repeats):
            b.execute_gpu()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / repeats
        timings[f"{engine},{int(order)}"] = ms
        if ms < best_ms:
            best, best_ms = (engine, order), ms
    with _LOCK:
        db = _load()
        db[key_for(builder)] = {"engine": best[0], "spatial_order": best[1], "ms": timings,
                                "sample": int(sub.shape[0])}
        _store(db)
    return best


def lookup(builder):
    entry = _load().get(key_for(builder))
    if entry is None:
        return None
    return entry["engine"], bool(entry["spatial_order"])


def _clone(builder, queries):
    b = type(builder).__new__(type(builder))
    b.__dict__.update(builder.__dict__)
    b.queries = queries
    return b
