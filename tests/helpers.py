"""Shared test helpers: fixtures, data generators and the reference's parity rules."""
from __future__ import annotations

import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "kats.json")


def load_kats():
    with open(GOLDEN) as f:
        kats = json.load(f)["kats"]
    for k in kats:
        dt = np.float64 if k["dtype"] == "f64" else np.float32
        if k["name"].startswith("tile_boundary_"):
            # src/kd_tree/query/within.rs:143-183: coordinates computed in f32
            n = len(k["points"])
            i = np.arange(n)
            k["np_points"] = np.stack([
                ((i * 5) % 97).astype(np.float32) / np.float32(97.0),
                ((i * 13 + 1) % 97).astype(np.float32) / np.float32(97.0),
                ((i * 23 + 2) % 97).astype(np.float32) / np.float32(97.0)], axis=1)
        else:
            k["np_points"] = np.asarray(k["points"], dtype=dt).reshape(len(k["points"]), -1)
        k["np_items"] = None if k["items"] is None else np.asarray(k["items"], dtype=np.uint32)
    return kats


def brute_dists(points, q, metric="sqeuclidean"):
    """Per-point distance with the reference's accumulation order."""
    import oracle
    return oracle.scan_dists(points, q, metric)


def gaussian_mixture(n, centres, sigma, background_frac, rng, dtype=np.float32):
    """Points of the C2 workload shape: a mixture of isotropic Gaussians with
    Dirichlet(1) weights plus a uniform background, in [0, 1)^3."""
    c = rng.random((centres, 3))
    w = rng.dirichlet(np.ones(centres))
    nb = int(round(n * background_frac))
    nm = n - nb
    lab = rng.choice(centres, size=nm, p=w)
    pts = c[lab] + rng.normal(0.0, sigma, size=(nm, 3))
    pts = np.concatenate([pts, rng.random((nb, 3))], axis=0)
    rng.shuffle(pts, axis=0)
    return pts.astype(dtype)


def assert_same_fixed(gd, gi, gc, od, oi, oc, label=""):
    """Bit-exact equality of dense (distance, item, count) outputs."""
    gd = np.asarray(gd)
    od = np.asarray(od)
    assert gd.shape == od.shape, label
    assert np.array_equal(np.asarray(gc).astype(np.int64), np.asarray(oc).astype(np.int64)), \
        f"{label}: counts differ"
    bad = ~((gd == od) | (np.isnan(gd) & np.isnan(od)))
    assert not bad.any(), f"{label}: {bad.sum()} distances differ, first at {np.argwhere(bad)[:3]}"
    gi = np.asarray(gi).astype(np.uint32)
    oi = np.asarray(oi).astype(np.uint32)
    badi = gi != oi
    assert not badi.any(), f"{label}: {badi.sum()} items differ, first at {np.argwhere(badi)[:3]}"


def assert_same_csr(g, o, label=""):
    go, gd, gi = (np.asarray(x) for x in g)
    oo, od, oi = (np.asarray(x) for x in o)
    assert np.array_equal(go.astype(np.int64), oo.astype(np.int64)), f"{label}: offsets differ"
    assert np.array_equal(gd, od), f"{label}: distances differ"
    assert np.array_equal(gi.astype(np.uint32), oi.astype(np.uint32)), f"{label}: items differ"


def ulps_apart(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    it = np.int64 if a.dtype == np.float64 else np.int32
    ia = a.view(it).astype(np.int64)
    ib = b.view(it).astype(np.int64)
    return np.abs(ia - ib)


def compare_nearest_n_reference_rule(dists, items, exp_d, exp_i, k):
    """tests/kd_tree_fuzz_v6.rs:272-340: distances within 4 ULP; equal-distance
    groups compared as item multisets except the tail group at the cut."""
    assert len(dists) == len(exp_d)
    assert np.all(ulps_apart(np.asarray(dists), np.asarray(exp_d)) <= 4)
    d = np.asarray(dists)
    tail = d[-1] if len(d) else None
    groups = {}
    for dd, ii in zip(d, items):
        groups.setdefault(float(dd), []).append(int(ii))
    egroups = {}
    for dd, ii in zip(exp_d, exp_i):
        egroups.setdefault(float(dd), []).append(int(ii))
    for key, lst in groups.items():
        if tail is not None and key == float(tail) and len(d) == k:
            assert len(lst) == len(egroups.get(key, []))
            continue
        assert sorted(lst) == sorted(egroups.get(key, [])), key


def flatvec_parts(tree):
    """The FlatVec form (src/leaf_strategy/flat_vec.rs:20-26, 189-210) of a
    host ImmutableKdTree: K point columns, items and (start, end) extents,
    read off its VecOfArenas tiles leaf by leaf."""
    K = tree.dims
    dt = np.dtype(tree.dtype)
    lb = tree.leaf_bytes()
    ex = tree.leaf_extents()
    cols = [[] for _ in range(K)]
    items = []
    extents = []
    start = 0
    for off, ln in ex:
        off, ln = int(off), int(ln)
        rem, pos = ln, off
        while rem:
            w = next(t for t in (32, 8, 4, 2, 1) if rem >= t)
            for d in range(K):
                cols[d].append(np.frombuffer(lb, dtype=dt, count=w, offset=pos + d * w * dt.itemsize))
            items.append(np.frombuffer(lb, dtype=np.uint32, count=w, offset=pos + K * w * dt.itemsize))
            pos += w * (K * dt.itemsize + 4)
            rem -= w
        extents.append((start, start + ln))
        start += ln
    cols = [np.concatenate(c) if c else np.zeros(0, dt) for c in cols]
    items = np.concatenate(items) if items else np.zeros(0, np.uint32)
    return cols, items, np.asarray(extents, dtype=np.uint32).reshape(-1, 2)


def vecofarrays_parts(tree, bucket=32):
    """The VecOfArrays form (src/leaf_strategy/vec_of_arrays.rs:51-97,
    append_leaf :249-275) of a host ImmutableKdTree: per leaf, content_points
    [K, B] and content_items [B] with the live entries first (zeros after) and
    the live-entry count."""
    cols, items, ext = flatvec_parts(tree)
    K = tree.dims
    L = ext.shape[0]
    pts = np.zeros((L, K, bucket), dtype=np.dtype(tree.dtype))
    its = np.zeros((L, bucket), dtype=np.uint32)
    sizes = np.zeros(L, dtype=np.uint64)
    for l, (a, b) in enumerate(ext):
        a, b = int(a), int(b)
        for d in range(K):
            pts[l, d, :b - a] = cols[d][a:b]
        its[l, :b - a] = items[a:b]
        sizes[l] = b - a
    return pts, its, sizes
