"""CPU oracle for kiddo's ImmutableKdTree query path (test infrastructure).

This package is the checker: a C++ restatement of the reference's construction
and scalar query path (see kiddo_oracle.hpp for the file:line map), wrapped with
ctypes.  Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline /
reference legs may import it; the product package ``kiddo_b200`` never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libkiddo_oracle.so")
_TIMING_PATH = os.path.join(_HERE, "libkiddo_oracle_timing.so")
_TIMING_STAMP = _TIMING_PATH + ".host"
_lib = None
_timing_lib = None

FAM_NEAREST_ONE = 0
FAM_APPROX = 1
FAM_NEAREST_N = 2
FAM_BEST_N_WITHIN = 3
FAM_PERIODIC_NEAREST_ONE = 4
FAM_PERIODIC_NEAREST_N = 5
FAM_WITHIN = 10
FAM_PERIODIC_WITHIN = 11

METRICS = {"sqeuclidean": 0, "manhattan": 1, "chebyshev": 2, "minkowski3": 3, "minkowski4": 4}


def build_library(force: bool = False) -> str:
    """Compile the oracle with its Makefile (g++, -ffp-contract=off)."""
    src = os.path.join(_HERE, "kiddo_oracle_capi.cpp")
    hdr = os.path.join(_HERE, "kiddo_oracle.hpp")
    stale = (not os.path.exists(_LIB_PATH)) or force or any(
        os.path.getmtime(p) > os.path.getmtime(_LIB_PATH) for p in (src, hdr))
    if stale:
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def host_cpu():
    """(CPU model name, logical CPUs, physical cores) of this host."""
    model, cores = "unknown", set()
    try:
        with open("/proc/cpuinfo") as f:
            phys = core = None
            for line in f:
                k, _, v = line.partition(":")
                k, v = k.strip(), v.strip()
                if k == "model name":
                    model = v
                elif k == "physical id":
                    phys = v
                elif k == "core id":
                    core = v
                elif not k and phys is not None:
                    cores.add((phys, core))
                    phys = core = None
            if phys is not None:
                cores.add((phys, core))
    except OSError:
        pass
    logical = os.cpu_count() or 1
    return model, logical, len(cores) or logical


def timing_lib():
    """The timed CPU baseline: the oracle's source built -O3 -march=native for
    THIS host (``make timing``), 3-D SquaredEuclidean trees only.  It is
    rebuilt when the library was built on another CPU model, so the
    instructions it uses always exist here.  Same API as ``lib()``."""
    global _timing_lib
    if _timing_lib is None:
        model = host_cpu()[0]
        src = [os.path.join(_HERE, f) for f in ("kiddo_oracle_capi.cpp", "kiddo_oracle.hpp")]
        stamp = None
        if os.path.exists(_TIMING_STAMP):
            with open(_TIMING_STAMP) as f:
                stamp = f.read().strip()
        if (stamp != model or not os.path.exists(_TIMING_PATH)
                or any(os.path.getmtime(p) > os.path.getmtime(_TIMING_PATH) for p in src)):
            subprocess.run(["make", "-s", "-C", _HERE, "timing"], check=True)
            with open(_TIMING_STAMP, "w") as f:
                f.write(model + "\n")
        _timing_lib = _declare(ctypes.CDLL(_TIMING_PATH))
    return _timing_lib


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build_library()
        _lib = _declare(ctypes.CDLL(_LIB_PATH))
    return _lib


def _declare(L):
    """ctypes signatures of the oracle's C API on library ``L``."""
    vp, u64, i32 = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int
    L.kor_build.restype = vp
    L.kor_build.argtypes = [i32, i32, vp, vp, u64]
    L.kor_build_ex.restype = vp
    L.kor_build_ex.argtypes = [i32, i32, vp, vp, u64, ctypes.c_uint32]
    L.kor_from_layout.restype = vp
    L.kor_from_layout.argtypes = [i32, i32, vp, u64, vp, u64, vp, u64, ctypes.c_int32, u64, u64]
    L.kor_from_layout_ex.restype = vp
    L.kor_from_layout_ex.argtypes = [i32, i32, vp, u64, vp, u64, vp, u64, ctypes.c_int32, u64,
                                     u64, ctypes.c_uint32]
    L.kor_free.argtypes = [vp]
    L.kor_build_mapped.restype = vp
    L.kor_build_mapped.argtypes = [i32, i32, vp, vp, u64, ctypes.c_uint32, i32, u64]
    L.kor_leaf_map_info.argtypes = [vp, vp]
    L.kor_copy_leaf_map.argtypes = [vp, vp]
    L.kor_set_leaf_map.argtypes = [vp, vp, u64, u64]
    L.kor_iter.argtypes = [vp, vp, vp]
    L.kor_layout_info.argtypes = [vp, vp]
    L.kor_copy_layout.argtypes = [vp, vp, vp, vp]
    L.kor_query_fixed.restype = i32
    L.kor_query_fixed.argtypes = [vp, i32, i32, vp, u64, ctypes.c_uint32, ctypes.c_double,
                                  i32, i32, vp, vp, vp, vp, i32, vp]
    L.kor_query_radius.restype = vp
    L.kor_query_radius.argtypes = [vp, i32, i32, vp, u64, ctypes.c_double, i32, i32, vp, i32, vp]
    L.kor_query_fixed_r.restype = i32
    L.kor_query_fixed_r.argtypes = [vp, i32, i32, vp, u64, ctypes.c_uint32, ctypes.c_double,
                                    vp, i32, i32, vp, vp, vp, vp, i32, vp]
    L.kor_query_radius_r.restype = vp
    L.kor_query_radius_r.argtypes = [vp, i32, i32, vp, u64, ctypes.c_double, vp, i32, i32, vp,
                                     i32, vp]
    L.kor_donnelly_path.argtypes = [ctypes.c_uint32, vp, u64, vp]
    L.kor_metric_f64x3.restype = i32
    L.kor_metric_f64x3.argtypes = [i32, vp, vp, ctypes.c_double, vp, i32, ctypes.c_double, vp]
    L.kor_radius_total.restype = u64
    L.kor_radius_total.argtypes = [vp]
    L.kor_radius_copy.argtypes = [vp, vp, vp, vp]
    L.kor_radius_free.argtypes = [vp]
    return L


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


class Layout:
    """A tree layout as the reference stores it (stems, arena bytes, extents);
    block_height 0 for the Eytzinger stem order (ImmutableKdTree), > 0 for
    Donnelly<block_height>."""

    def __init__(self, dtype, k, stems, leaf_bytes, extents, max_stem_level, size, max_leaf_len,
                 block_height=0):
        self.block_height = int(block_height)
        self.dtype = np.dtype(dtype)
        self.k = k
        self.stems = stems
        self.leaf_bytes = leaf_bytes
        self.extents = extents  # uint64 [leaf_count, 2]
        self.max_stem_level = int(max_stem_level)
        self.size = int(size)
        self.max_leaf_len = int(max_leaf_len)
        self.leaf_map = None  # Mapped resolution: uint64 per stem index (2^64 - 1 = None)
        self.map_min = 0

    @property
    def leaf_count(self):
        return int(self.extents.shape[0])


class OracleTree:
    """ImmutableKdTree<A, K> built and queried by the CPU restatement."""

    def __init__(self, handle, dtype, k, L=None):
        self._h = handle
        self.dtype = np.dtype(dtype)
        self.k = k
        self._L = L if L is not None else lib()

    @classmethod
    def build(cls, points, items=None, block_height=0, L=None):
        """Soft construction; block_height > 0 builds a Donnelly<block_height> tree.
        ``L`` picks the library (default the checker, ``lib()``; the timed
        baseline passes ``timing_lib()``)."""
        L = L if L is not None else lib()
        points = np.ascontiguousarray(points)
        assert points.dtype in (np.float32, np.float64) and points.ndim == 2
        n, k = points.shape
        it = None if items is None else np.ascontiguousarray(items, dtype=np.uint32)
        h = L.kor_build_ex(0 if points.dtype == np.float32 else 1, k, _ptr(points), _ptr(it), n,
                           int(block_height))
        if not h:
            raise ValueError("unsupported dtype/dimension for the oracle")
        return cls(h, points.dtype, k, L)

    @classmethod
    def build_mutable(cls, points, items=None, block_height=0, irregular_seed=None, L=None):
        """A tree with hard buckets and Mapped stem/leaf resolution, as
        MutableKdTree's bulk construction makes it (construction.rs:413-539,
        695-864, 972-1009); with `irregular_seed`, a Mapped tree of random leaf
        depths instead (Eytzinger stems), as leaf splits leave one."""
        L = L if L is not None else lib()
        points = np.ascontiguousarray(points)
        n, k = points.shape
        it = None if items is None else np.ascontiguousarray(items, dtype=np.uint32)
        kind = 0 if irregular_seed is None else 1
        h = L.kor_build_mapped(0 if points.dtype == np.float32 else 1, k, _ptr(points), _ptr(it),
                               n, int(block_height), kind, int(irregular_seed or 0))
        if not h:
            raise ValueError("unsplittable bucket, or unsupported dtype/dimension")
        return cls(h, points.dtype, k, L)

    def leaf_map(self):
        """(leaf_idx_map, min_stem_leaf_idx) of a Mapped tree (uint64, 2^64 - 1
        for None), or None for arithmetic resolution."""
        info = np.zeros(3, dtype=np.uint64)
        self._L.kor_leaf_map_info(self._h, _ptr(info))
        if not info[0]:
            return None
        m = np.empty(int(info[1]), dtype=np.uint64)
        if m.size:
            self._L.kor_copy_leaf_map(self._h, _ptr(m))
        return m, int(info[2])

    @classmethod
    def from_layout(cls, lay: Layout, L=None):
        L = L if L is not None else lib()
        dt = 0 if lay.dtype == np.float32 else 1
        stems = np.ascontiguousarray(lay.stems, dtype=lay.dtype)
        lb = np.ascontiguousarray(lay.leaf_bytes, dtype=np.uint8)
        ex = np.ascontiguousarray(lay.extents, dtype=np.uint64)
        h = L.kor_from_layout_ex(dt, lay.k, _ptr(stems), stems.size, _ptr(lb), lb.size,
                                 _ptr(ex), ex.shape[0], lay.max_stem_level, lay.size,
                                 lay.max_leaf_len, getattr(lay, "block_height", 0))
        if not h:
            raise ValueError("unsupported dtype/dimension for this oracle library")
        if getattr(lay, "leaf_map", None) is not None:
            m = np.ascontiguousarray(lay.leaf_map, dtype=np.uint64)
            L.kor_set_leaf_map(h, _ptr(m), m.size, int(getattr(lay, "map_min", 0)))
        return cls(h, lay.dtype, lay.k, L)

    def __del__(self):
        if getattr(self, "_h", None) and getattr(self, "_L", None) is not None:
            self._L.kor_free(self._h)
            self._h = None

    def layout(self) -> Layout:
        info = np.zeros(7, dtype=np.int64)
        self._L.kor_layout_info(self._h, _ptr(info))
        stems = np.empty(int(info[0]), dtype=self.dtype)
        lb = np.empty(int(info[1]), dtype=np.uint8)
        ex = np.empty((int(info[2]), 2), dtype=np.uint64)
        self._L.kor_copy_layout(self._h, _ptr(stems), _ptr(lb), _ptr(ex))
        lay = Layout(self.dtype, self.k, stems, lb, ex, info[3], info[4], info[5], info[6])
        lm = self.leaf_map()
        if lm is not None:
            lay.leaf_map, lay.map_min = lm
        return lay

    def iter(self):
        """(items[size], points[size, K]) in KdTreeIter order
        (src/kd_tree/iter.rs:64-90): leaf by leaf, each leaf's entries by
        position."""
        lay = self.layout()
        n = int(lay.size)
        items = np.empty(n, dtype=np.uint32)
        pts = np.empty((n, self.k), dtype=self.dtype)
        if n:
            self._L.kor_iter(self._h, _ptr(items), _ptr(pts))
        return items, pts

    def _q(self, queries):
        q = np.ascontiguousarray(queries, dtype=self.dtype)
        assert q.ndim == 2 and q.shape[1] == self.k
        return q

    def _radii(self, radius, nq):
        """(scalar radius, per-query radii array or None): an array-like
        radius gives every query its own radius, in the tree's dtype."""
        if np.ndim(radius) == 0:
            return float(radius), None
        r = np.ascontiguousarray(radius, dtype=self.dtype).reshape(-1)
        assert r.size == nq, "one radius per query"
        return 0.0, r

    def _box(self, box):
        if box is None:
            return None
        return np.ascontiguousarray(box, dtype=self.dtype).reshape(self.k)

    def query_fixed(self, family, queries, k=1, radius=np.inf, metric="sqeuclidean",
                    exclusive=False, sorted=True, box=None, threads=0, stats=False):
        q = self._q(queries)
        nq = q.shape[0]
        kk = max(1, int(k))
        d = np.empty(nq * kk, dtype=self.dtype)
        it = np.empty(nq * kk, dtype=np.uint32)
        c = np.empty(nq, dtype=np.uint32)
        st = np.zeros(3, dtype=np.uint64) if stats else None
        nth = threads if threads > 0 else (os.cpu_count() or 1)
        bx = self._box(box)
        r0, rr = self._radii(radius, nq)
        rc = self._L.kor_query_fixed_r(self._h, family, METRICS[metric], _ptr(q), nq, kk, r0,
                                     _ptr(rr), int(exclusive), int(sorted), _ptr(bx), _ptr(d),
                                     _ptr(it), _ptr(c), nth, _ptr(st))
        if rc != 0:
            raise ValueError("query family not supported on this tree by the oracle")
        out = (d.reshape(nq, kk), it.reshape(nq, kk), c)
        return out + (st,) if stats else out

    def query_radius(self, family, queries, radius, metric="sqeuclidean", exclusive=False,
                     sorted=True, box=None, threads=0, stats=False):
        q = self._q(queries)
        nq = q.shape[0]
        st = np.zeros(3, dtype=np.uint64) if stats else None
        nth = threads if threads > 0 else (os.cpu_count() or 1)
        bx = self._box(box)
        r0, rr = self._radii(radius, nq)
        r = self._L.kor_query_radius_r(self._h, family, METRICS[metric], _ptr(q), nq, r0, _ptr(rr),
                                     int(exclusive), int(sorted), _ptr(bx), nth, _ptr(st))
        if not r:
            raise ValueError("query family not supported on this tree by the oracle")
        total = self._L.kor_radius_total(r)
        off = np.empty(nq + 1, dtype=np.uint64)
        d = np.empty(total, dtype=self.dtype)
        it = np.empty(total, dtype=np.uint32)
        self._L.kor_radius_copy(r, _ptr(off), _ptr(d), _ptr(it))
        self._L.kor_radius_free(r)
        out = (off, d, it)
        return out + (st,) if stats else out

    # Convenience wrappers mirroring the reference families -----------------
    def nearest_one(self, queries, metric="sqeuclidean", **kw):
        d, i, _ = self.query_fixed(FAM_NEAREST_ONE, queries, metric=metric, **kw)[:3]
        return d[:, 0], i[:, 0]

    def approx_nearest_one(self, queries, metric="sqeuclidean", **kw):
        d, i, _ = self.query_fixed(FAM_APPROX, queries, metric=metric, **kw)[:3]
        return d[:, 0], i[:, 0]

    def nearest_n(self, queries, k, radius=np.inf, metric="sqeuclidean", exclusive=False,
                  sorted=True, **kw):
        return self.query_fixed(FAM_NEAREST_N, queries, k=k, radius=radius, metric=metric,
                                exclusive=exclusive, sorted=sorted, **kw)

    def best_n_within(self, queries, radius, n, metric="sqeuclidean", exclusive=False, **kw):
        return self.query_fixed(FAM_BEST_N_WITHIN, queries, k=n, radius=radius, metric=metric,
                                exclusive=exclusive, **kw)

    def within(self, queries, radius, metric="sqeuclidean", exclusive=False, sorted=True, **kw):
        return self.query_radius(FAM_WITHIN, queries, radius, metric=metric, exclusive=exclusive,
                                 sorted=sorted, **kw)

    def periodic_nearest_one(self, queries, box, metric="sqeuclidean", **kw):
        d, i, _ = self.query_fixed(FAM_PERIODIC_NEAREST_ONE, queries, metric=metric, box=box,
                                   **kw)[:3]
        return d[:, 0], i[:, 0]

    def periodic_nearest_n(self, queries, box, k, radius=np.inf, metric="sqeuclidean",
                           exclusive=False, sorted=True, **kw):
        return self.query_fixed(FAM_PERIODIC_NEAREST_N, queries, k=k, radius=radius,
                                metric=metric, exclusive=exclusive, sorted=sorted, box=box, **kw)

    def periodic_within(self, queries, box, radius, metric="sqeuclidean", exclusive=False,
                        sorted=True, **kw):
        return self.query_radius(FAM_PERIODIC_WITHIN, queries, radius, metric=metric,
                                 exclusive=exclusive, sorted=sorted, box=box, **kw)


def donnelly_path(bh, bits):
    """(stem index after traverse() along `bits`, (left, right) children of the
    node branch_relative() reaches along `bits`) in a Donnelly<bh> stem tree."""
    b = np.ascontiguousarray(np.asarray(bits, dtype=np.uint8))
    out = np.zeros(3, dtype=np.uint32)
    lib().kor_donnelly_path(int(bh), _ptr(b) if b.size else None, b.size, _ptr(out))
    return int(out[0]), (int(out[1]), int(out[2]))


def metric_f64x3(metric, a, b, rd, off, dim, new_off):
    """(dist(a, b), rect_dist_after_update(rd, off, dim, new_off)) of `metric`
    for f64 3-D points, the arithmetic the traversal uses."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    off = np.ascontiguousarray(off, dtype=np.float64)
    out = np.zeros(2)
    rc = lib().kor_metric_f64x3(METRICS[metric], _ptr(a), _ptr(b), float(rd), _ptr(off), int(dim),
                                float(new_off), _ptr(out))
    if rc != 0:
        raise ValueError(f"unknown metric {metric}")
    return float(out[0]), float(out[1])


# ---------------------------------------------------------------------------
# Point-projected queries (QueryBuilder::with_points).  The reference answers
# them with a scan of the whole tree in iteration order
# (src/kd_tree/query/builder.rs:2175-2305), not with the traversal; these
# functions restate those scans over ``OracleTree.iter()``.
# ---------------------------------------------------------------------------

def scan_dists(points, q, metric="sqeuclidean"):
    """D::dist(point, query) for every point (dist/*/mod.rs): components in
    axis order, accumulated from the first one, in the points' dtype."""
    P = np.asarray(points)
    q = np.asarray(q, dtype=P.dtype)
    acc = np.zeros(P.shape[0], dtype=P.dtype)
    for d in range(P.shape[1]):
        diff = (P[:, d] - q[d]).astype(P.dtype)
        if metric == "chebyshev":
            comp = np.abs(diff)
            acc = np.where(comp > acc, comp, acc).astype(P.dtype)
        elif metric in ("minkowski3", "minkowski4"):
            a = np.abs(diff)
            sq = (a * a).astype(P.dtype)
            comp = (a * sq) if metric == "minkowski3" else (sq * sq)  # llvm.powi expansion
            acc = (acc + comp.astype(P.dtype)).astype(P.dtype)
        else:
            acc = (acc + (diff * diff if metric == "sqeuclidean" else np.abs(diff))).astype(P.dtype)
    return acc


def _accepts(d, radius, exclusive):
    # boundary_accepts: inclusive d <= r, exclusive d < r
    return d < radius if exclusive else d <= radius


def projected_nearest_one(tree, query, metric="sqeuclidean"):
    """scan_projected_nearest_one (builder.rs:2175-2212): the first entry in
    iteration order whose distance is below every earlier one's.  Returns
    (distance, item, point, rank); an empty tree gives (inf, 0, zeros, None)."""
    items, pts = tree.iter()
    if items.size == 0:
        return tree.dtype.type(np.inf), 0, np.zeros(tree.k, tree.dtype), None
    d = scan_dists(pts, query, metric)
    r = int(np.argmin(d))  # first occurrence of the minimum
    return d[r], int(items[r]), pts[r].copy(), r


def projected_nearest(tree, query, metric="sqeuclidean", radius=None, max_qty=None,
                      sorted=True, exclusive=False):
    """scan_projected_nearest_results (builder.rs:2214-2260): every entry in
    iteration order that the radius accepts; sorted by distance when asked or
    when max_qty is given, then cut to max_qty.  The reference sorts with
    slice::sort_unstable, which leaves the order of equal distances
    unspecified; this restatement keeps them in iteration order.  Returns
    (distances, items, points, ranks)."""
    items, pts = tree.iter()
    d = scan_dists(pts, query, metric)
    keep = np.arange(items.size) if radius is None else np.nonzero(
        _accepts(d, tree.dtype.type(radius), exclusive))[0]
    if sorted or max_qty is not None:
        keep = keep[np.argsort(d[keep], kind="stable")]
        if max_qty is not None:
            keep = keep[:max_qty]
    return d[keep], items[keep], pts[keep], keep


def projected_best(tree, query, radius, max_qty, metric="sqeuclidean", exclusive=False):
    """scan_projected_best_results (builder.rs:2262-2305): the max_qty entries
    with the smallest (item, distance) among those the radius accepts, as the
    heap's set; returned sorted by (item, distance)."""
    items, pts = tree.iter()
    d = scan_dists(pts, query, metric)
    keep = np.nonzero(_accepts(d, tree.dtype.type(radius), exclusive))[0]
    keep = keep[np.lexsort((d[keep], items[keep]))][:max_qty]
    return d[keep], items[keep], pts[keep], keep
