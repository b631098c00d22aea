"""kiddo_b200 — a batched B200 query engine for kiddo's ImmutableKdTree.

Host-side mirror of the reference's fluent query surface
(``KdTree::query(&q) -> QueryBuilder -> .execute()``,
src/kd_tree/query/builder.rs:2318-2331, :1546-1565, :1693) with a batched
``.execute_gpu()`` terminal.  Everything below the builder runs in
``libkiddo_gpu.so`` (CUDA, sm_100a) through the C ABI of include/kiddo_gpu.h.

    tree = ImmutableKdTree.new_from_slice(points)          # construction.rs:278-303
    res = tree.query(queries).nearest_n(SquaredEuclidean, 16).execute_gpu()
    res.distances, res.items, res.counts

Query families and modifiers follow builder.rs:1994-2077:
``nearest_one``, ``.approx()``, ``nearest_n``, ``nearest_n(...).within(r)``,
``within``, ``.unsorted()``, ``best_n_within``, ``.exclusive_boundaries()``,
``periodic_boundary_condition(box)`` (chosen before the query type).
Radii are in metric units (squared distance for SquaredEuclidean), exactly as
the reference's ``within::<SquaredEuclidean<_>>(radius)``.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _capi as C
from ._capi import KiddoGpuError, launch_count

__all__ = ["ImmutableKdTree", "GpuTree", "Forest", "CapturedGraph", "SquaredEuclidean",
           "Manhattan", "Chebyshev", "Minkowski", "KiddoGpuError", "NearestOneResult",
           "NearestNResult", "WithinResult", "launch_count"]


class SquaredEuclidean:
    """dist/squared_euclidean/mod.rs:21-40 — radius in squared units."""
    code = C.SQUARED_EUCLIDEAN


class Manhattan:
    """dist/manhattan/mod.rs:21-48."""
    code = C.MANHATTAN


class Chebyshev:
    """dist/chebyshev/mod.rs:19-59 — the largest per-axis |difference|; not
    with periodic boundary conditions."""
    code = C.CHEBYSHEV


class _Minkowski3:
    """dist/minkowski/mod.rs:19-58 with P = 3: the sum of |dx|^3."""
    code = C.MINKOWSKI3


class _Minkowski4:
    """dist/minkowski/mod.rs:19-58 with P = 4: the sum of |dx|^4."""
    code = C.MINKOWSKI4


def Minkowski(p: int):
    """The Minkowski<P> metric (the sum of |dx|^P, without the root) for P = 3
    or 4; not with periodic boundary conditions."""
    if p == 3:
        return _Minkowski3
    if p == 4:
        return _Minkowski4
    raise ValueError("Minkowski<P> is served for P = 3 and 4 (use Manhattan for 1, "
                     "SquaredEuclidean for 2)")


def _metric_code(m) -> int:
    if m in (SquaredEuclidean, "sqeuclidean", "squared_euclidean"):
        return C.SQUARED_EUCLIDEAN
    if m in (Manhattan, "manhattan"):
        return C.MANHATTAN
    if m in (Chebyshev, "chebyshev"):
        return C.CHEBYSHEV
    if m in (_Minkowski3, "minkowski3"):
        return C.MINKOWSKI3
    if m in (_Minkowski4, "minkowski4"):
        return C.MINKOWSKI4
    raise TypeError(f"unsupported metric {m!r} (SquaredEuclidean, Manhattan, Chebyshev or "
                    "Minkowski(3|4))")


def _vp(a: np.ndarray):
    return ctypes.c_void_p(a.ctypes.data) if a is not None and a.size else None


def _host_array(shape, dtype):
    """Result buffer in pinned host memory when torch can provide it (the
    library then copies results back at full bus speed), else pageable."""
    n = int(np.prod(shape))
    if n * np.dtype(dtype).itemsize >= (1 << 20):
        try:
            import torch
            if torch.cuda.is_available():
                tdt = {np.dtype(np.float32): torch.float32, np.dtype(np.float64): torch.float64,
                       np.dtype(np.uint32): torch.int32}[np.dtype(dtype)]
                return torch.empty(n, dtype=tdt, pin_memory=True).numpy().view(dtype).reshape(shape)
        except Exception:
            pass
    return np.empty(shape, dtype=dtype)


def _is_torch_cuda(x) -> bool:
    try:
        import torch
        return isinstance(x, torch.Tensor) and x.is_cuda
    except ImportError:
        return False


class ImmutableKdTree:
    """Host copy of an ImmutableKdTree<A, K> layout (stems, arena, extents).

    Built with the reference's soft construction by ``kgpu_layout_build``, or
    wrapped around a layout the reference itself produced (``from_layout``).
    ``block_height`` 3 or 4 builds the same tree over Donnelly<block_height>
    stems (``KdTree<A, u32, Donnelly<BH>, VecOfArenas<..>, K, 32>``,
    src/lib.rs:235) instead of the Eytzinger order; those trees are queried by
    the reference's scalar backtracking, and the same results come back.
    """

    def __init__(self, desc: C.TreeDesc, keepalive, dtype, dims):
        self._desc = desc
        self._keep = keepalive
        self.dtype = np.dtype(dtype)
        self.dims = int(dims)
        self._gpu: Optional[GpuTree] = None

    # ---- construction (construction.rs:278-303, 403-409) -------------------
    @classmethod
    def new_from_slice(cls, points, threads: int = 0, block_height: int = 0) -> "ImmutableKdTree":
        return cls._build(points, None, threads, block_height)

    @classmethod
    def new_from_entries(cls, items, points, threads: int = 0,
                         block_height: int = 0) -> "ImmutableKdTree":
        return cls._build(points, np.ascontiguousarray(items, dtype=np.uint32), threads,
                          block_height)

    @classmethod
    def _build(cls, points, items, threads, block_height=0):
        pts = np.ascontiguousarray(points)
        if pts.dtype not in (np.float32, np.float64) or pts.ndim != 2:
            raise TypeError("points must be a 2-D float32 or float64 array")
        n, k = pts.shape
        if items is not None and items.shape[0] != n:
            raise ValueError("items and points differ in length")
        L = C.lib()
        h = ctypes.c_void_p()
        C.check(L.kgpu_layout_build_stems(C.F32 if pts.dtype == np.float32 else C.F64, k,
                                          _vp(pts), _vp(items), n,
                                          C.STEM_DONNELLY if block_height else C.STEM_EYTZINGER,
                                          int(block_height), threads, ctypes.byref(h)))
        holder = _LayoutHandle(h)
        desc = C.TreeDesc()
        C.check(L.kgpu_layout_describe(h, ctypes.byref(desc)))
        return cls(desc, holder, pts.dtype, k)

    @classmethod
    def from_layout(cls, dtype, dims, stems, leaf_bytes, extents, max_stem_level, size,
                    max_leaf_len, block_height: int = 0) -> "ImmutableKdTree":
        """Wrap the reference's own layout arrays (KdTreeAccessor, traits/kd_tree.rs:15-46);
        block_height > 0 for Donnelly<block_height> stems."""
        dt = np.dtype(dtype)
        stems = np.ascontiguousarray(stems, dtype=dt)
        lb = np.ascontiguousarray(leaf_bytes, dtype=np.uint8)
        ex = np.ascontiguousarray(extents, dtype=np.uint64).reshape(-1, 2)
        d = C.TreeDesc()
        d.abi_version = C.ABI_VERSION
        d.dtype = C.F32 if dt == np.float32 else C.F64
        d.dims = dims
        d.item_size = 4
        d.bucket_size = 32
        d.stem_strategy = C.STEM_DONNELLY if block_height else C.STEM_EYTZINGER
        d.block_height = int(block_height)
        d.resolution = C.RES_ARITHMETIC
        d.stems = stems.ctypes.data if stems.size else None
        d.stem_count = stems.size
        d.leaf_bytes = lb.ctypes.data if lb.size else None
        d.leaf_bytes_len = lb.size
        d.leaf_extents = ex.ctypes.data if ex.size else None
        d.leaf_count = ex.shape[0]
        d.max_stem_level = int(max_stem_level)
        d.size = int(size)
        d.max_leaf_len = int(max_leaf_len)
        return cls(d, (stems, lb, ex), dt, dims)

    # ---- KdTreeAccessor -----------------------------------------------------
    def size(self) -> int:
        return int(self._desc.size)

    def leaf_count(self) -> int:
        return int(self._desc.leaf_count)

    def max_stem_level(self) -> int:
        return int(self._desc.max_stem_level)

    def max_leaf_len(self) -> int:
        return int(self._desc.max_leaf_len)

    def block_height(self) -> int:
        """0 for Eytzinger stems, else the Donnelly block height."""
        return int(self._desc.block_height)

    def stems(self) -> np.ndarray:
        n = int(self._desc.stem_count)
        if n == 0:
            return np.empty(0, dtype=self.dtype)
        buf = (ctypes.c_char * (n * self.dtype.itemsize)).from_address(self._desc.stems)
        return np.frombuffer(buf, dtype=self.dtype).copy()

    def leaf_bytes(self) -> np.ndarray:
        n = int(self._desc.leaf_bytes_len)
        if n == 0:
            return np.empty(0, dtype=np.uint8)
        buf = (ctypes.c_char * n).from_address(self._desc.leaf_bytes)
        return np.frombuffer(buf, dtype=np.uint8).copy()

    def leaf_extents(self) -> np.ndarray:
        n = int(self._desc.leaf_count)
        if n == 0:
            return np.empty((0, 2), dtype=np.uint64)
        buf = (ctypes.c_char * (n * 16)).from_address(self._desc.leaf_extents)
        return np.frombuffer(buf, dtype=np.uint64).reshape(n, 2).copy()

    # ---- device -------------------------------------------------------------
    def to_gpu(self, stream=None) -> "GpuTree":
        if self._gpu is None:
            self._gpu = GpuTree(self, stream)
        return self._gpu

    def query(self, queries) -> "QueryBuilder":
        """KdTree::query (builder.rs:2318-2331), batched: rows of `queries`."""
        return self.to_gpu().query(queries)


class _LayoutHandle:
    def __init__(self, h):
        self.h = h

    def __del__(self):
        if self.h and C._lib is not None:
            C._lib.kgpu_layout_free(self.h)
            self.h = None


class GpuTree:
    """A tree resident in HBM: uploaded from a host layout (kgpu_tree_create),
    or built on the device from device points (``GpuTree.build``)."""

    def __init__(self, host: Optional[ImmutableKdTree], stream=None, _handle=None, dtype=None,
                 dims=None):
        self.host = host
        if _handle is not None:
            self._h = _handle
            self.dtype = np.dtype(dtype)
            self.dims = int(dims)
            return
        L = C.lib()
        self.dtype = host.dtype
        self.dims = host.dims
        h = ctypes.c_void_p()
        C.check(L.kgpu_tree_create(ctypes.byref(host._desc), _stream_ptr(stream), ctypes.byref(h)))
        self._h = h

    @classmethod
    def from_flatvec(cls, stems, leaf_points, leaf_items, leaf_extents, max_stem_level,
                     block_height=0, stream=None) -> "GpuTree":
        """A tree whose leaves use the FlatVec strategy
        (src/leaf_strategy/flat_vec.rs:20-26): `stems` in the stem order of the
        strategy (Eytzinger, or Donnelly<block_height>), `leaf_points` the K
        point columns ([K, n] or K arrays), `leaf_items` n uint32 values and
        `leaf_extents` one (start, end) pair of point indices per leaf
        (kgpu_tree_create_flatvec)."""
        cols = [np.ascontiguousarray(c) for c in leaf_points]
        dt = cols[0].dtype if cols else np.dtype(np.float64)
        if dt not in (np.float32, np.float64) or any(c.dtype != dt for c in cols):
            raise TypeError("leaf_points must be K float32 or float64 columns of one dtype")
        st = np.ascontiguousarray(stems, dtype=dt)
        items = np.ascontiguousarray(leaf_items, dtype=np.uint32)
        ext = np.ascontiguousarray(leaf_extents, dtype=np.uint32).reshape(-1, 2)
        n = int(items.shape[0])
        if any(c.shape != (n,) for c in cols):
            raise ValueError("every leaf_points column needs one value per item")
        d = C.FlatVecDesc()
        d.abi_version = C.ABI_VERSION
        d.dtype = C.F32 if dt == np.float32 else C.F64
        d.dims = len(cols)
        d.stem_strategy = C.STEM_DONNELLY if block_height else 0
        d.block_height = int(block_height)
        d.max_stem_level = int(max_stem_level)
        d.stems = st.ctypes.data if st.size else None
        d.stem_count = st.size
        for j, c in enumerate(cols[:4]):
            d.columns[j] = c.ctypes.data if c.size else None
        d.items = items.ctypes.data if items.size else None
        d.extents = ext.ctypes.data if ext.size else None
        d.leaf_count = ext.shape[0]
        d.size = n
        h = ctypes.c_void_p()
        C.check(C.lib().kgpu_tree_create_flatvec(ctypes.byref(d), _stream_ptr(stream),
                                                 ctypes.byref(h)))
        return cls(None, _handle=h, dtype=dt, dims=len(cols))

    @staticmethod
    def _archive_format(dtype, dims, block_height, pointer_width):
        f = C.ArchiveFormat()
        f.abi_version = C.ABI_VERSION
        f.dtype = C.F32 if np.dtype(dtype) == np.float32 else C.F64
        f.dims = int(dims)
        f.stem_strategy = C.STEM_DONNELLY if block_height else C.STEM_EYTZINGER
        f.block_height = int(block_height)
        f.pointer_width = int(pointer_width)
        f.big_endian = 0
        return f

    @staticmethod
    def _archive_bytes(source):
        """(buffer, address, length, keepalive) of a path (mapped read-only)
        or a bytes-like object."""
        import mmap
        import os as _os
        if isinstance(source, (str, _os.PathLike)):
            with open(source, "rb") as fh:
                size = _os.fstat(fh.fileno()).st_size
                if size == 0:
                    raise ValueError("empty archive file")
                mm = mmap.mmap(fh.fileno(), 0, access=mmap.ACCESS_READ)
            arr = np.frombuffer(mm, dtype=np.uint8)
            return arr, arr.ctypes.data, size, (mm, arr)
        arr = np.frombuffer(source, dtype=np.uint8)
        return arr, arr.ctypes.data if arr.size else None, arr.size, (source, arr)

    @classmethod
    def inspect_archive(cls, source, dtype, dims, block_height=0, pointer_width=4) -> dict:
        """The fields of an rkyv archive of a KdTree (kgpu_archive_inspect),
        read in place; no device work."""
        arr, addr, n, keep = cls._archive_bytes(source)
        f = cls._archive_format(dtype, dims, block_height, pointer_width)
        info = C.ArchiveInfo()
        C.check(C.lib().kgpu_archive_inspect(addr, n, ctypes.byref(f), ctypes.byref(info)))
        del keep
        return {name: getattr(info, name) for name, _ in C.ArchiveInfo._fields_}

    @classmethod
    def from_archive(cls, source, dtype, dims, block_height=0, pointer_width=4,
                     stream=None) -> "GpuTree":
        """A tree uploaded straight from an rkyv 0.8 archive of
        `KdTree<dtype, u32, SS, VecOfArenas<..>, dims, 32>` (what kiddo writes
        with `rkyv::to_bytes(&tree)` and reads with `rkyv::access`,
        src/kd_tree/mod.rs:282-372, src/rkyv/adapters.rs:114-237): `source` is
        a file path, mapped read-only, or a bytes-like object.  The archive
        has no type information, so the caller names the coordinate dtype,
        dims, the Donnelly block height (0 for Eytzinger) and rkyv's pointer
        width in bytes (4 unless the crate was built with rkyv's
        pointer_width_16 or _64 feature) (kgpu_tree_create_from_archive)."""
        arr, addr, n, keep = cls._archive_bytes(source)
        f = cls._archive_format(dtype, dims, block_height, pointer_width)
        h = ctypes.c_void_p()
        C.check(C.lib().kgpu_tree_create_from_archive(addr, n, ctypes.byref(f),
                                                      _stream_ptr(stream), ctypes.byref(h)))
        del keep
        return cls(None, _handle=h, dtype=np.dtype(dtype), dims=dims)

    @staticmethod
    def _leaf_map(leaf_idx_map, min_stem_leaf_idx):
        m = np.ascontiguousarray(leaf_idx_map, dtype=np.uint64).reshape(-1)
        lm = C.LeafMap()
        lm.leaf_idx_map = m.ctypes.data if m.size else None
        lm.len = m.size
        lm.min_stem_leaf_idx = int(min_stem_leaf_idx)
        return lm, m

    @classmethod
    def from_mapped_layout(cls, dtype, dims, stems, leaf_bytes, extents, max_stem_level, size,
                           max_leaf_len, leaf_idx_map, min_stem_leaf_idx=0, block_height=0,
                           stream=None) -> "GpuTree":
        """A tree with Mapped stem/leaf resolution (OwnedStemLeafResolution::
        Mapped, src/kd_tree/stem_leaf_resolution.rs:53-66), as a MutableKdTree
        holds it: the layout arrays of ``ImmutableKdTree.from_layout`` plus the
        leaf index of each terminal stem (``leaf_idx_map[i]`` for stem
        ``min_stem_leaf_idx + i``, 2^64 - 1 for None) (kgpu_tree_create_mapped)."""
        host = ImmutableKdTree.from_layout(dtype, dims, stems, leaf_bytes, extents,
                                           max_stem_level, size, max_leaf_len, block_height)
        host._desc.resolution = C.RES_MAPPED
        lm, keep = cls._leaf_map(leaf_idx_map, min_stem_leaf_idx)
        h = ctypes.c_void_p()
        C.check(C.lib().kgpu_tree_create_mapped(ctypes.byref(host._desc), ctypes.byref(lm),
                                                _stream_ptr(stream), ctypes.byref(h)))
        del keep
        return cls(None, _handle=h, dtype=np.dtype(dtype), dims=dims)

    @classmethod
    def from_vec_of_arrays(cls, stems, content_points, content_items, sizes, max_stem_level,
                           block_height=0, stream=None, leaf_idx_map=None,
                           min_stem_leaf_idx=0) -> "GpuTree":
        """A tree whose leaves use the VecOfArrays strategy
        (src/leaf_strategy/vec_of_arrays.rs:51-97): `stems` in the stem order of
        the strategy, each leaf's `content_points` ([leaf_count, K, B]) and
        `content_items` ([leaf_count, B], uint32) and its live-entry count in
        `sizes` ([leaf_count]) (kgpu_tree_create_vecofarrays); with
        `leaf_idx_map`, a MutableKdTree's Mapped resolution
        (kgpu_tree_create_vecofarrays_mapped)."""
        pts = np.ascontiguousarray(content_points)
        if pts.dtype not in (np.float32, np.float64) or pts.ndim != 3:
            raise TypeError("content_points must be a float32 or float64 [leaf_count, K, B] array")
        L_, K, B = pts.shape
        items = np.ascontiguousarray(content_items, dtype=np.uint32).reshape(L_, B)
        sz = np.ascontiguousarray(sizes, dtype=np.uint64).reshape(L_)
        st = np.ascontiguousarray(stems, dtype=pts.dtype)
        d = C.VecOfArraysDesc()
        d.abi_version = C.ABI_VERSION
        d.dtype = C.F32 if pts.dtype == np.float32 else C.F64
        d.dims = K
        d.stem_strategy = C.STEM_DONNELLY if block_height else 0
        d.block_height = int(block_height)
        d.max_stem_level = int(max_stem_level)
        d.stems = st.ctypes.data if st.size else None
        d.stem_count = st.size
        d.bucket = B
        d.content_points = pts.ctypes.data if pts.size else None
        d.content_items = items.ctypes.data if items.size else None
        d.sizes = sz.ctypes.data if sz.size else None
        d.leaf_count = L_
        h = ctypes.c_void_p()
        if leaf_idx_map is None:
            C.check(C.lib().kgpu_tree_create_vecofarrays(ctypes.byref(d), _stream_ptr(stream),
                                                         ctypes.byref(h)))
        else:
            # a MutableKdTree's own leaves and Mapped resolution
            lm, keep = cls._leaf_map(leaf_idx_map, min_stem_leaf_idx)
            C.check(C.lib().kgpu_tree_create_vecofarrays_mapped(ctypes.byref(d),
                                                                ctypes.byref(lm),
                                                                _stream_ptr(stream),
                                                                ctypes.byref(h)))
            del keep
        return cls(None, _handle=h, dtype=pts.dtype, dims=K)

    @classmethod
    def build(cls, points, items=None, stream=None) -> "GpuTree":
        """The ImmutableKdTree of CUDA tensor `points` ([n, dims], float32 or
        float64) built on the device (kgpu_tree_build): the same layout, byte for
        byte, as ``ImmutableKdTree.new_from_slice`` / ``new_from_entries``
        (`items`: uint32 values in an int32 CUDA tensor) build on the host."""
        import torch
        if not (isinstance(points, torch.Tensor) and points.is_cuda and points.dim() == 2):
            raise TypeError("points must be a 2-D CUDA tensor")
        if points.dtype not in (torch.float32, torch.float64):
            raise TypeError("points must be float32 or float64")
        pts = points.contiguous()
        it = None
        if items is not None:
            it = items.contiguous()
            if it.shape[0] != pts.shape[0] or it.element_size() != 4:
                raise ValueError("items must be one 32-bit value per point")
        h = ctypes.c_void_p()
        dt = np.float32 if pts.dtype == torch.float32 else np.float64
        C.check(C.lib().kgpu_tree_build(C.F32 if dt == np.float32 else C.F64, pts.shape[1],
                                        ctypes.c_void_p(pts.data_ptr()),
                                        None if it is None else ctypes.c_void_p(it.data_ptr()),
                                        pts.shape[0], _stream_ptr(stream), ctypes.byref(h)))
        return cls(None, _handle=h, dtype=dt, dims=pts.shape[1])

    def read_layout(self):
        """(stems, leaf_bytes, extents) copied back from the device; extents as
        (byte offset, len) pairs like the reference's leaf_extents."""
        inf = self.info()
        stems = np.empty(int(inf["stem_count"]), dtype=self.dtype)
        lb = np.empty(int(inf["leaf_bytes_len"]), dtype=np.uint8)
        ex = np.empty((int(inf["leaf_count"]), 2), dtype=np.uint64)
        C.check(C.lib().kgpu_tree_read_layout(self._h, _vp(stems), _vp(lb), _vp(ex), None))
        return stems, lb, ex

    def size(self) -> int:
        return int(self.info()["size"])

    def __del__(self):
        if getattr(self, "_h", None) and C._lib is not None:
            C._lib.kgpu_tree_destroy(self._h)
            self._h = None

    def info(self):
        a = np.zeros(8, dtype=np.int64)
        C.check(C.lib().kgpu_tree_info(self._h, _vp(a)))
        return dict(zip(["dtype", "dims", "size", "leaf_count", "max_stem_level", "stem_count",
                         "leaf_bytes_len", "device_bytes"], a.tolist()))

    def iter(self, stream=None):
        """The tree's entries as CUDA tensors (items [size] int32 holding the
        uint32 values, points [size, dims]) in the reference's iteration order
        (KdTree::iter, src/kd_tree/iter.rs:64-90): leaf by leaf, each leaf's
        entries in stored order (kgpu_tree_iter)."""
        import torch
        n = self.size()
        tdt = torch.float32 if self.dtype == np.float32 else torch.float64
        items = torch.empty(max(n, 1), dtype=torch.int32, device="cuda")
        pts = torch.empty((max(n, 1), self.dims), dtype=tdt, device="cuda")
        st = stream if stream is not None else torch.cuda.current_stream()
        C.check(C.lib().kgpu_tree_iter(self._h, ctypes.c_void_p(items.data_ptr()),
                                       ctypes.c_void_p(pts.data_ptr()), _stream_ptr(st)))
        return items[:n], pts[:n]

    def project(self, items, stream=None):
        """(ranks, points) of result items (a CUDA int32 tensor of any shape):
        each item's position in iteration order (-1 as int32 when the item is
        not in the tree) and its stored point (kgpu_tree_project).  Needs
        distinct items in the tree."""
        import torch
        tdt = torch.float32 if self.dtype == np.float32 else torch.float64
        it = items.contiguous()
        ranks = torch.empty(it.shape, dtype=torch.int32, device=it.device)
        pts = torch.empty(tuple(it.shape) + (self.dims,), dtype=tdt, device=it.device)
        st = stream if stream is not None else torch.cuda.current_stream(it.device)
        C.check(C.lib().kgpu_tree_project(self._h, ctypes.c_void_p(it.data_ptr()), it.numel(),
                                          ctypes.c_void_p(ranks.data_ptr()),
                                          ctypes.c_void_p(pts.data_ptr()), _stream_ptr(st)))
        return ranks, pts

    def _self_forest(self):
        # made per call: a forest cached on the tree would hold the tree in a
        # reference cycle and keep its device memory until a garbage-collector pass
        return Forest([self])

    def query(self, queries) -> "QueryBuilder":
        return QueryBuilder(self, queries)


def _stream_ptr(stream):
    if stream is None:
        return None
    if hasattr(stream, "cuda_stream"):
        return ctypes.c_void_p(stream.cuda_stream)
    return ctypes.c_void_p(int(stream))


@dataclass
class NearestOneResult:
    distances: object
    items: object
    points: object = None  # with_points(): [nq, dims]


@dataclass
class NearestNResult:
    distances: object
    items: object
    counts: object
    points: object = None  # with_points(): [nq, max_qty, dims], zeros in unused slots


@dataclass
class WithinResult:
    offsets: object
    distances: object
    items: object
    points: object = None  # with_points(): [total, dims]

    def __len__(self):
        return len(self.offsets) - 1

    def __getitem__(self, i):
        a, b = int(self.offsets[i]), int(self.offsets[i + 1])
        if self.points is not None:
            return self.distances[a:b], self.items[a:b], self.points[a:b]
        return self.distances[a:b], self.items[a:b]

    def iter(self):
        """Yields (query index, distance, item, point) per hit, query by query,
        each query's hits in the result's order; fields left out by
        without_distances / without_items / no with_points are None."""
        off = self.offsets
        for i in range(len(off) - 1):
            for j in range(int(off[i]), int(off[i + 1])):
                yield (i,
                       None if self.distances is None else self.distances[j],
                       None if self.items is None else self.items[j],
                       None if self.points is None else self.points[j])

    def visit(self, visitor):
        """Calls visitor(query index, distance, item, point) once per hit, in
        the order of ``iter()``."""
        for hit in self.iter():
            visitor(*hit)


def _csr_order(offsets, ranks, dists=None):
    """Permutation of a CSR result's entries that orders each row by
    iteration rank, or by (distance, rank) when `dists` is given; rows keep
    their places.  Ranks are int32 holding uint32 values."""
    import torch
    nq = offsets.shape[0] - 1
    rows = torch.repeat_interleave(torch.arange(nq, device=offsets.device),
                                   offsets[1:] - offsets[:-1], output_size=ranks.shape[0])
    order = torch.argsort(rows.to(torch.int64) * (1 << 32) +
                          ranks.to(torch.int64).remainder(1 << 32), stable=True)
    if dists is not None:
        o2 = torch.argsort(dists[order], stable=True)
        order = order[o2][torch.argsort(rows[order][o2], stable=True)]
    return order


def _metric_dist(points, q, metric):
    """D::dist(point, query) row by row (dist/*/mod.rs): components in axis
    order, accumulated from zero in the points' dtype."""
    import torch
    acc = torch.zeros(points.shape[0], dtype=points.dtype, device=points.device)
    for d in range(points.shape[1]):
        diff = points[:, d] - q[:, d]
        if metric == C.CHEBYSHEV:
            a = diff.abs()
            acc = torch.where(a > acc, a, acc)
        elif metric in (C.MINKOWSKI3, C.MINKOWSKI4):
            a = diff.abs()
            sq = a * a
            acc = acc + (a * sq if metric == C.MINKOWSKI3 else sq * sq)
        else:
            acc = acc + (diff * diff if metric == C.SQUARED_EUCLIDEAN else diff.abs())
    return acc


def _first_by_rank(r, ranks, pts, q, metric, tree, stream):
    """scan_projected_nearest_one's answer from a radius result holding every
    entry at each query's least distance: the row's entry of least rank.  A
    row with no entry is a query whose distance to every entry is NaN (a NaN
    coordinate): no candidate is below the first one, so the scan keeps the
    first entry in iteration order, at its own (NaN) distance."""
    import torch
    order = _csr_order(r.offsets, ranks)
    nq = r.offsets.shape[0] - 1
    nonempty = r.offsets[1:] > r.offsets[:-1]
    total = int(order.shape[0])
    if total == 0:
        first = torch.zeros(nq, dtype=torch.int64, device=q.device)
        d, it, p = (torch.zeros(nq, dtype=q.dtype, device=q.device),
                    torch.zeros(nq, dtype=torch.int32, device=q.device),
                    torch.zeros((nq, q.shape[1]), dtype=q.dtype, device=q.device))
    else:
        first = order[r.offsets[:-1].clamp(max=total - 1)]  # each row's least rank
        d, it, p = r.distances[first], r.items[first], pts[first]
    if bool(nonempty.all()):
        return NearestOneResult(d, it, p)
    items0, pts0 = tree.iter(stream)
    p0 = pts0[:1].expand(nq, -1)
    d0 = _metric_dist(p0, q, metric)
    keep = nonempty[:, None]
    return NearestOneResult(torch.where(nonempty, d, d0), torch.where(nonempty, it, items0[0]),
                            torch.where(keep, p, p0))


def _row_order(dists, ranks):
    """Per row of [nq, k] results, the column order by distance, equal
    distances by iteration rank; unused slots (rank 0xFFFFFFFF, distance +inf)
    stay last."""
    import torch
    o1 = torch.argsort(ranks.to(torch.int64).remainder(1 << 32), dim=1, stable=True)
    o2 = torch.argsort(torch.gather(dists, 1, o1), dim=1, stable=True)
    return torch.gather(o1, 1, o2)


class QueryBuilder:
    """Runtime mirror of the typestate QueryBuilder (builder.rs:1373-1398)."""

    def __init__(self, tree: GpuTree, queries):
        self.tree = tree
        self.queries = queries
        self.family = None
        self.metric = None
        self.max_qty = 0
        self.radius = None
        self.exclusive = False
        self.sorted = True
        self.box = None
        self.spatial_order = None  # None: the library decides
        self.engine = None
        self.refill = None  # idle lanes before a warp refills (None: 24)
        self.chunk = None   # queries handed to a warp at a time (None: 64)
        self.stream = None
        self.points = False
        self.want_items = True
        self.want_distances = True

    # ---- space --------------------------------------------------------------
    def periodic_boundary_condition(self, box_size) -> "QueryBuilder":
        if self.family is not None:
            raise TypeError("periodic_boundary_condition must be chosen before the query type")
        if self.points:
            raise TypeError("with_points() is available only for non-periodic queries")
        box = np.ascontiguousarray(box_size, dtype=self.tree.dtype).reshape(-1)
        if box.size != self.tree.dims:
            raise ValueError("box_size must have one entry per axis")
        if not np.all(box > 0):
            raise ValueError("periodic box sizes must be strictly positive")
        self.box = box
        return self

    # ---- query type -----------------------------------------------------------
    def nearest_one(self, metric) -> "QueryBuilder":
        self._set_family(C.NEAREST_ONE, metric)
        return self

    def nearest_n(self, metric, max_qty: int) -> "QueryBuilder":
        if int(max_qty) < 1:
            raise ValueError("max_qty must be non-zero (NonZeroUsize)")
        self._set_family(C.NEAREST_N, metric)
        self.max_qty = int(max_qty)
        return self

    def within(self, *args) -> "QueryBuilder":
        """``within(metric, radius)`` selects a radius query;
        ``nearest_n(...).within(radius)`` bounds a k-NN query."""
        if self.family == C.NEAREST_N and len(args) == 1:
            self.family = C.NEAREST_N_WITHIN
            self.radius = float(args[0])
            return self
        if len(args) != 2:
            raise TypeError("within(metric, radius) or nearest_n(metric, k).within(radius)")
        self._set_family(C.WITHIN, args[0])
        self.radius = float(args[1])
        return self

    def best_n_within(self, metric, radius, max_qty: int) -> "QueryBuilder":
        if self.box is not None:
            raise TypeError("best_n_within is Cartesian-only")
        if int(max_qty) < 1:
            raise ValueError("max_qty must be non-zero")
        self._set_family(C.BEST_N_WITHIN, metric)
        self.radius = float(radius)
        self.max_qty = int(max_qty)
        return self

    # ---- options ---------------------------------------------------------------
    def approx(self) -> "QueryBuilder":
        if self.family != C.NEAREST_ONE or self.box is not None:
            raise TypeError("approx() is available only after a Cartesian nearest_one()")
        self.family = C.APPROX_NEAREST_ONE
        return self

    def unsorted(self) -> "QueryBuilder":
        if self.family not in (C.WITHIN, C.NEAREST_N, C.NEAREST_N_WITHIN):
            raise TypeError("unsorted() applies to within and nearest_n queries")
        self.sorted = False
        if self.family == C.WITHIN:
            self.family = C.WITHIN_UNSORTED
        return self

    def exclusive_boundaries(self) -> "QueryBuilder":
        if self.family not in (C.WITHIN, C.WITHIN_UNSORTED, C.NEAREST_N_WITHIN, C.BEST_N_WITHIN):
            raise TypeError("exclusive_boundaries() applies to radius-bounded queries")
        self.exclusive = True
        return self

    # ---- projections ----------------------------------------------------------
    def with_points(self) -> "QueryBuilder":
        """Return each hit's stored point too (QueryBuilder::with_points,
        src/kd_tree/query/builder.rs:1982-1987; non-periodic queries only).

        The reference answers these queries by scanning the tree in iteration
        order (builder.rs:2175-2305), and so does the result here:
          * nearest_one (and approx, which the scan makes exact): the first
            entry in iteration order at the least distance;
          * within().unsorted(): the hits in iteration order;
          * within, nearest_n, nearest_n().within (sorted or not): by distance,
            equal distances in iteration order.  The reference sorts with
            slice::sort_unstable, whose order of equal distances, and choice
            among equal distances at the max_qty cut, Rust leaves unspecified;
            here the cut follows nearest_n's own rule;
          * best_n_within: ascending item.
        Items must be distinct (KGPU_EUNSUPPORTED otherwise); nearest_one takes
        Eytzinger trees."""
        if self.box is not None:
            raise TypeError("with_points() is available only for non-periodic queries")
        self.points = True
        return self

    def without_points(self) -> "QueryBuilder":
        """Leave the stored points out again (builder.rs:1926-1933)."""
        self.points = False
        return self

    def with_items(self) -> "QueryBuilder":
        """Include the items in the results (builder.rs:1935-1942), the default."""
        self.want_items = True
        return self

    def without_items(self) -> "QueryBuilder":
        """Leave the items out of the results: ``items`` is None
        (builder.rs:1944-1951).  The query itself is unchanged."""
        self.want_items = False
        return self

    def with_distances(self) -> "QueryBuilder":
        """Include the distances in the results (builder.rs:1953-1960), the default."""
        self.want_distances = True
        return self

    def without_distances(self) -> "QueryBuilder":
        """Leave the distances out of the results: ``distances`` is None
        (builder.rs:1962-1969).  The query itself is unchanged."""
        self.want_distances = False
        return self

    def with_spatial_order(self, on: Optional[bool] = True) -> "QueryBuilder":
        """Process the batch grouped by leaf (True), in the given order (False),
        or let the library decide (None, the default).  Results are identical."""
        self.spatial_order = None if on is None else bool(on)
        return self

    def with_engine(self, engine: Optional[str]) -> "QueryBuilder":
        """Force the kernel variant: "warp" (one warp per query), "thread"
        (one thread per query) or "coop" (one walk per thread, each leaf
        scanned by the whole warp; sorted nearest_n with k <= 32, other
        families as "thread"); None lets the library choose.  Same results."""
        if engine not in (None, "warp", "thread", "coop"):
            raise ValueError("engine must be None, 'warp', 'thread' or 'coop'")
        self.engine = engine
        return self

    def with_tuning(self, refill: Optional[int] = None, chunk: Optional[int] = None
                    ) -> "QueryBuilder":
        """Launch knobs of the lane-refilled kernels (kgpu_query_desc::tuning):
        refill a warp's idle lanes once `refill` (1..32) are idle, hand queries
        to a warp `chunk` (a power of two, 32..1024) at a time; None keeps the
        defaults (24, 64).  Same results."""
        if refill is not None and not 1 <= int(refill) <= 32:
            raise ValueError("refill must be 1..32")
        if chunk is not None and (int(chunk) < 32 or int(chunk) > 1024 or
                                  int(chunk) & (int(chunk) - 1)):
            raise ValueError("chunk must be a power of two in 32..1024")
        self.refill = None if refill is None else int(refill)
        self.chunk = None if chunk is None else int(chunk)
        return self

    def autotuned(self, tune_if_missing: bool = True) -> "QueryBuilder":
        """Apply the cached autotuner choice of engine and processing order for
        this kind of query (kiddo_b200.autotune); tune on a sample of this batch
        if there is none yet.  Device batches only; results are unchanged."""
        from . import autotune
        if self.family is None:
            raise TypeError("choose a query type before autotuned()")
        choice = autotune.lookup(self)
        if choice is None and tune_if_missing and _is_torch_cuda(self.queries):
            choice = autotune.tune(self)
        if choice is not None:
            self.engine = choice["engine"]
            self.spatial_order = choice["spatial_order"]
            self.with_tuning(choice.get("refill"), choice.get("chunk"))
        return self

    def on_stream(self, stream) -> "QueryBuilder":
        self.stream = stream
        return self

    def _set_family(self, fam, metric):
        if self.family is not None:
            raise TypeError("query type already chosen")
        self.family = fam
        self.metric = _metric_code(metric)

    # ---- terminal ---------------------------------------------------------------
    def _desc(self, host: bool) -> C.QueryDesc:
        d = C.QueryDesc()
        d.abi_version = C.ABI_VERSION
        d.family = self.family
        d.metric = self.metric
        d.max_qty = self.max_qty
        d.radius = float(self.radius) if self.radius is not None else float("inf")
        d.exclusive = int(self.exclusive)
        d.sorted = int(self.sorted)
        d.periodic_box = self.box.ctypes.data if self.box is not None else None
        d.flags = (C.FLAG_HOST_BUFFERS if host else 0) | (
            C.FLAG_SPATIAL_ORDER if self.spatial_order else 0) | (
            C.FLAG_NO_SPATIAL_ORDER if self.spatial_order is False else 0) | (
            C.FLAG_ENGINE_WARP if self.engine == "warp" else 0) | (
            C.FLAG_ENGINE_THREAD if self.engine == "thread" else 0) | (
            C.FLAG_ENGINE_COOP if self.engine == "coop" else 0)
        d.tuning = (self.refill or 0) | ((int(self.chunk).bit_length() - 1) << 8
                                         if self.chunk else 0)
        return d

    def traversal_stats(self):
        """[stem visits, leaf visits, points scanned] over the batch
        (exact_query_stats.rs:23-60), measured by the GPU traversal."""
        if self.family is None:
            raise TypeError("choose a query type first")
        q = np.ascontiguousarray(self.queries, dtype=self.tree.dtype).reshape(-1, self.tree.dims)
        out = np.zeros(3, dtype=np.uint64)
        d = self._desc(True)
        C.check(C.lib().kgpu_query_stats(self.tree._h, ctypes.byref(d), _vp(q), q.shape[0],
                                         _vp(out), _stream_ptr(self.stream)))
        return out

    def execute_gpu(self):
        if self.family is None:
            raise TypeError("choose a query type before execute_gpu()")
        if self.points:
            res = self._execute_points()
        elif _is_torch_cuda(self.queries):
            res = self._execute_device()
        else:
            res = self._execute_host()
        if not self.want_items:
            res.items = None
        if not self.want_distances:
            res.distances = None
        return res

    def visit(self, visitor):
        """within().unsorted().visit (builder.rs:1643-1665, 5136-5184) for the
        batch: runs the query, then calls visitor(query index, distance, item,
        point) per hit, each query's hits in the reference's visiting order
        (traversal order; iteration order with with_points())."""
        self._check_streaming()
        self.execute_gpu().visit(visitor)

    def iter(self):
        """within().unsorted().iter (builder.rs:5187-5230) for the batch: the
        hits of ``visit`` as an iterator over the batch's result."""
        self._check_streaming()
        return self.execute_gpu().iter()

    def _check_streaming(self):
        if self.family != C.WITHIN_UNSORTED:
            raise TypeError("visit() and iter() follow within(...).unsorted()")

    def _sub(self, family, queries):
        """A copy of this builder without projections, for another family."""
        b = QueryBuilder(self.tree, queries)
        b.__dict__.update({k: v for k, v in self.__dict__.items() if k != "queries"})
        b.points = False
        b.want_items = b.want_distances = True
        b.family = family
        return b

    def _execute_points(self):
        import torch
        host = not _is_torch_cuda(self.queries)
        if host:
            qh = np.ascontiguousarray(self.queries, dtype=self.tree.dtype)
            if qh.ndim == 1:
                qh = qh.reshape(1, -1)
            q = torch.from_numpy(qh).cuda()
        else:
            q = self.queries.contiguous()
        if q.shape[1] != self.tree.dims:
            raise ValueError("query dimensionality does not match the tree")
        nq = q.shape[0]
        stream = self.stream if self.stream is not None else torch.cuda.current_stream(q.device)
        fam = self.family
        if fam in (C.NEAREST_ONE, C.APPROX_NEAREST_ONE):
            res = self._points_nearest_one(q, stream)
        elif fam in (C.WITHIN, C.WITHIN_UNSORTED):
            r = self._sub(C.WITHIN_UNSORTED, q)._execute_device()
            ranks, pts = self.tree.project(r.items, stream)
            order = _csr_order(r.offsets, ranks, r.distances if fam == C.WITHIN else None)
            res = WithinResult(r.offsets, r.distances[order], r.items[order], pts[order])
        else:
            r = self._sub(fam, q)
            if fam != C.BEST_N_WITHIN:
                r.sorted = True
            r = r._execute_device()
            ranks, pts = self.tree.project(r.items, stream)
            if fam == C.BEST_N_WITHIN:
                res = NearestNResult(r.distances, r.items, r.counts, pts)
            else:
                order = _row_order(r.distances, ranks)
                res = NearestNResult(torch.gather(r.distances, 1, order),
                                     torch.gather(r.items, 1, order), r.counts,
                                     pts[torch.arange(nq, device=q.device)[:, None], order])
        if not host:
            return res
        torch.cuda.synchronize()
        out = {}
        for k, v in res.__dict__.items():
            a = v.cpu().numpy() if v is not None else None
            if a is not None and k in ("items", "counts") and a.dtype == np.int32:
                a = a.view(np.uint32)
            if a is not None and k == "offsets":
                a = a.astype(np.uint64)
            out[k] = a
        return type(res)(**out)

    def _points_nearest_one(self, q, stream):
        """scan_projected_nearest_one (builder.rs:2175-2212): the first entry in
        iteration order at the least distance.  The least distance comes from
        the nearest_one traversal, every entry at that distance from a radius
        query with one radius per query, and the earliest of them by rank."""
        import torch
        nq, K = q.shape[0], self.tree.dims
        tdt = q.dtype
        if self.tree.size() == 0:
            return NearestOneResult(torch.full((nq,), float("inf"), dtype=tdt, device=q.device),
                                    torch.zeros(nq, dtype=torch.int32, device=q.device),
                                    torch.zeros((nq, K), dtype=tdt, device=q.device))
        best = self._sub(C.NEAREST_ONE, q)._execute_device().distances
        fq = self.tree._self_forest().query(q, torch.zeros(nq, dtype=torch.int32, device=q.device),
                                            best)
        fq.stream = self.stream
        fq.family, fq.metric = C.WITHIN_UNSORTED, self.metric
        fq.radius = float("inf")
        r = fq.execute_gpu()
        ranks, pts = self.tree.project(r.items, stream)
        return _first_by_rank(r, ranks, pts, q, self.metric, self.tree, stream)

    def _execute_host(self):
        L = C.lib()
        q = np.ascontiguousarray(self.queries, dtype=self.tree.dtype)
        if q.ndim == 1:
            q = q.reshape(1, -1)
        if q.shape[1] != self.tree.dims:
            raise ValueError("query dimensionality does not match the tree")
        nq = q.shape[0]
        d = self._desc(True)
        st = _stream_ptr(self.stream)
        if self.family in (C.WITHIN, C.WITHIN_UNSORTED):
            off = np.empty(nq + 1, dtype=np.uint64)
            C.check(L.kgpu_query_radius_count(self.tree._h, ctypes.byref(d), _vp(q), nq, _vp(off),
                                              st))
            total = int(off[-1])
            dist = np.empty(total, dtype=self.tree.dtype)
            items = np.empty(total, dtype=np.uint32)
            C.check(L.kgpu_query_radius_fill(self.tree._h, ctypes.byref(d), _vp(q), nq, _vp(off),
                                             _vp(dist), _vp(items), st))
            return WithinResult(off, dist, items)
        w = 1 if self.family in (C.NEAREST_ONE, C.APPROX_NEAREST_ONE) else self.max_qty
        dist = _host_array((nq, w), self.tree.dtype)
        items = _host_array((nq, w), np.uint32)
        counts = _host_array((nq,), np.uint32)
        C.check(L.kgpu_query(self.tree._h, ctypes.byref(d), _vp(q), nq, _vp(dist), _vp(items),
                             _vp(counts), st))
        if w == 1 and self.family in (C.NEAREST_ONE, C.APPROX_NEAREST_ONE):
            return NearestOneResult(dist[:, 0], items[:, 0])
        return NearestNResult(dist, items, counts)

    def _execute_device(self):
        import torch
        L = C.lib()
        tdt = torch.float32 if self.tree.dtype == np.float32 else torch.float64
        q = self.queries
        if q.dtype != tdt:
            raise TypeError("device queries must match the tree dtype")
        q = q.contiguous()
        nq = q.shape[0]
        d = self._desc(False)
        stream = self.stream if self.stream is not None else torch.cuda.current_stream(q.device)
        st = _stream_ptr(stream)
        dev = q.device
        if self.family in (C.WITHIN, C.WITHIN_UNSORTED):
            off = torch.empty(nq + 1, dtype=torch.int64, device=dev)
            C.check(L.kgpu_query_radius_count(self.tree._h, ctypes.byref(d),
                                              ctypes.c_void_p(q.data_ptr()), nq,
                                              ctypes.c_void_p(off.data_ptr()), st))
            total = int(off[-1].item())
            dist = torch.empty(max(total, 1), dtype=tdt, device=dev)
            items = torch.empty(max(total, 1), dtype=torch.int32, device=dev)
            C.check(L.kgpu_query_radius_fill(self.tree._h, ctypes.byref(d),
                                             ctypes.c_void_p(q.data_ptr()), nq,
                                             ctypes.c_void_p(off.data_ptr()),
                                             ctypes.c_void_p(dist.data_ptr()),
                                             ctypes.c_void_p(items.data_ptr()), st))
            return WithinResult(off, dist[:total], items[:total])
        w = 1 if self.family in (C.NEAREST_ONE, C.APPROX_NEAREST_ONE) else self.max_qty
        dist = torch.empty((nq, w), dtype=tdt, device=dev)
        items = torch.empty((nq, w), dtype=torch.int32, device=dev)
        counts = torch.empty(nq, dtype=torch.int32, device=dev)
        C.check(L.kgpu_query(self.tree._h, ctypes.byref(d), ctypes.c_void_p(q.data_ptr()), nq,
                             ctypes.c_void_p(dist.data_ptr()), ctypes.c_void_p(items.data_ptr()),
                             ctypes.c_void_p(counts.data_ptr()), st))
        if self.family in (C.NEAREST_ONE, C.APPROX_NEAREST_ONE):
            return NearestOneResult(dist[:, 0], items[:, 0])
        return NearestNResult(dist, items, counts)


class Forest:
    """Many uploaded trees of one dtype/dimensionality answered in one launch.

    ``forest.query(queries, tree_of, radii=None)`` takes CUDA tensors: queries
    [nq, dims], tree_of [nq] (int32 index into ``trees``) and optionally one
    radius per query.  The builder is the same as a single tree's.
    """

    def __init__(self, trees, stream=None):
        gts = [t.to_gpu() if isinstance(t, ImmutableKdTree) else t for t in trees]
        if not gts:
            raise ValueError("a forest needs at least one tree")
        self.trees = gts
        self.dtype = gts[0].dtype
        self.dims = gts[0].dims
        arr = (ctypes.c_void_p * len(gts))(*[g._h.value for g in gts])
        h = ctypes.c_void_p()
        C.check(C.lib().kgpu_forest_create(arr, len(gts), _stream_ptr(stream), ctypes.byref(h)))
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None) and C._lib is not None:
            C._lib.kgpu_forest_destroy(self._h)
            self._h = None

    def query(self, queries, tree_of, radii=None) -> "ForestQueryBuilder":
        return ForestQueryBuilder(self, queries, tree_of, radii)


class ForestQueryBuilder(QueryBuilder):
    def __init__(self, forest: Forest, queries, tree_of, radii):
        super().__init__(forest, queries)
        self.tree_of = tree_of
        self.radii = radii

    def execute_gpu(self):
        import torch
        if self.family is None:
            raise TypeError("choose a query type before execute_gpu()")
        L = C.lib()
        f = self.tree
        tdt = torch.float32 if f.dtype == np.float32 else torch.float64
        q = self.queries
        if not (_is_torch_cuda(q) and _is_torch_cuda(self.tree_of)):
            raise TypeError("forest queries take CUDA tensors")
        q = q.contiguous()
        tof = self.tree_of.to(torch.int32).contiguous()
        rad = None if self.radii is None else self.radii.to(tdt).contiguous()
        nq = q.shape[0]
        d = self._desc(False)
        stream = self.stream if self.stream is not None else torch.cuda.current_stream(q.device)
        st = _stream_ptr(stream)
        vp = ctypes.c_void_p
        rp = vp(rad.data_ptr()) if rad is not None else None
        dev = q.device
        if self.family in (C.WITHIN, C.WITHIN_UNSORTED):
            off = torch.empty(nq + 1, dtype=torch.int64, device=dev)
            C.check(L.kgpu_forest_query_radius_count(f._h, ctypes.byref(d), vp(q.data_ptr()),
                                                     vp(tof.data_ptr()), rp, nq,
                                                     vp(off.data_ptr()), st))
            total = int(off[-1].item())
            dist = torch.empty(max(total, 1), dtype=tdt, device=dev)
            items = torch.empty(max(total, 1), dtype=torch.int32, device=dev)
            status = torch.zeros(1, dtype=torch.int32, device=dev)
            C.check(L.kgpu_forest_query_radius_fill(f._h, ctypes.byref(d), vp(q.data_ptr()),
                                                    vp(tof.data_ptr()), rp, nq,
                                                    vp(off.data_ptr()), total,
                                                    vp(dist.data_ptr()), vp(items.data_ptr()),
                                                    vp(status.data_ptr()), st))
            if int(status.item()) != 0:
                raise KiddoGpuError(int(status.item()), "forest fill overflowed its capacity")
            return WithinResult(off, dist[:total], items[:total])
        w = 1 if self.family in (C.NEAREST_ONE, C.APPROX_NEAREST_ONE) else self.max_qty
        dist = torch.empty((nq, w), dtype=tdt, device=dev)
        items = torch.empty((nq, w), dtype=torch.int32, device=dev)
        counts = torch.empty(nq, dtype=torch.int32, device=dev)
        C.check(L.kgpu_forest_query(f._h, ctypes.byref(d), vp(q.data_ptr()), vp(tof.data_ptr()),
                                    rp, nq, vp(dist.data_ptr()), vp(items.data_ptr()),
                                    vp(counts.data_ptr()), st))
        if self.family in (C.NEAREST_ONE, C.APPROX_NEAREST_ONE):
            return NearestOneResult(dist[:, 0], items[:, 0])
        return NearestNResult(dist, items, counts)


class CapturedGraph:
    """CUDA-graph capture of device-pointer engine calls on a stream.

        g = CapturedGraph(stream)
        with g:                      # cudaStreamBeginCapture ... EndCapture
            forest.query(...).best_n_within(...).on_stream(stream).execute_gpu()
        g.replay()
    Only calls that never read back to the host can be captured (see
    include/kiddo_gpu.h).
    """

    def __init__(self, stream):
        self.stream = stream
        self._g = None

    def __enter__(self):
        C.check(C.lib().kgpu_graph_begin(_stream_ptr(self.stream)))
        return self

    def __exit__(self, exc_type, exc, tb):
        h = ctypes.c_void_p()
        st = C.lib().kgpu_graph_end(_stream_ptr(self.stream), ctypes.byref(h))
        if exc_type is None:
            C.check(st)
            self._g = h
        return False

    def replay(self):
        C.check(C.lib().kgpu_graph_launch(self._g, _stream_ptr(self.stream)))

    def __del__(self):
        if getattr(self, "_g", None) and C._lib is not None:
            C._lib.kgpu_graph_destroy(self._g)
            self._g = None
