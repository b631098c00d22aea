"""ctypes binding of libkiddo_gpu.so (declarations of include/kiddo_gpu.h).

The library is loaded from this package directory.  There is no fallback: if
the shared library is missing or cannot be loaded, every call raises.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libkiddo_gpu.so")

ABI_VERSION = 1

KGPU_OK, KGPU_EINVAL, KGPU_EUNSUPPORTED, KGPU_ENOMEM, KGPU_ECUDA, KGPU_ETIMEDOUT, \
    KGPU_EOVERFLOW, KGPU_ENOTREADY = range(8)

F32, F64 = 0, 1
STEM_EYTZINGER, STEM_DONNELLY = 0, 1
RES_ARITHMETIC, RES_MAPPED, RES_PRISTINE = 0, 1, 2
SQUARED_EUCLIDEAN, MANHATTAN, CHEBYSHEV, MINKOWSKI3, MINKOWSKI4 = 0, 1, 2, 3, 4
NEAREST_ONE, APPROX_NEAREST_ONE, NEAREST_N, NEAREST_N_WITHIN, WITHIN, WITHIN_UNSORTED, \
    BEST_N_WITHIN = range(7)
FLAG_HOST_BUFFERS = 0x1
FLAG_SPATIAL_ORDER = 0x2
FLAG_ENGINE_WARP = 0x4
FLAG_ENGINE_THREAD = 0x8
FLAG_ENGINE_COOP = 0x20
FLAG_NO_SPATIAL_ORDER = 0x10

# Every symbol include/kiddo_gpu.h declares.
EXPORTED_SYMBOLS = [
    "kgpu_last_error", "kgpu_status_string", "kgpu_abi_version", "kgpu_layout_build",
    "kgpu_layout_build_stems", "kgpu_tree_build", "kgpu_tree_read_layout",
    "kgpu_layout_describe", "kgpu_layout_free", "kgpu_tree_create", "kgpu_tree_destroy",
    "kgpu_tree_info", "kgpu_tree_iter", "kgpu_tree_project", "kgpu_query",
    "kgpu_query_radius_count", "kgpu_query_radius_fill",
    "kgpu_launch_count", "kgpu_query_stats", "kgpu_query_radius_count_noalloc",
    "kgpu_forest_create", "kgpu_forest_destroy", "kgpu_forest_query",
    "kgpu_forest_query_radius_count", "kgpu_forest_query_radius_fill", "kgpu_graph_begin",
    "kgpu_graph_end", "kgpu_graph_launch", "kgpu_graph_destroy", "kgpu_chamfer_loss",
    "kgpu_chamfer_backward", "kgpu_tree_create_flatvec", "kgpu_tree_create_vecofarrays",
    "kgpu_scratch_stats", "kgpu_scratch_trim", "kgpu_archive_inspect",
    "kgpu_tree_create_from_archive", "kgpu_tree_create_mapped",
    "kgpu_tree_create_vecofarrays_mapped",
]


class TreeDesc(ctypes.Structure):
    _fields_ = [
        ("abi_version", ctypes.c_uint32), ("dtype", ctypes.c_int32), ("dims", ctypes.c_uint32),
        ("item_size", ctypes.c_uint32), ("bucket_size", ctypes.c_uint32),
        ("stem_strategy", ctypes.c_int32), ("block_height", ctypes.c_uint32),
        ("resolution", ctypes.c_int32), ("stems", ctypes.c_void_p),
        ("stem_count", ctypes.c_uint64), ("leaf_bytes", ctypes.c_void_p),
        ("leaf_bytes_len", ctypes.c_uint64), ("leaf_extents", ctypes.c_void_p),
        ("leaf_count", ctypes.c_uint64), ("max_stem_level", ctypes.c_int32),
        ("reserved0", ctypes.c_uint32), ("size", ctypes.c_uint64),
        ("max_leaf_len", ctypes.c_uint64),
    ]


class FlatVecDesc(ctypes.Structure):
    _fields_ = [
        ("abi_version", ctypes.c_uint32), ("dtype", ctypes.c_int32), ("dims", ctypes.c_uint32),
        ("stem_strategy", ctypes.c_int32), ("block_height", ctypes.c_uint32),
        ("max_stem_level", ctypes.c_int32), ("stems", ctypes.c_void_p),
        ("stem_count", ctypes.c_uint64), ("columns", ctypes.c_void_p * 4),
        ("items", ctypes.c_void_p), ("extents", ctypes.c_void_p),
        ("leaf_count", ctypes.c_uint64), ("size", ctypes.c_uint64),
    ]


class VecOfArraysDesc(ctypes.Structure):
    _fields_ = [
        ("abi_version", ctypes.c_uint32), ("dtype", ctypes.c_int32), ("dims", ctypes.c_uint32),
        ("stem_strategy", ctypes.c_int32), ("block_height", ctypes.c_uint32),
        ("max_stem_level", ctypes.c_int32), ("stems", ctypes.c_void_p),
        ("stem_count", ctypes.c_uint64), ("bucket", ctypes.c_uint32),
        ("reserved0", ctypes.c_uint32), ("content_points", ctypes.c_void_p),
        ("content_items", ctypes.c_void_p), ("sizes", ctypes.c_void_p),
        ("leaf_count", ctypes.c_uint64),
    ]


class LeafMap(ctypes.Structure):
    _fields_ = [("leaf_idx_map", ctypes.c_void_p), ("len", ctypes.c_uint64),
                ("min_stem_leaf_idx", ctypes.c_uint64)]


class ArchiveFormat(ctypes.Structure):
    _fields_ = [
        ("abi_version", ctypes.c_uint32), ("dtype", ctypes.c_int32), ("dims", ctypes.c_uint32),
        ("stem_strategy", ctypes.c_int32), ("block_height", ctypes.c_uint32),
        ("pointer_width", ctypes.c_uint32), ("big_endian", ctypes.c_uint32),
        ("reserved0", ctypes.c_uint32)]


class ArchiveInfo(ctypes.Structure):
    _fields_ = [
        ("root_offset", ctypes.c_uint64), ("stems_offset", ctypes.c_uint64),
        ("stem_count", ctypes.c_uint64), ("extents_offset", ctypes.c_uint64),
        ("leaf_count", ctypes.c_uint64), ("leaf_bytes_offset", ctypes.c_uint64),
        ("leaf_bytes_len", ctypes.c_uint64), ("resolution", ctypes.c_int32),
        ("max_stem_level", ctypes.c_int32), ("stems_depth", ctypes.c_uint64),
        ("resolution_leaf_count", ctypes.c_uint64), ("size", ctypes.c_uint64),
        ("leaves_size", ctypes.c_uint64), ("max_leaf_len", ctypes.c_uint64),
        ("map_offset", ctypes.c_uint64), ("map_len", ctypes.c_uint64),
        ("min_stem_leaf_idx", ctypes.c_uint64)]


class QueryDesc(ctypes.Structure):
    _fields_ = [
        ("abi_version", ctypes.c_uint32), ("family", ctypes.c_int32), ("metric", ctypes.c_int32),
        ("max_qty", ctypes.c_uint32), ("radius", ctypes.c_double), ("exclusive", ctypes.c_int32),
        ("sorted", ctypes.c_int32), ("periodic_box", ctypes.c_void_p), ("flags", ctypes.c_uint32),
        ("tuning", ctypes.c_uint32),
    ]


class KiddoGpuError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"kiddo_gpu status {status}: {message}")
        self.status = status


_lib = None


def lib():
    """Load libkiddo_gpu.so once; raise if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: run `python -m kiddo_b200.build` first")
    L = ctypes.CDLL(LIB_PATH)
    vp, u64, u32, i32 = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int32
    L.kgpu_last_error.restype = ctypes.c_char_p
    L.kgpu_status_string.restype = ctypes.c_char_p
    L.kgpu_status_string.argtypes = [i32]
    L.kgpu_abi_version.restype = u32
    L.kgpu_layout_build.restype = i32
    L.kgpu_layout_build.argtypes = [i32, u32, vp, vp, u64, i32, ctypes.POINTER(vp)]
    L.kgpu_tree_build.restype = i32
    L.kgpu_tree_build.argtypes = [i32, u32, vp, vp, u64, vp, ctypes.POINTER(vp)]
    L.kgpu_tree_read_layout.restype = i32
    L.kgpu_tree_read_layout.argtypes = [vp, vp, vp, vp, vp]
    L.kgpu_layout_build_stems.restype = i32
    L.kgpu_layout_build_stems.argtypes = [i32, u32, vp, vp, u64, i32, u32, i32, ctypes.POINTER(vp)]
    L.kgpu_layout_describe.restype = i32
    L.kgpu_layout_describe.argtypes = [vp, ctypes.POINTER(TreeDesc)]
    L.kgpu_layout_free.restype = i32
    L.kgpu_layout_free.argtypes = [vp]
    L.kgpu_tree_create.restype = i32
    L.kgpu_tree_create.argtypes = [ctypes.POINTER(TreeDesc), vp, ctypes.POINTER(vp)]
    L.kgpu_tree_create_flatvec.restype = i32
    L.kgpu_tree_create_flatvec.argtypes = [ctypes.POINTER(FlatVecDesc), vp, ctypes.POINTER(vp)]
    L.kgpu_tree_create_vecofarrays.restype = i32
    L.kgpu_tree_create_vecofarrays.argtypes = [ctypes.POINTER(VecOfArraysDesc), vp,
                                               ctypes.POINTER(vp)]
    L.kgpu_tree_destroy.restype = i32
    L.kgpu_tree_destroy.argtypes = [vp]
    L.kgpu_tree_info.restype = i32
    L.kgpu_tree_info.argtypes = [vp, vp]
    L.kgpu_tree_iter.restype = i32
    L.kgpu_tree_iter.argtypes = [vp, vp, vp, vp]
    L.kgpu_tree_project.restype = i32
    L.kgpu_tree_project.argtypes = [vp, vp, u64, vp, vp, vp]
    L.kgpu_query.restype = i32
    L.kgpu_query.argtypes = [vp, ctypes.POINTER(QueryDesc), vp, u64, vp, vp, vp, vp]
    L.kgpu_query_radius_count.restype = i32
    L.kgpu_query_radius_count.argtypes = [vp, ctypes.POINTER(QueryDesc), vp, u64, vp, vp]
    L.kgpu_query_radius_fill.restype = i32
    L.kgpu_query_radius_fill.argtypes = [vp, ctypes.POINTER(QueryDesc), vp, u64, vp, vp, vp, vp]
    L.kgpu_launch_count.restype = u64
    L.kgpu_query_radius_count_noalloc.restype = i32
    L.kgpu_query_radius_count_noalloc.argtypes = [vp, ctypes.POINTER(QueryDesc), vp, u64, vp, vp]
    L.kgpu_query_stats.restype = i32
    L.kgpu_query_stats.argtypes = [vp, ctypes.POINTER(QueryDesc), vp, u64, vp, vp]
    L.kgpu_forest_create.restype = i32
    L.kgpu_forest_create.argtypes = [vp, u32, vp, ctypes.POINTER(vp)]
    L.kgpu_forest_destroy.restype = i32
    L.kgpu_forest_destroy.argtypes = [vp]
    L.kgpu_forest_query.restype = i32
    L.kgpu_forest_query.argtypes = [vp, ctypes.POINTER(QueryDesc), vp, vp, vp, u64, vp, vp, vp, vp]
    L.kgpu_forest_query_radius_count.restype = i32
    L.kgpu_forest_query_radius_count.argtypes = [vp, ctypes.POINTER(QueryDesc), vp, vp, vp, u64,
                                                 vp, vp]
    L.kgpu_forest_query_radius_fill.restype = i32
    L.kgpu_forest_query_radius_fill.argtypes = [vp, ctypes.POINTER(QueryDesc), vp, vp, vp, u64,
                                                vp, u64, vp, vp, vp, vp]
    L.kgpu_graph_begin.restype = i32
    L.kgpu_graph_begin.argtypes = [vp]
    L.kgpu_graph_end.restype = i32
    L.kgpu_graph_end.argtypes = [vp, ctypes.POINTER(vp)]
    L.kgpu_graph_launch.restype = i32
    L.kgpu_graph_launch.argtypes = [vp, vp]
    L.kgpu_graph_destroy.restype = i32
    L.kgpu_graph_destroy.argtypes = [vp]
    L.kgpu_chamfer_loss.restype = i32
    L.kgpu_chamfer_loss.argtypes = [vp, vp, u64, u32, ctypes.c_double, vp, vp, vp]
    L.kgpu_tree_create_mapped.restype = i32
    L.kgpu_tree_create_mapped.argtypes = [ctypes.POINTER(TreeDesc), ctypes.POINTER(LeafMap), vp,
                                          ctypes.POINTER(vp)]
    L.kgpu_tree_create_vecofarrays_mapped.restype = i32
    L.kgpu_tree_create_vecofarrays_mapped.argtypes = [ctypes.POINTER(VecOfArraysDesc),
                                                      ctypes.POINTER(LeafMap), vp,
                                                      ctypes.POINTER(vp)]
    L.kgpu_archive_inspect.restype = i32
    L.kgpu_archive_inspect.argtypes = [vp, u64, ctypes.POINTER(ArchiveFormat),
                                       ctypes.POINTER(ArchiveInfo)]
    L.kgpu_tree_create_from_archive.restype = i32
    L.kgpu_tree_create_from_archive.argtypes = [vp, u64, ctypes.POINTER(ArchiveFormat), vp,
                                                ctypes.POINTER(vp)]
    L.kgpu_scratch_stats.restype = i32
    L.kgpu_scratch_stats.argtypes = [ctypes.c_int32, vp]
    L.kgpu_scratch_trim.restype = i32
    L.kgpu_scratch_trim.argtypes = [ctypes.c_int32]
    L.kgpu_chamfer_backward.restype = i32
    L.kgpu_chamfer_backward.argtypes = [vp, u64, vp, u64, vp, vp, u32, vp, vp, ctypes.c_double,
                                        ctypes.c_float, vp, vp, vp]
    if L.kgpu_abi_version() != ABI_VERSION:
        raise ImportError("libkiddo_gpu.so ABI version mismatch")
    _lib = L
    return L


def check(status):
    if status != KGPU_OK:
        msg = lib().kgpu_last_error().decode(errors="replace")
        raise KiddoGpuError(status, msg)


def launch_count() -> int:
    return int(lib().kgpu_launch_count())


def scratch_stats(device: int = 0):
    """(bytes in use, high-water mark, bytes held) of the library's own
    scratch pool on `device`."""
    import numpy as np
    out = np.zeros(3, dtype=np.uint64)
    check(lib().kgpu_scratch_stats(int(device), ctypes.c_void_p(out.ctypes.data)))
    return tuple(int(x) for x in out)


def scratch_trim(device: int = 0):
    """Give the scratch pool's cached bytes on `device` back to the driver."""
    check(lib().kgpu_scratch_trim(int(device)))
