"""C ABI checks that need no GPU: the library loads, exports every symbol that
include/kiddo_gpu.h declares, and rejects bad input with a status code (the
reference panics instead: periodic.rs:710-717, builder.rs:1538-1543)."""
import ctypes
import os
import re

import numpy as np
import pytest

import kiddo_b200 as kb
from kiddo_b200 import _capi as C

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "kiddo_gpu.h")).read()
    return sorted(set(re.findall(r"\b(kgpu_[a-z_0-9]+)\s*\(", txt)))


def test_exports_every_declared_symbol():
    L = C.lib()
    syms = header_symbols()
    assert len(syms) >= 10
    for s in syms:
        assert hasattr(L, s), f"{s} declared in include/kiddo_gpu.h but not exported"
    assert sorted(C.EXPORTED_SYMBOLS) == syms


def test_no_device_only_code_reached_from_host():
    """nvcc gives a device-only function called from host code (through
    --expt-relaxed-constexpr or a template) a host body of exit(1), which ends
    the caller's process with no message.  The library must import no exit."""
    import shutil
    import subprocess
    nm = shutil.which("nm")
    if nm is None:
        pytest.skip("nm not available")
    out = subprocess.run([nm, "-D", "--undefined-only", C.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    names = {line.split()[-1].split("@")[0] for line in out.splitlines() if line.strip()}
    assert "exit" not in names and "_exit" not in names


def test_version_and_status_strings():
    L = C.lib()
    assert L.kgpu_abi_version() == C.ABI_VERSION
    assert L.kgpu_status_string(C.KGPU_EUNSUPPORTED) == b"unsupported layout or option"


def _desc_of(tree):
    d = C.TreeDesc()
    ctypes.memmove(ctypes.byref(d), ctypes.byref(tree._desc), ctypes.sizeof(d))
    return d


def _create(d):
    h = ctypes.c_void_p()
    return C.lib().kgpu_tree_create(ctypes.byref(d), None, ctypes.byref(h))


def test_tree_create_rejects_bad_layouts_before_touching_the_device():
    t = kb.ImmutableKdTree.new_from_slice(np.random.default_rng(0).random((1000, 3)))
    cases = [
        ("abi_version", 99, C.KGPU_EINVAL),
        ("dtype", 7, C.KGPU_EINVAL),
        ("dims", 9, C.KGPU_EUNSUPPORTED),
        ("item_size", 8, C.KGPU_EUNSUPPORTED),
        ("bucket_size", 16, C.KGPU_EUNSUPPORTED),
        ("stem_strategy", C.STEM_DONNELLY, C.KGPU_EUNSUPPORTED),
        ("resolution", C.RES_MAPPED, C.KGPU_EINVAL),  # a Mapped tree needs its leaf map
        ("max_stem_level", 40, C.KGPU_EUNSUPPORTED),
        ("leaf_count", 5, C.KGPU_EINVAL),
        ("size", 999, C.KGPU_EINVAL),
        ("leaf_bytes_len", 100, C.KGPU_EINVAL),
    ]
    for field, value, status in cases:
        d = _desc_of(t)
        setattr(d, field, value)
        assert _create(d) == status, field
        assert C.lib().kgpu_last_error()


def test_tree_create_rejects_f32_3d_offsets_off_16_bytes():
    """f32 3-D leaves take 16 bytes per point, so the reference's leaf offsets
    are multiples of 16, and the device reads each point as one aligned
    16-byte row; an offset that is only 8-byte aligned is rejected."""
    t = kb.ImmutableKdTree.new_from_slice(
        np.random.default_rng(1).random((1000, 3)).astype(np.float32))
    ex = t.leaf_extents().astype(np.uint64).copy()
    assert ex.shape[0] >= 2 and all(int(o) % 16 == 0 for o in ex[:, 0])
    ex[1, 0] += 8
    d = _desc_of(t)
    d.leaf_extents = ex.ctypes.data
    assert _create(d) == C.KGPU_EINVAL
    assert b"multiple of 16" in C.lib().kgpu_last_error()


def test_flatvec_create_rejects_bad_layouts_before_touching_the_device():
    """kgpu_tree_create_flatvec checks the FlatVec arrays on the host."""
    L = C.lib()
    n = 100
    cols = [np.zeros(n, dtype=np.float32) for _ in range(3)]
    items = np.arange(n, dtype=np.uint32)

    def create(extents, size=n, columns=cols, it=items, dims=3):
        ext = np.ascontiguousarray(extents, dtype=np.uint32).reshape(-1, 2)
        d = C.FlatVecDesc()
        d.abi_version = C.ABI_VERSION
        d.dtype = C.F32
        d.dims = dims
        d.max_stem_level = -1
        for j, c in enumerate(columns):
            d.columns[j] = c.ctypes.data if c is not None else None
        d.items = it.ctypes.data if it is not None else None
        d.extents = ext.ctypes.data
        d.leaf_count = ext.shape[0]
        d.size = size
        h = ctypes.c_void_p()
        return L.kgpu_tree_create_flatvec(ctypes.byref(d), None, ctypes.byref(h))

    assert create([(0, 60), (60, 101)]) == C.KGPU_EINVAL       # past the points
    assert create([(0, 60), (50, 40)]) == C.KGPU_EINVAL        # start after end
    assert create([(0, 60), (60, 90)]) == C.KGPU_EINVAL        # lengths do not sum to size
    assert create([(0, 100)], columns=cols[:2] + [None]) == C.KGPU_EINVAL
    assert create([(0, 100)], it=None) == C.KGPU_EINVAL
    assert create([(0, 100)], dims=5) == C.KGPU_EUNSUPPORTED
    big = [np.zeros(2000, dtype=np.float32) for _ in range(3)]
    assert create([(0, 2000)], size=2000, columns=big,
                  it=np.arange(2000, dtype=np.uint32)) == C.KGPU_EINVAL  # leaf over 1024
    assert L.kgpu_last_error()


def test_flatvec_parts_round_trip():
    """The test helper's FlatVec form holds every point once, leaf by leaf."""
    from helpers import flatvec_parts
    P = np.random.default_rng(4).random((5000, 3))
    t = kb.ImmutableKdTree.new_from_slice(P)
    cols, items, ext = flatvec_parts(t)
    assert ext.shape == (t.leaf_count(), 2) and int(ext[-1, 1]) == 5000
    assert np.array_equal(np.sort(items), np.arange(5000, dtype=np.uint32))
    assert np.array_equal(np.stack(cols, 1), P[items])


def test_layout_build_rejects_bad_arguments():
    L = C.lib()
    h = ctypes.c_void_p()
    pts = np.zeros((10, 3), dtype=np.float32)
    assert L.kgpu_layout_build(5, 3, pts.ctypes.data, None, 10, 1, ctypes.byref(h)) == C.KGPU_EINVAL
    assert L.kgpu_layout_build(0, 9, pts.ctypes.data, None, 10, 1, ctypes.byref(h)) == \
        C.KGPU_EUNSUPPORTED
    assert L.kgpu_layout_build(0, 3, None, None, 10, 1, ctypes.byref(h)) == C.KGPU_EINVAL
    # a chunk of more than 1024 identical points exceeds the leaf scratch capacity
    # (leaf_view/mod.rs:18, 58-65), which the reference asserts at construction
    same = np.zeros((2000, 3), dtype=np.float32)
    assert L.kgpu_layout_build(0, 3, same.ctypes.data, None, 2000, 1, ctypes.byref(h)) == \
        C.KGPU_EOVERFLOW


def test_query_builder_typestate_errors():
    # runtime mirror of the reference's compile-time typestate (builder.rs:1994-2077)
    t = kb.ImmutableKdTree.new_from_slice(np.random.default_rng(0).random((100, 3)))
    q = np.zeros((1, 3))

    class Dummy:
        pass

    b = kb.QueryBuilder.__new__(kb.QueryBuilder)
    kb.QueryBuilder.__init__(b, type("T", (), {"dtype": np.dtype(np.float64), "dims": 3})(), q)
    with pytest.raises(TypeError):
        b.approx()
    b.nearest_n(kb.SquaredEuclidean, 3)
    with pytest.raises(TypeError):
        b.approx()
    with pytest.raises(TypeError):
        b.periodic_boundary_condition([1, 1, 1])
    with pytest.raises(ValueError):
        kb.QueryBuilder(b.tree, q).nearest_n(kb.SquaredEuclidean, 0)
    with pytest.raises(ValueError):
        kb.QueryBuilder(b.tree, q).periodic_boundary_condition([1.0, 0.0, 1.0])
    with pytest.raises(TypeError):
        kb.QueryBuilder(b.tree, q).periodic_boundary_condition([1, 1, 1]).best_n_within(
            kb.SquaredEuclidean, 0.1, 3)
    with pytest.raises(TypeError):
        kb.QueryBuilder(b.tree, q).nearest_one(Dummy)
    with pytest.raises(TypeError):
        kb.QueryBuilder(b.tree, q).nearest_one(kb.SquaredEuclidean).exclusive_boundaries()
    with pytest.raises(TypeError):
        kb.QueryBuilder(b.tree, q).execute_gpu()


def test_vecofarrays_create_rejects_bad_leaves_before_touching_the_device():
    """kgpu_tree_create_vecofarrays checks the leaf arrays on the host."""
    import ctypes
    from kiddo_b200 import _capi as C
    L = C.lib()
    pts = np.zeros((2, 3, 4), np.float32)
    its = np.zeros((2, 4), np.uint32)

    def create(sizes, bucket=4, dims=3):
        sz = np.ascontiguousarray(sizes, dtype=np.uint64)
        d = C.VecOfArraysDesc()
        d.abi_version = C.ABI_VERSION
        d.dtype = C.F32
        d.dims = dims
        d.max_stem_level = 0
        d.bucket = bucket
        d.content_points = pts.ctypes.data
        d.content_items = its.ctypes.data
        d.sizes = sz.ctypes.data
        d.leaf_count = 2
        h = ctypes.c_void_p()
        return L.kgpu_tree_create_vecofarrays(ctypes.byref(d), None, ctypes.byref(h))

    assert create([4, 5]) == C.KGPU_EINVAL     # a leaf larger than its bucket
    assert create([1, 1], bucket=0) == C.KGPU_EINVAL
    assert create([1, 1], dims=5) == C.KGPU_EINVAL


def test_descriptor_layouts_match_the_header(tmp_path):
    """Every ctypes mirror of a descriptor struct has the C header's size and
    field offsets (gcc compiles a probe against include/kiddo_gpu.h)."""
    import shutil
    import subprocess
    from kiddo_b200 import _capi as C
    if shutil.which("gcc") is None:
        pytest.skip("no gcc")
    pairs = {"kgpu_tree_desc": C.TreeDesc, "kgpu_flatvec_desc": C.FlatVecDesc,
             "kgpu_vecofarrays_desc": C.VecOfArraysDesc, "kgpu_query_desc": C.QueryDesc}
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "kiddo_gpu.h"',
             "int main(void) {"]
    for cname, cls in pairs.items():
        lines.append(f'  printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "probe.c"
    src.write_text("\n".join(lines) + "\n")
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-I", inc, str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    for line in out.splitlines():
        cname, fname, value = line.split()
        cls = pairs[cname]
        want = ctypes.sizeof(cls) if fname == "sizeof" else getattr(cls, fname).offset
        assert int(value) == want, (cname, fname, int(value), want)


def test_mapped_create_rejects_bad_leaf_maps_before_touching_the_device():
    """kgpu_tree_create_mapped checks the map against the stems: leaf indices
    inside leaf_count, and every walk from the root ending at a mapped
    terminal stem (where the reference would panic)."""
    import oracle
    rng = np.random.default_rng(1)
    o = oracle.OracleTree.build_mutable(rng.random((3000, 3)))
    lay = o.layout()
    m, mn = o.leaf_map()
    t = kb.ImmutableKdTree.from_layout(np.float64, 3, lay.stems, lay.leaf_bytes, lay.extents,
                                       lay.max_stem_level, lay.size, lay.max_leaf_len)

    def create(mp):
        d = _desc_of(t)
        d.resolution = C.RES_MAPPED
        lm = C.LeafMap()
        mp = np.ascontiguousarray(mp, dtype=np.uint64)
        lm.leaf_idx_map = mp.ctypes.data if mp.size else None
        lm.len = mp.size
        lm.min_stem_leaf_idx = mn
        h = ctypes.c_void_p()
        return C.lib().kgpu_tree_create_mapped(ctypes.byref(d), ctypes.byref(lm), None,
                                               ctypes.byref(h))
    bad = m.copy()
    bad[np.nonzero(bad != 2 ** 64 - 1)[0][0]] = lay.leaf_count  # beyond the leaves
    assert create(bad) == C.KGPU_EINVAL
    bad = m.copy()
    bad[np.nonzero(bad != 2 ** 64 - 1)[0][-1]] = 2 ** 64 - 1  # a walk with no leaf
    assert create(bad) == C.KGPU_EINVAL
    assert b"reaches no leaf" in C.lib().kgpu_last_error()
    d = _desc_of(t)  # a map needs the Mapped resolution
    lm = C.LeafMap()
    assert C.lib().kgpu_tree_create_mapped(ctypes.byref(d), ctypes.byref(lm), None,
                                           ctypes.byref(ctypes.c_void_p())) == C.KGPU_EINVAL
