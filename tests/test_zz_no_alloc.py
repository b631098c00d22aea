"""The radius counting pass that allocates nothing (kgpu_query_radius_count_noalloc).

Some callers cannot allocate device memory while they query: a process whose
HBM is reserved up front by its own pool, a latency-critical loop, a framework
that owns every device buffer.  For them the engine keeps the prefix-sum
scratch in a fixed device array instead of allocating it.  This file runs last
(pytest collects it after every other test file) and must also pass on its own
in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import kiddo_b200 as kb
from kiddo_b200 import _capi as C

pytestmark = pytest.mark.gpu

MAX_QUERIES = 1 << 24


def _desc(radius, family=C.WITHIN, flags=0):
    d = C.QueryDesc()
    d.abi_version = C.ABI_VERSION
    d.family = family
    d.metric = C.SQUARED_EUCLIDEAN
    d.radius = radius
    d.sorted = 1 if family == C.WITHIN else 0
    d.flags = flags
    return d


def _count(fn, tree, d, dq, nq, offsets):
    import torch
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    return fn(tree._h, ctypes.byref(d), ctypes.c_void_p(dq.data_ptr()), nq,
              ctypes.c_void_p(offsets.data_ptr()), st)


def _default_pool_usage():
    """(bytes in use, high-water mark, bytes held) of the device's default
    stream-ordered pool, read through the CUDA runtime bindings."""
    from cuda.bindings import runtime as rt
    err, pool = rt.cudaDeviceGetDefaultMemPool(0)
    assert err == rt.cudaError_t.cudaSuccess
    out = []
    for a in (rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemCurrent,
              rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemHigh,
              rt.cudaMemPoolAttr.cudaMemPoolAttrReservedMemCurrent):
        err, v = rt.cudaMemPoolGetAttribute(pool, a)
        assert err == rt.cudaError_t.cudaSuccess
        out.append(int(v))
    return tuple(out), pool


def _reset_default_pool_high(pool):
    from cuda.bindings import driver, runtime as rt
    err, = rt.cudaMemPoolSetAttribute(pool, rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemHigh,
                                      driver.cuuint64_t(0))
    assert err == rt.cudaError_t.cudaSuccess


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("block_height", [0, 4])
@pytest.mark.parametrize("family", [C.WITHIN, C.WITHIN_UNSORTED])
def test_noalloc_count_matches_the_allocating_count_on_two_calls_in_a_row(dtype, block_height,
                                                                        family):
    import torch
    L = C.lib()
    rng = np.random.default_rng(4)
    P = rng.random((200_000, 3)).astype(dtype)
    tree = kb.ImmutableKdTree.new_from_slice(P, block_height=block_height).to_gpu()
    # different batches and radii back to back: each call must not see
    # anything the previous one left in the shared scratch (the sizes cover
    # an empty batch, one query, exactly one scan tile and one past it)
    for nq, radius in ((300_000, 2e-4), (70_001, 5e-5), (0, 1e-4), (1, 1e-3), (2048, 1e-4),
                       (2049, 3e-4)):
        Q = rng.random((max(nq, 1), 3)).astype(dtype)
        dq = torch.from_numpy(Q).cuda()
        ref = torch.empty(nq + 1, dtype=torch.int64, device="cuda")
        got = torch.full((nq + 1,), -1, dtype=torch.int64, device="cuda")
        d = _desc(radius, family)
        C.check(_count(L.kgpu_query_radius_count, tree, d, dq, nq, ref))
        torch.cuda.synchronize()
        C.check(_count(L.kgpu_query_radius_count_noalloc, tree, d, dq, nq, got))
        torch.cuda.synchronize()
        assert torch.equal(got, ref), (nq, radius)  # integer offsets: exact
        if nq >= 2048:
            assert int(got[-1]) > 0


def test_noalloc_count_allocates_nothing():
    """Neither the library's scratch pool, nor the device's default pool, nor
    torch's allocator gains a byte (not even transiently: the high-water marks
    are reset first) across two calls."""
    import torch
    L = C.lib()
    rng = np.random.default_rng(6)
    tree = kb.ImmutableKdTree.new_from_slice(rng.random((100_000, 3)).astype(np.float32)).to_gpu()
    nq = 500_000
    dq = torch.from_numpy(rng.random((nq, 3)).astype(np.float32)).cuda()
    got = torch.empty(nq + 1, dtype=torch.int64, device="cuda")
    ref = torch.empty(nq + 1, dtype=torch.int64, device="cuda")
    d = _desc(2e-4)
    C.check(_count(L.kgpu_query_radius_count_noalloc, tree, d, dq, nq, got))  # first-call set-up
    torch.cuda.synchronize()
    C.scratch_trim(0)
    lib_before = C.scratch_stats(0)
    default_before, pool = _default_pool_usage()
    _reset_default_pool_high(pool)
    default_before, _ = _default_pool_usage()
    torch_before = (torch.cuda.memory_allocated(), torch.cuda.memory_reserved())
    for _ in range(2):
        C.check(_count(L.kgpu_query_radius_count_noalloc, tree, d, dq, nq, got))
    torch.cuda.synchronize()
    lib_after = C.scratch_stats(0)
    default_after, _ = _default_pool_usage()
    assert lib_after[0] == lib_before[0] and lib_after[2] == lib_before[2]
    assert lib_after[1] == lib_before[1]  # high-water mark: no transient allocation
    assert default_after == default_before
    assert (torch.cuda.memory_allocated(), torch.cuda.memory_reserved()) == torch_before
    # and the allocating count does use the library's pool, so the probe can see one
    C.check(_count(L.kgpu_query_radius_count, tree, d, dq, nq, ref))
    torch.cuda.synchronize()
    assert C.scratch_stats(0)[1] > lib_before[1]
    assert torch.equal(got, ref)


def test_noalloc_count_rejects_host_buffers_and_oversized_batches():
    import torch
    L = C.lib()
    P = np.random.default_rng(5).random((5000, 3)).astype(np.float32)
    tree = kb.ImmutableKdTree.new_from_slice(P).to_gpu()
    # buffers really hold MAX_QUERIES + 1 rows, so nothing could read out of
    # bounds even if the size check were missing
    n = MAX_QUERIES + 1
    dq = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
    off = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
    assert _count(L.kgpu_query_radius_count_noalloc, tree, _desc(1e-4), dq, n, off) == \
        C.KGPU_EOVERFLOW
    assert b"16,777,216" in L.kgpu_last_error()
    assert _count(L.kgpu_query_radius_count_noalloc, tree,
                  _desc(1e-4, flags=C.FLAG_HOST_BUFFERS), dq, 10, off) == C.KGPU_EINVAL
    assert _count(L.kgpu_query_radius_count_noalloc, tree,
                  _desc(1e-4, family=C.NEAREST_ONE), dq, 10, off) == C.KGPU_EINVAL
