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
    d.sorted = 1
    d.flags = flags
    return d


def _count(fn, tree, d, dq, nq, offsets):
    import torch
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    return fn(tree._h, ctypes.byref(d), ctypes.c_void_p(dq.data_ptr()), nq,
              ctypes.c_void_p(offsets.data_ptr()), st)


def test_noalloc_count_matches_the_allocating_count_on_two_calls_in_a_row():
    import torch
    L = C.lib()
    rng = np.random.default_rng(4)
    P = rng.random((200_000, 3)).astype(np.float32)
    tree = kb.ImmutableKdTree.new_from_slice(P).to_gpu()
    # two different batches and radii back to back: the second call must not
    # see anything the first left in the shared scratch
    for nq, radius in ((300_000, 2e-4), (70_001, 5e-5)):
        Q = rng.random((nq, 3)).astype(np.float32)
        dq = torch.from_numpy(Q).cuda()
        ref = torch.empty(nq + 1, dtype=torch.int64, device="cuda")
        got = torch.full((nq + 1,), -1, dtype=torch.int64, device="cuda")
        d = _desc(radius)
        C.check(_count(L.kgpu_query_radius_count, tree, d, dq, nq, ref))
        C.check(_count(L.kgpu_query_radius_count_noalloc, tree, d, dq, nq, got))
        torch.cuda.synchronize()
        assert torch.equal(got, ref)  # integer offsets: exact
        assert int(got[-1]) > 0


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
