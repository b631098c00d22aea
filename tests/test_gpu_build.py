"""Device construction (kgpu_tree_build) writes exactly the host builder's
bytes: stems, leaf arena and extents of the reference's soft construction
(src/kd_tree/construction.rs:413-539, 868-968, 1089-1175), and a tree built on
the device answers queries like the oracle."""
import numpy as np
import pytest

import kiddo_b200 as kb
import oracle
from helpers import assert_same_fixed

pytestmark = pytest.mark.gpu


def _device_vs_host(P, items=None):
    import torch
    host = kb.ImmutableKdTree.new_from_slice(P) if items is None else \
        kb.ImmutableKdTree.new_from_entries(items, P)
    ti = None if items is None else torch.from_numpy(items.view(np.int32)).cuda()
    dev = kb.GpuTree.build(torch.from_numpy(P).cuda(), ti)
    stems, lb, ex = dev.read_layout()
    info = dev.info()
    assert info["max_stem_level"] == host.max_stem_level()
    assert info["size"] == host.size()
    assert np.array_equal(stems.view(np.uint8), host.stems().view(np.uint8))
    assert np.array_equal(ex, host.leaf_extents())
    assert np.array_equal(lb, host.leaf_bytes())
    return dev, host


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("dims", [1, 2, 3, 4])
@pytest.mark.parametrize("n", [0, 1, 5, 32, 33, 64, 65, 100, 1000, 100_000])
def test_device_build_matches_host(dtype, dims, n):
    P = np.random.default_rng(n * 7 + dims).random((n, dims)).astype(dtype)
    _device_vs_host(P)


@pytest.mark.parametrize("case", ["all_same", "repeated", "quantized", "axis_degenerate", "grid",
                                  "clustered"])
def test_device_build_adversarial(case):
    """Unsplittable chunks, long and empty leaves, duplicate runs at the pivot
    (the nudge rule of update_pivot, construction.rs:1089-1175)."""
    rng = np.random.default_rng(1)
    if case == "all_same":
        P = np.full((1000, 3), 0.5)
    elif case == "repeated":
        P = np.repeat(rng.random((50, 3)), 20, axis=0)
    elif case == "quantized":
        P = np.round(rng.random((20000, 3)) * 8) / 8
    elif case == "axis_degenerate":
        P = rng.random((20000, 3))
        P[:, 1] = 0.25
    elif case == "grid":
        g = np.linspace(0, 1, 30)
        P = np.stack(np.meshgrid(g, g, g), -1).reshape(-1, 3)
    else:
        P = (rng.random((8, 3))[rng.integers(0, 8, 50000)] +
             rng.normal(0, 1e-3, (50000, 3))).astype(np.float32)
    _device_vs_host(np.ascontiguousarray(P))


def test_device_build_explicit_items_and_large():
    rng = np.random.default_rng(2)
    P = rng.random((1_000_000, 3)).astype(np.float32)
    items = (rng.permutation(1_000_000).astype(np.uint32) * 3 + 7).astype(np.uint32)
    _device_vs_host(P, items)


def test_device_built_tree_answers_like_the_oracle():
    import torch
    rng = np.random.default_rng(3)
    P = rng.random((200_000, 3)).astype(np.float32)
    Q = rng.random((20_000, 3)).astype(np.float32)
    dev = kb.GpuTree.build(torch.from_numpy(P).cuda())
    o = oracle.OracleTree.build(P)
    g = dev.query(torch.from_numpy(Q).cuda()).nearest_n(kb.SquaredEuclidean, 16).execute_gpu()
    d, i, c = (x.cpu().numpy() for x in (g.distances, g.items, g.counts))
    assert_same_fixed(d, i.view(np.uint32), c, *o.nearest_n(Q, 16), "knn16 on a device-built tree")


def test_device_build_rejects_overlong_leaves():
    """More than 1024 equal points in a leaf exceed the reference's leaf
    scratch (leaf_view/mod.rs:18,58-65), on the device as on the host."""
    import torch
    P = np.full((5000, 3), 0.25, dtype=np.float32)
    with pytest.raises(Exception):
        kb.GpuTree.build(torch.from_numpy(P).cuda())


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("dims", [1, 2, 3, 4])
def test_uploaded_tree_reads_back_the_reference_bytes(dtype, dims):
    """A tree uploaded from the reference's layout reads back unchanged, also
    where the device re-encodes the leaves (f32 3-D rows)."""
    rng = np.random.default_rng(dims)
    for n in (0, 7, 33, 5000, 100_000):
        host = kb.ImmutableKdTree.new_from_slice(rng.random((n, dims)).astype(dtype))
        stems, lb, ex = host.to_gpu().read_layout()
        assert np.array_equal(lb, host.leaf_bytes())
        assert np.array_equal(ex, host.leaf_extents())
        assert np.array_equal(stems.view(np.uint8), host.stems().view(np.uint8))
