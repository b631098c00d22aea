"""Trees with FlatVec leaves (src/leaf_strategy/flat_vec.rs:20-26) through
kgpu_tree_create_flatvec.

Construction hands FlatVec::append_leaf (flat_vec.rs:189-210) the same leaf
chunks, in the same point order, as VecOfArenas::append_leaf, so a FlatVec tree
of the same points has the same stems and leaves as the ImmutableKdTree.  The
upload re-encodes its columns as the VecOfArenas tiles: it reads back as the
ImmutableKdTree's bytes and answers every family like the oracle.
"""
import numpy as np
import pytest

import kiddo_b200 as kb
import oracle
from helpers import assert_same_csr, assert_same_fixed, flatvec_parts, vecofarrays_parts

pytestmark = pytest.mark.gpu


def _flat_pair(P, bh=0):
    host = kb.ImmutableKdTree.new_from_slice(P, block_height=bh)
    cols, items, ext = flatvec_parts(host)
    g = kb.GpuTree.from_flatvec(host.stems(), cols, items, ext, host.max_stem_level(),
                                block_height=bh)
    return host, g


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("dims", [1, 2, 3, 4])
def test_flatvec_upload_reads_back_the_arena(dtype, dims):
    rng = np.random.default_rng(dims)
    for n in (0, 7, 33, 20000):
        host, g = _flat_pair(rng.random((n, dims)).astype(dtype))
        stems, lb, ex = g.read_layout()
        assert np.array_equal(lb, host.leaf_bytes())
        assert np.array_equal(ex, host.leaf_extents())
        assert np.array_equal(stems.view(np.uint8), host.stems().view(np.uint8))


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("bh", [0, 3])
def test_flatvec_tree_answers_like_the_oracle(dtype, bh):
    rng = np.random.default_rng(11 + bh)
    P = rng.random((30000, 3)).astype(dtype)
    Q = np.concatenate([rng.random((2000, 3)).astype(dtype), P[:100]])
    _, g = _flat_pair(P, bh)
    o = oracle.OracleTree.build(P, block_height=bh)
    r = g.query(Q).nearest_one(kb.SquaredEuclidean).execute_gpu()
    od, oi = o.nearest_one(Q)
    assert_same_fixed(r.distances, r.items, np.ones(len(Q)), od, oi, np.ones(len(Q)), "nn1")
    r = g.query(Q).nearest_n(kb.Manhattan, 16).execute_gpu()
    assert_same_fixed(r.distances, r.items, r.counts, *o.nearest_n(Q, 16, metric="manhattan"),
                      "nearest_n(16)")
    r = g.query(Q).best_n_within(kb.SquaredEuclidean, 0.002, 5).execute_gpu()
    assert_same_fixed(r.distances, r.items, r.counts, *o.best_n_within(Q, 0.002, 5), "best_n")
    r = g.query(Q).within(kb.Chebyshev, 0.02).execute_gpu()
    assert_same_csr((r.offsets, r.distances, r.items), o.within(Q, 0.02, metric="chebyshev"),
                    "within")


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("dims", [2, 3])
def test_vecofarrays_upload_reads_back_and_answers(dtype, dims):
    """A VecOfArrays tree (vec_of_arrays.rs:51-97) of the same points holds the
    same leaf chunks; kgpu_tree_create_vecofarrays re-encodes its live slots as
    VecOfArenas tiles, so it reads back as the ImmutableKdTree's bytes."""
    rng = np.random.default_rng(40 + dims)
    for n in (0, 5, 20000):
        P = rng.random((n, dims)).astype(dtype)
        host = kb.ImmutableKdTree.new_from_slice(P)
        pts, its, sizes = vecofarrays_parts(host)
        g = kb.GpuTree.from_vec_of_arrays(host.stems(), pts, its, sizes, host.max_stem_level())
        stems, lb, ex = g.read_layout()
        assert np.array_equal(lb, host.leaf_bytes())
        assert np.array_equal(ex, host.leaf_extents())
    Q = np.concatenate([rng.random((1000, dims)).astype(dtype), P[:50]])
    o = oracle.OracleTree.build(P)
    r = g.query(Q).nearest_n(kb.SquaredEuclidean, 8).execute_gpu()
    assert_same_fixed(r.distances, r.items, r.counts, *o.nearest_n(Q, 8), "nearest_n(8)")
