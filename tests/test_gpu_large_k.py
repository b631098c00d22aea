"""nearest_n and best_n_within with k above 32 (up to 256): the warp engine
with each warp's list in shared memory, bit-exact with the oracle's
collectors (the reference's ThresholdVec, results/result_collection.rs:136-215:
the k smallest by (distance, arrival order), arrival order kept for an
unsorted list that never filled; best_n_within.rs:88-196: the n smallest
items among the hits)."""
import numpy as np
import pytest

import kiddo_b200 as kb
import oracle
from helpers import assert_same_fixed

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("dims", [2, 3, 4])
def test_large_k_matches_the_oracle(dtype, dims):
    rng = np.random.default_rng(dims * 7)
    P = (np.floor(rng.random((20000, dims)) * 64) / 64).astype(dtype)  # ties at every distance
    Q = np.concatenate([rng.random((600, dims)).astype(dtype), P[:100]])
    t = kb.ImmutableKdTree.new_from_slice(P)
    o = oracle.OracleTree.build(P)
    for k in (33, 64, 100, 192, 256):
        g = t.query(Q).nearest_n(kb.SquaredEuclidean, k).execute_gpu()
        assert_same_fixed(g.distances, g.items, g.counts, *o.nearest_n(Q, k), f"k={k}")
    if dims in (2, 3):
        # up to k = 64 both engines serve it: per-thread lists (128-thread
        # blocks) by default, warp lists on request
        for engine in ("thread", "warp"):
            g = t.query(Q).with_engine(engine).nearest_n(kb.SquaredEuclidean, 48).execute_gpu()
            assert_same_fixed(g.distances, g.items, g.counts, *o.nearest_n(Q, 48),
                              f"k=48 engine={engine}")
    for k in (48, 200):
        g = t.query(Q).nearest_n(kb.Manhattan, k).unsorted().execute_gpu()
        assert_same_fixed(g.distances, g.items, g.counts,
                          *o.nearest_n(Q, k, metric="manhattan", sorted=False), f"unsorted k={k}")
        for excl in (False, True):
            b = t.query(Q).nearest_n(kb.SquaredEuclidean, k).within(0.002)
            if excl:
                b = b.exclusive_boundaries()
            g = b.execute_gpu()
            assert_same_fixed(g.distances, g.items, g.counts,
                              *o.nearest_n(Q, k, radius=0.002, exclusive=excl),
                              f"within k={k} excl={excl}")


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_large_best_n_matches_the_oracle(dtype):
    rng = np.random.default_rng(21)
    P = rng.random((30000, 3)).astype(dtype)
    items = (rng.permutation(30000) % 9000).astype(np.uint32)  # repeated items
    Q = rng.random((800, 3)).astype(dtype)
    t = kb.ImmutableKdTree.new_from_entries(items, P)
    o = oracle.OracleTree.build(P, items)
    for n in (33, 100, 256):
        for excl in (False, True):
            b = t.query(Q).best_n_within(kb.SquaredEuclidean, 0.004, n)
            if excl:
                b = b.exclusive_boundaries()
            g = b.execute_gpu()
            assert_same_fixed(g.distances, g.items, g.counts,
                              *o.best_n_within(Q, 0.004, n, exclusive=excl),
                              f"best_n({n}) excl={excl}")


def test_large_k_small_trees_and_counters():
    rng = np.random.default_rng(5)
    for n in (0, 1, 40, 300):
        P = rng.random((n, 3))
        Q = rng.random((200, 3))
        t = kb.ImmutableKdTree.new_from_slice(P)
        o = oracle.OracleTree.build(P)
        g = t.query(Q).nearest_n(kb.SquaredEuclidean, 128).execute_gpu()
        assert_same_fixed(g.distances, g.items, g.counts, *o.nearest_n(Q, 128), f"n={n}")
    P = rng.random((50000, 3)).astype(np.float32)
    Q = rng.random((5000, 3)).astype(np.float32)
    t = kb.ImmutableKdTree.new_from_slice(P)
    _, _, _, ost = oracle.OracleTree.build(P).nearest_n(Q, 100, stats=True)
    assert np.array_equal(t.query(Q).nearest_n(kb.SquaredEuclidean, 100).traversal_stats(), ost)


def test_large_k_limits():
    rng = np.random.default_rng(6)
    P = rng.random((5000, 3))
    Q = rng.random((10, 3))
    t = kb.ImmutableKdTree.new_from_slice(P)
    with pytest.raises(kb.KiddoGpuError):
        t.query(Q).nearest_n(kb.SquaredEuclidean, 257).execute_gpu()
    with pytest.raises(kb.KiddoGpuError):
        t.query(Q).best_n_within(kb.SquaredEuclidean, 0.1, 257).execute_gpu()
    with pytest.raises(kb.KiddoGpuError):
        t.query(Q).periodic_boundary_condition(np.ones(3)).nearest_n(
            kb.SquaredEuclidean, 64).execute_gpu()
    d = kb.ImmutableKdTree.new_from_slice(P, block_height=3)
    with pytest.raises(kb.KiddoGpuError):
        d.query(Q).nearest_n(kb.SquaredEuclidean, 64).execute_gpu()
    with pytest.raises(kb.KiddoGpuError):
        d.query(Q).best_n_within(kb.SquaredEuclidean, 0.1, 64).execute_gpu()
