"""nearest_n and best_n_within with k above 32: up to 256 the warp engine
with each warp's list in shared memory, beyond that (and on Donnelly trees,
and for periodic queries) lists in the output rows; bit-exact with the oracle's
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


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("dims", [2, 3])
@pytest.mark.parametrize("bh", [0, 4])
def test_lists_beyond_256_and_donnelly_lists_match_the_oracle(dtype, dims, bh):
    """Lists held in the output rows (BinaryHeap range of the reference,
    result_collection.rs:365-560): nearest_n above 256 and best_n_within above
    256 on Eytzinger trees, every length above 32 on Donnelly trees."""
    rng = np.random.default_rng(dims * 11 + bh)
    P = np.concatenate([rng.random((12_000, dims)),
                        (np.floor(rng.random((4_000, dims)) * 16) / 16)]).astype(dtype)
    items = (rng.permutation(len(P)) % 7000).astype(np.uint32)  # repeated items for best_n
    Q = np.concatenate([rng.random((300, dims)), P[:60]]).astype(dtype)
    t = kb.ImmutableKdTree.new_from_entries(items, P, block_height=bh)
    o = oracle.OracleTree.build(P, items, block_height=bh)
    ks = (33, 100, 300, 1100) if bh else (257, 600, 1500)
    for k in ks:
        g = t.query(Q).nearest_n(kb.SquaredEuclidean, k).execute_gpu()
        assert_same_fixed(g.distances, g.items, g.counts, *o.nearest_n(Q, k), f"k={k}")
        g = t.query(Q).nearest_n(kb.Manhattan, k).within(0.05).unsorted().execute_gpu()
        assert_same_fixed(g.distances, g.items, g.counts,
                          *o.nearest_n(Q, k, radius=0.05, metric="manhattan", sorted=False),
                          f"within unsorted k={k}")
        g = t.query(Q).nearest_n(kb.Chebyshev, k).within(0.02).exclusive_boundaries().execute_gpu()
        assert_same_fixed(g.distances, g.items, g.counts,
                          *o.nearest_n(Q, k, radius=0.02, metric="chebyshev", exclusive=True),
                          f"chebyshev exclusive k={k}")
    for n in ((40, 300) if bh else (300, 700)):
        for excl in (False, True):
            b = t.query(Q).best_n_within(kb.SquaredEuclidean, 0.01, n)
            if excl:
                b = b.exclusive_boundaries()
            g = b.execute_gpu()
            assert_same_fixed(g.distances, g.items, g.counts,
                              *o.best_n_within(Q, 0.01, n, exclusive=excl), f"best_n({n})")


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("dims", [2, 3])
def test_periodic_lists_above_32_match_the_oracle(dtype, dims):
    """periodic nearest_n with k above 32 (the reference's BinaryHeap,
    periodic.rs:682-791), lists in the output rows."""
    rng = np.random.default_rng(dims + 40)
    P = rng.random((15_000, dims)).astype(dtype)
    Q = np.concatenate([rng.random((400, dims)), rng.random((100, dims)) * 0.01,
                        1 - rng.random((100, dims)) * 0.01]).astype(dtype)
    box = np.ones(dims, dtype=dtype)
    t = kb.ImmutableKdTree.new_from_slice(P)
    o = oracle.OracleTree.build(P)
    for k, r in ((33, None), (100, 0.002), (400, None)):
        b = t.query(Q).periodic_boundary_condition(box).nearest_n(kb.SquaredEuclidean, k)
        if r is not None:
            b = b.within(r)
        g = b.execute_gpu()
        ref = o.periodic_nearest_n(Q, box, k, radius=np.inf if r is None else r)
        assert_same_fixed(g.distances, g.items, g.counts, *ref, f"periodic k={k}")


def test_unsorted_rows_between_25_and_32_come_out_sorted():
    """Above 24 entries the reference's unsorted nearest_n collects into a
    BinaryHeap (nearest_n_within.rs:27), so rows that never fill come out
    sorted like the oracle's; at 24 and below they keep arrival order."""
    rng = np.random.default_rng(8)
    P = rng.random((20_000, 3)).astype(np.float32)
    Q = rng.random((2_000, 3)).astype(np.float32)
    t = kb.ImmutableKdTree.new_from_slice(P)
    o = oracle.OracleTree.build(P)
    for k in (20, 24, 25, 30, 32):
        for engine in (None, "warp", "thread"):
            g = t.query(Q).with_engine(engine).nearest_n(kb.SquaredEuclidean, k).within(2e-4) \
                .unsorted().execute_gpu()
            ref = o.nearest_n(Q, k, radius=2e-4, sorted=False)
            assert (ref[2] < k).any()
            assert_same_fixed(g.distances, g.items, g.counts, *ref, f"k={k} engine={engine}")


def test_large_k_limits():
    rng = np.random.default_rng(6)
    Q4 = rng.random((10, 4))
    t4 = kb.ImmutableKdTree.new_from_slice(rng.random((5000, 4)))
    with pytest.raises(kb.KiddoGpuError):
        t4.query(Q4).nearest_n(kb.SquaredEuclidean, 257).execute_gpu()
    with pytest.raises(kb.KiddoGpuError):
        t4.query(Q4).periodic_boundary_condition(np.ones(4)).nearest_n(
            kb.SquaredEuclidean, 33).execute_gpu()
    t = kb.ImmutableKdTree.new_from_slice(rng.random((5000, 3)))
    with pytest.raises(kb.KiddoGpuError):
        t.query(rng.random((10, 3))).nearest_n(kb.SquaredEuclidean, (1 << 20) + 1).execute_gpu()
