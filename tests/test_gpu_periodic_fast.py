"""Periodic sorted nearest_n on batches large enough for the plain-walk fast
path (kgpu_periodic_fast.cu: the plain walk answers every row the box's faces
cannot change, the periodic walk the others), against the oracle's periodic
walk (kd_tree/query/periodic.rs:455-619), bit for bit.

The batches mix queries deep inside the box, queries within a list radius of
a face, queries exactly on a face, NaN rows, and tie-heavy grids where many
points sit at the same distance, so both kinds of row and the tie rule are
exercised; trees with points on or outside the box's edges must fall back to
the periodic walk for every row and still agree."""
import numpy as np
import pytest

import kiddo_b200 as kb
import oracle
from helpers import assert_same_fixed

pytestmark = pytest.mark.gpu

METRICS = {"sqeuclidean": kb.SquaredEuclidean, "manhattan": kb.Manhattan,
           "chebyshev": kb.Chebyshev, "minkowski3": kb.Minkowski(3)}


def _queries(rng, n, dims, dtype):
    q = [rng.random((n - 4000, dims)),
         rng.random((1500, dims)) * 0.003,          # within a list radius of the low faces
         1.0 - rng.random((1500, dims)) * 0.003,    # and of the high faces
         np.zeros((500, dims)),                     # exactly on a face
         rng.random((500, dims))]
    Q = np.concatenate(q).astype(dtype)
    Q[-500:, 0] = np.nan                            # rows that find nothing
    return Q


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("dims", [2, 3])
@pytest.mark.parametrize("metric", sorted(METRICS))
def test_fast_path_matches_the_periodic_walk(dtype, dims, metric):
    rng = np.random.default_rng(dims * 7 + len(metric))
    n = 120_000
    c = rng.random((256, dims))
    P = np.concatenate([(c[rng.integers(0, 256, n // 2)] + rng.normal(0, 0.003, (n // 2, dims))) % 1.0,
                        rng.random((n - n // 2, dims))]).astype(dtype)
    P[P >= 1.0] = 0.0
    Q = _queries(rng, 80_000, dims, dtype)
    box = np.ones(dims, dtype=dtype)
    t = kb.ImmutableKdTree.new_from_slice(P)
    o = oracle.OracleTree.build(P)
    M = METRICS[metric]
    for k, radius in ((32, None), (8, None), (32, 0.01 if metric != "minkowski3" else 1e-6)):
        b = t.query(Q).periodic_boundary_condition(box).nearest_n(M, k)
        if radius is not None:
            b = b.within(radius)
        g = b.execute_gpu()
        ref = o.periodic_nearest_n(Q, box, k, radius=np.inf if radius is None else radius,
                                   metric=metric)
        assert_same_fixed(g.distances, g.items, g.counts, *ref, f"pnn{k} r={radius}")


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_fast_path_on_a_tie_heavy_grid(dtype):
    """Points on an integer grid scaled into the box: most distances tie, so
    the rows depend on the walk's arrival order at every cut."""
    g1 = np.arange(40) / 40.0
    P = np.stack(np.meshgrid(g1, g1, g1, indexing="ij"), -1).reshape(-1, 3).astype(dtype)
    P = np.concatenate([P, P[::3]])  # duplicated points: equal distances, distinct items
    rng = np.random.default_rng(3)
    Q = np.concatenate([rng.integers(0, 40, (70_000, 3)) / 40.0,
                        rng.random((10_000, 3))]).astype(dtype)
    box = np.ones(3, dtype=dtype)
    t = kb.ImmutableKdTree.new_from_slice(P)
    o = oracle.OracleTree.build(P)
    for k in (7, 32):
        g = t.query(Q).periodic_boundary_condition(box).nearest_n(kb.SquaredEuclidean, k).execute_gpu()
        assert_same_fixed(g.distances, g.items, g.counts, *o.periodic_nearest_n(Q, box, k),
                          f"grid pnn{k}")


def test_points_outside_the_box_take_the_periodic_walk():
    """A tree with points at or beyond the box's far edge (where the min-image
    bound no longer holds) answers through the periodic walk for every row."""
    rng = np.random.default_rng(11)
    P = rng.random((100_000, 3))
    P[:50] = 1.0 + rng.random((50, 3)) * 0.01
    P[50:60] = 1.0
    Q = rng.random((70_000, 3))
    box = np.ones(3)
    t = kb.ImmutableKdTree.new_from_slice(P)
    o = oracle.OracleTree.build(P)
    g = t.query(Q).periodic_boundary_condition(box).nearest_n(kb.SquaredEuclidean, 16).execute_gpu()
    assert_same_fixed(g.distances, g.items, g.counts, *o.periodic_nearest_n(Q, box, 16), "outside")


def test_fast_path_launches_the_extra_kernels_only_for_large_batches():
    """Below 65,536 queries the periodic walk runs alone (one kernel); above,
    the plain walk, the check and the periodic walk over the listed rows."""
    rng = np.random.default_rng(5)
    P = rng.random((50_000, 3))
    box = np.ones(3)
    t = kb.ImmutableKdTree.new_from_slice(P)
    import torch
    small = torch.from_numpy(rng.random((1000, 3))).cuda()
    large = torch.from_numpy(rng.random((70_000, 3))).cuda()
    for q in (small, large):  # first use measures the tree's bounds once
        t.query(q).periodic_boundary_condition(box).nearest_n(kb.SquaredEuclidean, 8).execute_gpu()
    torch.cuda.synchronize()

    def launches(q):
        n0 = kb.launch_count()
        t.query(q).with_spatial_order(False).periodic_boundary_condition(box).nearest_n(
            kb.SquaredEuclidean, 8).execute_gpu()
        torch.cuda.synchronize()
        return kb.launch_count() - n0

    assert launches(small) == 1
    assert launches(large) == 3


@pytest.mark.parametrize("k", [40, 100])
def test_fast_path_with_lists_beyond_32(k):
    """Lists above 32 entries: the periodic rows go through the row-list
    kernel, the plain rows through the plain engines."""
    rng = np.random.default_rng(k)
    P = rng.random((150_000, 3))
    Q = _queries(rng, 70_000, 3, np.float64)
    box = np.ones(3)
    t = kb.ImmutableKdTree.new_from_slice(P)
    o = oracle.OracleTree.build(P)
    g = t.query(Q).periodic_boundary_condition(box).nearest_n(kb.SquaredEuclidean, k).execute_gpu()
    assert_same_fixed(g.distances, g.items, g.counts, *o.periodic_nearest_n(Q, box, k), f"pnn{k}")


def test_warp_engine_batches_keep_the_periodic_walk():
    """A large batch that asks for the warp engine takes its periodic walk for
    every row, with the same rows as the oracle."""
    rng = np.random.default_rng(21)
    P = rng.random((80_000, 3))
    Q = _queries(rng, 70_500, 3, np.float64)[:-500]  # without the NaN rows
    box = np.ones(3)
    t = kb.ImmutableKdTree.new_from_slice(P)
    o = oracle.OracleTree.build(P)
    g = (t.query(Q).with_engine("warp").periodic_boundary_condition(box)
         .nearest_n(kb.SquaredEuclidean, 8).execute_gpu())
    assert_same_fixed(g.distances, g.items, g.counts, *o.periodic_nearest_n(Q, box, 8), "warp")
