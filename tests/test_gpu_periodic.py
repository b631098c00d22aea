"""Periodic boundary conditions on the GPU vs the oracle, bit for bit
(kd_tree/query/periodic.rs: nearest_one via home + image queries; plural
families via the interval-aware traversal with min-image leaf distances)."""
import numpy as np
import pytest

import kiddo_b200 as kb
import oracle
from helpers import assert_same_csr, assert_same_fixed, load_kats

pytestmark = pytest.mark.gpu


def _data(dtype, dims, rng, n):
    # clumps wrapped into the box plus a uniform part, so many queries sit
    # near a face and need image shifts
    c = rng.random((64, dims))
    P = np.concatenate([(c[rng.integers(0, 64, n // 2)] + rng.normal(0, 0.01, (n // 2, dims))) % 1.0,
                        rng.random((n - n // 2, dims))])
    return P.astype(dtype)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("dims", [2, 3])
@pytest.mark.parametrize("metric", ["sqeuclidean", "manhattan", "chebyshev", "minkowski3",
                                    "minkowski4"])
def test_periodic_families(dtype, dims, metric):
    rng = np.random.default_rng(dims * 10 + (metric == "manhattan"))
    P = _data(dtype, dims, rng, 20000)
    Q = np.concatenate([rng.random((1500, dims)), rng.random((300, dims)) * 0.01,
                        1 - rng.random((300, dims)) * 0.01, P[:100]]).astype(dtype)
    box = np.ones(dims, dtype=dtype)
    t = kb.ImmutableKdTree.new_from_slice(P)
    o = oracle.OracleTree.build(P)
    M = {"sqeuclidean": kb.SquaredEuclidean, "manhattan": kb.Manhattan,
         "chebyshev": kb.Chebyshev, "minkowski3": kb.Minkowski(3),
         "minkowski4": kb.Minkowski(4)}[metric]
    g = t.query(Q).periodic_boundary_condition(box).nearest_one(M).execute_gpu()
    od, oi = o.periodic_nearest_one(Q, box, metric=metric)
    assert_same_fixed(g.distances, g.items, np.ones(len(Q)), od, oi, np.ones(len(Q)), "pnn1")
    r = {"sqeuclidean": 1e-4, "manhattan": 0.02, "chebyshev": 0.008, "minkowski3": 1e-6,
         "minkowski4": 1e-8}[metric]
    for k in (1, 8, 32):
        for radius in (None, r):
            for excl in ((False, True) if radius else (False,)):
                b = t.query(Q).periodic_boundary_condition(box).nearest_n(M, k)
                if radius is not None:
                    b = b.within(radius)
                    if excl:
                        b = b.exclusive_boundaries()
                g = b.execute_gpu()
                ref = o.periodic_nearest_n(Q, box, k, radius=np.inf if radius is None else radius,
                                           metric=metric, exclusive=excl)
                assert_same_fixed(g.distances, g.items, g.counts, *ref, f"pnn{k} r={radius}")
    for sorted_ in (True, False):
        b = t.query(Q).periodic_boundary_condition(box).within(M, r)
        if not sorted_:
            b = b.unsorted()
        g = b.execute_gpu()
        ref = o.periodic_within(Q, box, r, metric=metric, sorted=sorted_)
        assert_same_csr((g.offsets, g.distances, g.items), ref, f"pwithin sorted={sorted_}")


def test_periodic_non_unit_box_and_small_trees():
    rng = np.random.default_rng(3)
    box = np.array([2.0, 0.5, 1.5])
    for n in (0, 1, 31, 33, 500):
        P = rng.random((n, 3)) * box
        Q = rng.random((400, 3)) * box
        t = kb.ImmutableKdTree.new_from_slice(P)
        o = oracle.OracleTree.build(P)
        g = t.query(Q).periodic_boundary_condition(box).nearest_one(kb.SquaredEuclidean).execute_gpu()
        od, oi = o.periodic_nearest_one(Q, box)
        assert_same_fixed(g.distances, g.items, np.ones(400), od, oi, np.ones(400), f"n={n}")
        g = t.query(Q).periodic_boundary_condition(box).nearest_n(kb.SquaredEuclidean, 5).execute_gpu()
        assert_same_fixed(g.distances, g.items, g.counts, *o.periodic_nearest_n(Q, box, 5), "pnn5")


def test_periodic_known_answers():
    for kat in load_kats():
        if "box" not in kat:
            continue
        P = kat["np_points"]
        t = kb.ImmutableKdTree.new_from_slice(P)
        box = np.asarray(kat["box"])
        for chk in kat["checks"]:
            q = np.asarray([chk["query"]])
            if chk["family"] == "periodic_nearest_one":
                g = t.query(q).periodic_boundary_condition(box).nearest_one(kb.SquaredEuclidean).execute_gpu()
                assert g.items.tolist() == chk["expect_items"]
            else:
                g = t.query(q).periodic_boundary_condition(box).nearest_n(
                    kb.SquaredEuclidean, chk["k"]).within(chk["radius"]).execute_gpu()
                assert int(g.counts[0]) == chk["expect_len"]


def test_periodic_rejections():
    t = kb.ImmutableKdTree.new_from_slice(np.random.default_rng(0).random((100, 3)))
    q = np.zeros((1, 3))
    with pytest.raises(TypeError):
        t.query(q).periodic_boundary_condition(np.ones(3)).nearest_one(kb.SquaredEuclidean).approx()
