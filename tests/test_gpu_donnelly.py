"""Bit-exact parity of the CUDA engine with the CPU oracle on Donnelly<BH> trees.

A Donnelly tree (stem_strategy/donnelly/core.rs) has the same leaves as the
ImmutableKdTree of the same points but its stems in block-packed order, padded
at the root to a multiple of the block height; the reference answers its
queries with scalar backtracking over an explicit stack (orchestrator/mod.rs:
265-345, 607-669).  Each case uploads one layout to the GPU and to the oracle
and compares distances, items and traversal counters bit for bit.
"""
import zlib

import numpy as np
import pytest

import kiddo_b200 as kb
import oracle
from helpers import assert_same_csr, assert_same_fixed, gaussian_mixture

pytestmark = pytest.mark.gpu

DATASETS = {
    "uniform": lambda rng, n, k, dt: rng.random((n, k)).astype(dt),
    "quantized": lambda rng, n, k, dt: (np.floor(rng.random((n, k)) * 16) / 16).astype(dt),
    "clustered": lambda rng, n, k, dt: (rng.random((8, k))[rng.integers(0, 8, n)]
                                        + rng.normal(0, 0.002, (n, k))).astype(dt),
}


def _pair(P, bh, items=None):
    if items is None:
        t = kb.ImmutableKdTree.new_from_slice(P, block_height=bh)
    else:
        t = kb.ImmutableKdTree.new_from_entries(items, P, block_height=bh)
    o = oracle.OracleTree.build(P, items, block_height=bh)
    return t, o


def _metric(m):
    return {"sqeuclidean": kb.SquaredEuclidean, "manhattan": kb.Manhattan,
            "chebyshev": kb.Chebyshev, "minkowski3": kb.Minkowski(3),
            "minkowski4": kb.Minkowski(4)}[m]


@pytest.mark.parametrize("bh", [3, 4])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("dims", [2, 3])
@pytest.mark.parametrize("metric", ["sqeuclidean", "manhattan", "chebyshev",
                                    "minkowski3", "minkowski4"])
@pytest.mark.parametrize("data", ["uniform", "quantized", "clustered"])
def test_fixed_families_donnelly(bh, dtype, dims, metric, data):
    rng = np.random.default_rng(zlib.crc32(f"don{bh}{dims}{metric}{data}".encode()))
    P = DATASETS[data](rng, 20000, dims, dtype)
    Q = np.concatenate([DATASETS[data](rng, 1500, dims, dtype), P[:200]])  # on-point queries
    t, o = _pair(P, bh)
    M = _metric(metric)
    g = t.query(Q).nearest_one(M).execute_gpu()
    od, oi = o.nearest_one(Q, metric=metric)
    assert_same_fixed(g.distances, g.items, np.ones(len(Q)), od, oi, np.ones(len(Q)), "nn1")
    g = t.query(Q).nearest_one(M).approx().execute_gpu()
    od, oi = o.approx_nearest_one(Q, metric=metric)
    assert_same_fixed(g.distances, g.items, np.ones(len(Q)), od, oi, np.ones(len(Q)), "approx")
    r = {"sqeuclidean": 0.001, "manhattan": 0.03, "chebyshev": 0.015, "minkowski3": 3e-5,
         "minkowski4": 1e-6}[metric]
    for k in (1, 5, 16, 32):
        g = t.query(Q).nearest_n(M, k).execute_gpu()
        assert_same_fixed(g.distances, g.items, g.counts, *o.nearest_n(Q, k, metric=metric),
                          f"nearest_n({k})")
        g = t.query(Q).nearest_n(M, k).unsorted().execute_gpu()
        assert_same_fixed(g.distances, g.items, g.counts,
                          *o.nearest_n(Q, k, metric=metric, sorted=False), f"unsorted({k})")
        for excl in (False, True):
            b = t.query(Q).nearest_n(M, k).within(r)
            if excl:
                b = b.exclusive_boundaries()
            g = b.execute_gpu()
            assert_same_fixed(g.distances, g.items, g.counts,
                              *o.nearest_n(Q, k, radius=r, metric=metric, exclusive=excl),
                              f"nearest_n({k}).within excl={excl}")
    for excl in (False, True):
        b = t.query(Q).best_n_within(M, r, 5)
        if excl:
            b = b.exclusive_boundaries()
        g = b.execute_gpu()
        assert_same_fixed(g.distances, g.items, g.counts,
                          *o.best_n_within(Q, r, 5, metric=metric, exclusive=excl), "best_n")


@pytest.mark.parametrize("bh", [3, 4])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("metric", ["sqeuclidean", "manhattan", "chebyshev",
                                    "minkowski3", "minkowski4"])
def test_within_families_donnelly(bh, dtype, metric):
    rng = np.random.default_rng(17 + bh)
    P = DATASETS["uniform"](rng, 30000, 3, dtype)
    Q = DATASETS["uniform"](rng, 2000, 3, dtype)
    t, o = _pair(P, bh)
    M = _metric(metric)
    cases = {"sqeuclidean": ((1e-5, 2000), (3e-4, 2000), (4e-3, 2000), (0.15, 120)),
             "manhattan": ((0.005, 2000), (0.04, 2000), (0.2, 2000), (0.6, 120)),
             "chebyshev": ((0.003, 2000), (0.03, 2000), (0.1, 2000), (0.3, 120)),
             "minkowski3": ((3e-8, 2000), (5e-6, 2000), (2.5e-4, 2000), (0.06, 120)),
             "minkowski4": ((1e-10, 2000), (8e-8, 2000), (1.6e-5, 2000), (0.023, 120))}[metric]
    for r, nq in cases:
        Qr = Q[:nq]
        for excl in (False, True):
            for sorted_ in (True, False):
                b = t.query(Qr).within(M, r)
                if not sorted_:
                    b = b.unsorted()
                if excl:
                    b = b.exclusive_boundaries()
                g = b.execute_gpu()
                ref = o.within(Qr, r, metric=metric, exclusive=excl, sorted=sorted_)
                assert_same_csr((g.offsets, g.distances, g.items), ref,
                                f"within r={r} excl={excl} sorted={sorted_}")


@pytest.mark.parametrize("bh", [3, 4])
@pytest.mark.parametrize("n", [0, 1, 31, 33, 64, 65, 257, 1000])
def test_small_and_ragged_donnelly_trees(bh, n):
    """Trees from no stems up to a few blocks, with and without root padding."""
    rng = np.random.default_rng(n + 10 * bh)
    P = rng.random((n, 3))
    Q = rng.random((300, 3))
    t, o = _pair(P, bh)
    g = t.query(Q).nearest_one(kb.SquaredEuclidean).execute_gpu()
    od, oi = o.nearest_one(Q)
    assert_same_fixed(g.distances, g.items, np.ones(300), od, oi, np.ones(300), "nn1")
    g = t.query(Q).nearest_n(kb.SquaredEuclidean, 7).execute_gpu()
    assert_same_fixed(g.distances, g.items, g.counts, *o.nearest_n(Q, 7), "nn7")
    g = t.query(Q).nearest_one(kb.SquaredEuclidean).approx().execute_gpu()
    od, oi = o.approx_nearest_one(Q)
    assert_same_fixed(g.distances, g.items, np.ones(300), od, oi, np.ones(300), "approx")
    g = t.query(Q).within(kb.SquaredEuclidean, 0.05).execute_gpu()
    assert_same_csr((g.offsets, g.distances, g.items), o.within(Q, 0.05), "within")


@pytest.mark.parametrize("bh", [3, 4])
def test_donnelly_traversal_counters_and_leaf_order(bh):
    """The GPU walks exactly the reference's scalar backtracking: its stem,
    leaf and point counters equal the oracle's, and leaf-grouped processing
    leaves results unchanged."""
    rng = np.random.default_rng(5)
    P = gaussian_mixture(200_000, 64, 0.01, 0.2, rng)
    Q = gaussian_mixture(70_000, 64, 0.01, 0.2, rng)
    t, o = _pair(P, bh)
    b = t.query(Q).nearest_n(kb.SquaredEuclidean, 16)
    _, _, _, ost = o.nearest_n(Q, 16, stats=True)
    assert np.array_equal(b.traversal_stats(), ost)
    for order in (True, False):
        g = t.query(Q).with_spatial_order(order).nearest_n(kb.SquaredEuclidean, 16).execute_gpu()
        assert_same_fixed(g.distances, g.items, g.counts, *o.nearest_n(Q, 16), f"order={order}")


def test_donnelly_explicit_items_and_rejections():
    rng = np.random.default_rng(9)
    P = rng.random((5000, 3)).astype(np.float32)
    items = rng.permutation(5000).astype(np.uint32) * 3 + 7
    t, o = _pair(P, 4, items)
    Q = rng.random((500, 3)).astype(np.float32)
    g = t.query(Q).best_n_within(kb.SquaredEuclidean, 0.01, 4).execute_gpu()
    assert_same_fixed(g.distances, g.items, g.counts, *o.best_n_within(Q, 0.01, 4), "best_n")
    # the warp engine walks Eytzinger stems only; a forest takes one stem order
    with pytest.raises(Exception):
        t.query(Q).with_engine("warp").nearest_one(kb.SquaredEuclidean).execute_gpu()
    with pytest.raises(Exception):
        kb.Forest([t, kb.ImmutableKdTree.new_from_slice(P)])
    with pytest.raises(Exception):
        kb.Forest([t, kb.ImmutableKdTree.new_from_slice(P, block_height=3)])


@pytest.mark.parametrize("bh", [3, 4])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("dims", [2, 3])
@pytest.mark.parametrize("metric", ["sqeuclidean", "manhattan", "chebyshev", "minkowski4"])
def test_periodic_families_donnelly(bh, dtype, dims, metric):
    """periodic_backtracking_query over Donnelly stems (periodic.rs:455-619 is
    generic over the stem strategy) and periodic nearest_one as home plus
    image queries over the scalar backtracking (periodic.rs:156-214)."""
    rng = np.random.default_rng(zlib.crc32(f"pdon{bh}{dims}{metric}".encode()))
    c = rng.random((32, dims))
    P = np.concatenate([(c[rng.integers(0, 32, 8000)] + rng.normal(0, 0.01, (8000, dims))) % 1.0,
                        rng.random((8000, dims))]).astype(dtype)
    Q = np.concatenate([rng.random((800, dims)), rng.random((200, dims)) * 0.01,
                        1 - rng.random((200, dims)) * 0.01, P[:100]]).astype(dtype)
    box = np.ones(dims, dtype=dtype)
    t, o = _pair(P, bh)
    M = _metric(metric)
    g = t.query(Q).periodic_boundary_condition(box).nearest_one(M).execute_gpu()
    od, oi = o.periodic_nearest_one(Q, box, metric=metric)
    assert_same_fixed(g.distances, g.items, np.ones(len(Q)), od, oi, np.ones(len(Q)), "pnn1")
    r = {"sqeuclidean": 2e-4, "manhattan": 0.03, "chebyshev": 0.01, "minkowski4": 1e-8}[metric]
    for k in (1, 8, 32, 70):
        for radius in (None, r):
            b = t.query(Q).periodic_boundary_condition(box).nearest_n(M, k)
            if radius is not None:
                b = b.within(radius)
            g = b.execute_gpu()
            ref = o.periodic_nearest_n(Q, box, k, radius=np.inf if radius is None else radius,
                                       metric=metric)
            assert_same_fixed(g.distances, g.items, g.counts, *ref, f"pnn{k} r={radius}")
    for sorted_ in (True, False):
        b = t.query(Q).periodic_boundary_condition(box).within(M, r)
        if not sorted_:
            b = b.unsorted()
        g = b.execute_gpu()
        ref = o.periodic_within(Q, box, r, metric=metric, sorted=sorted_)
        assert_same_csr((g.offsets, g.distances, g.items), ref, f"pwithin sorted={sorted_}")


@pytest.mark.parametrize("bh", [3, 4])
def test_donnelly_forest_matches_the_oracle(bh):
    """Many Donnelly trees of one block height in one launch: every family,
    one radius per query for the radius families, each row against the
    oracle tree it names."""
    import torch
    rng = np.random.default_rng(40 + bh)
    sizes = [20, 700, 5000, 30000]
    pts = [rng.random((n, 3)).astype(np.float32) for n in sizes]
    trees = [kb.ImmutableKdTree.new_from_slice(p, block_height=bh) for p in pts]
    oracles = [oracle.OracleTree.build(p, block_height=bh) for p in pts]
    forest = kb.Forest(trees)
    nq = 6000
    tree_of = rng.integers(0, len(pts), nq).astype(np.int32)
    Q = rng.random((nq, 3)).astype(np.float32)
    radii = (np.exp(rng.uniform(np.log(1e-4), np.log(1e-2), nq))).astype(np.float32)
    dq, dt, dr = (torch.from_numpy(x).cuda() for x in (Q, tree_of, radii))
    g1 = forest.query(dq, dt).nearest_one(kb.SquaredEuclidean).execute_gpu()
    g16 = forest.query(dq, dt).nearest_n(kb.SquaredEuclidean, 16).execute_gpu()
    gb = forest.query(dq, dt, dr).best_n_within(kb.SquaredEuclidean, 0.0, 5).execute_gpu()
    gw = forest.query(dq, dt, dr).within(kb.SquaredEuclidean, 0.0).execute_gpu()
    off = gw.offsets.cpu().numpy()
    wd, wi = gw.distances.cpu().numpy(), gw.items.cpu().numpy().view(np.uint32)
    for t in range(len(pts)):
        sel = np.nonzero(tree_of == t)[0]
        od, oi = oracles[t].nearest_one(Q[sel])
        assert_same_fixed(g1.distances.cpu().numpy()[sel], g1.items.cpu().numpy()[sel],
                          np.ones(len(sel)), od, oi, np.ones(len(sel)), f"nn1 tree {t}")
        assert_same_fixed(g16.distances.cpu().numpy()[sel], g16.items.cpu().numpy()[sel],
                          g16.counts.cpu().numpy()[sel], *oracles[t].nearest_n(Q[sel], 16),
                          f"knn tree {t}")
        assert_same_fixed(gb.distances.cpu().numpy()[sel], gb.items.cpu().numpy()[sel],
                          gb.counts.cpu().numpy()[sel],
                          *oracles[t].best_n_within(Q[sel], radii[sel], 5), f"best tree {t}")
        oo, od, oi = oracles[t].within(Q[sel], radii[sel])
        got_d = np.concatenate([wd[off[j]:off[j + 1]] for j in sel])
        got_i = np.concatenate([wi[off[j]:off[j + 1]] for j in sel])
        assert np.array_equal(np.diff(off)[sel], np.diff(oo).astype(np.int64))
        assert np.array_equal(got_d, od) and np.array_equal(got_i, oi), f"within tree {t}"
