"""Trees with Mapped stem/leaf resolution (MutableKdTree and trees whose
leaves sit at different depths) on the GPU against the oracle, bit for bit.

The reference walks such trees with its scalar backtracking, checking at
every stem whether it maps straight to a leaf (orchestrator/mod.rs:214-345,
607-669; stem_leaf_resolution.rs:53-120).  The trees come from the oracle:
MutableKdTree's hard-bucket bulk construction (construction.rs:413-539,
695-864, 972-1009), and irregular trees of random leaf depths.
"""
import numpy as np
import pytest

import kiddo_b200 as kb
import oracle
from helpers import assert_same_csr, assert_same_fixed, vecofarrays_parts

pytestmark = pytest.mark.gpu

METRICS = {"sqeuclidean": kb.SquaredEuclidean, "manhattan": kb.Manhattan,
           "chebyshev": kb.Chebyshev}
RADII = {"sqeuclidean": 2e-3, "manhattan": 0.06, "chebyshev": 0.03}


def _upload(o, dims, dtype, leaves="arena"):
    lay = o.layout()
    m, mn = o.leaf_map()
    if leaves == "arena":
        return kb.GpuTree.from_mapped_layout(dtype, dims, lay.stems, lay.leaf_bytes, lay.extents,
                                             lay.max_stem_level, lay.size, lay.max_leaf_len, m,
                                             mn, block_height=lay.block_height)
    host = kb.ImmutableKdTree.from_layout(dtype, dims, lay.stems, lay.leaf_bytes, lay.extents,
                                          lay.max_stem_level, lay.size, lay.max_leaf_len,
                                          lay.block_height)
    pts, its, sizes = vecofarrays_parts(host)
    return kb.GpuTree.from_vec_of_arrays(lay.stems, pts, its, sizes, lay.max_stem_level,
                                         block_height=lay.block_height, leaf_idx_map=m,
                                         min_stem_leaf_idx=mn)


def _tree(kind, P, bh=0):
    if kind == "mutable":
        return oracle.OracleTree.build_mutable(P, block_height=bh)
    return oracle.OracleTree.build_mutable(P, irregular_seed=int(P.shape[0]) + 7)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("dims", [2, 3])
@pytest.mark.parametrize("kind", ["mutable", "mutable_donnelly", "irregular"])
@pytest.mark.parametrize("metric", ["sqeuclidean", "manhattan", "chebyshev"])
def test_mapped_trees_match_the_oracle(dtype, dims, kind, metric):
    rng = np.random.default_rng(dims * 100 + len(kind) + len(metric))
    P = np.concatenate([rng.random((12_000, dims)),
                        np.floor(rng.random((3_000, dims)) * 32) / 32]).astype(dtype)
    Q = np.concatenate([rng.random((1_500, dims)), P[:200]]).astype(dtype)
    o = _tree("mutable" if kind != "irregular" else kind, P, 4 if kind == "mutable_donnelly" else 0)
    g = _upload(o, dims, dtype, "arrays" if kind == "mutable" else "arena")
    M = METRICS[metric]
    r = RADII[metric]
    res = g.query(Q).nearest_one(M).execute_gpu()
    od, oi = o.nearest_one(Q, metric=metric)
    assert_same_fixed(res.distances, res.items, np.ones(len(Q)), od, oi, np.ones(len(Q)), "nn1")
    res = g.query(Q).nearest_one(M).approx().execute_gpu()
    od, oi = o.approx_nearest_one(Q, metric=metric)
    assert_same_fixed(res.distances, res.items, np.ones(len(Q)), od, oi, np.ones(len(Q)), "approx")
    for k in (1, 5, 16, 40):
        res = g.query(Q).nearest_n(M, k).execute_gpu()
        assert_same_fixed(res.distances, res.items, res.counts, *o.nearest_n(Q, k, metric=metric),
                          f"nearest_n({k})")
        res = g.query(Q).nearest_n(M, k).within(r).exclusive_boundaries().execute_gpu()
        assert_same_fixed(res.distances, res.items, res.counts,
                          *o.nearest_n(Q, k, radius=r, metric=metric, exclusive=True),
                          f"nearest_n({k}).within")
    res = g.query(Q).best_n_within(M, r, 5).execute_gpu()
    assert_same_fixed(res.distances, res.items, res.counts, *o.best_n_within(Q, r, 5, metric=metric),
                      "best_n")
    for sorted_ in (True, False):
        b = g.query(Q).within(M, r)
        if not sorted_:
            b = b.unsorted()
        res = b.execute_gpu()
        assert_same_csr((res.offsets, res.distances, res.items),
                        o.within(Q, r, metric=metric, sorted=sorted_), f"within {sorted_}")
    box = np.ones(dims, dtype=dtype)
    res = g.query(Q).periodic_boundary_condition(box).nearest_one(M).execute_gpu()
    od, oi = o.periodic_nearest_one(Q, box, metric=metric)
    assert_same_fixed(res.distances, res.items, np.ones(len(Q)), od, oi, np.ones(len(Q)), "pnn1")
    res = g.query(Q).periodic_boundary_condition(box).nearest_n(M, 8).within(r).execute_gpu()
    assert_same_fixed(res.distances, res.items, res.counts,
                      *o.periodic_nearest_n(Q, box, 8, radius=r, metric=metric), "pnn8")
    res = g.query(Q).periodic_boundary_condition(box).within(M, r).execute_gpu()
    assert_same_csr((res.offsets, res.distances, res.items),
                    o.periodic_within(Q, box, r, metric=metric), "pwithin")


@pytest.mark.parametrize("n", [0, 1, 31, 32, 33, 65, 1000])
def test_small_mapped_trees(n):
    rng = np.random.default_rng(n)
    P = rng.random((n, 3))
    Q = rng.random((300, 3))
    for kind in ("mutable", "irregular"):
        o = _tree(kind, P)
        g = _upload(o, 3, np.float64)
        res = g.query(Q).nearest_n(kb.SquaredEuclidean, 7).execute_gpu()
        assert_same_fixed(res.distances, res.items, res.counts, *o.nearest_n(Q, 7), f"{kind} nn7")
        res = g.query(Q).within(kb.SquaredEuclidean, 0.05).execute_gpu()
        assert_same_csr((res.offsets, res.distances, res.items), o.within(Q, 0.05), kind)


def test_mapped_traversal_counters_order_and_forest():
    """The GPU walk visits exactly the oracle's stems, leaves and points;
    leaf-grouped order leaves results unchanged; a forest of Mapped trees
    answers like each tree's oracle."""
    import torch
    rng = np.random.default_rng(12)
    P = rng.random((200_000, 3)).astype(np.float32)
    Q = rng.random((80_000, 3)).astype(np.float32)
    o = oracle.OracleTree.build_mutable(P)
    g = _upload(o, 3, np.float32)
    _, _, _, ost = o.nearest_n(Q, 16, stats=True)
    assert np.array_equal(g.query(Q).nearest_n(kb.SquaredEuclidean, 16).traversal_stats(), ost)
    for order in (True, False):
        res = g.query(Q).with_spatial_order(order).nearest_n(kb.SquaredEuclidean, 16).execute_gpu()
        assert_same_fixed(res.distances, res.items, res.counts, *o.nearest_n(Q, 16),
                          f"order={order}")
    pts = [rng.random((n, 3)).astype(np.float32) for n in (40, 3000, 50_000)]
    oracles = [oracle.OracleTree.build_mutable(p) for p in pts]
    forest = kb.Forest([_upload(t, 3, np.float32) for t in oracles])
    nq = 9000
    tree_of = rng.integers(0, 3, nq).astype(np.int32)
    Qf = rng.random((nq, 3)).astype(np.float32)
    res = forest.query(torch.from_numpy(Qf).cuda(), torch.from_numpy(tree_of).cuda()).nearest_n(
        kb.SquaredEuclidean, 8).execute_gpu()
    for t in range(3):
        sel = np.nonzero(tree_of == t)[0]
        assert_same_fixed(res.distances.cpu().numpy()[sel], res.items.cpu().numpy()[sel],
                          res.counts.cpu().numpy()[sel], *oracles[t].nearest_n(Qf[sel], 8),
                          f"forest tree {t}")
