"""The oracle's iteration order and point-projected scans, pinned to the
reference's own known answers (CPU only).

KdTree::iter's documented results (src/kd_tree/construction.rs:255-271,
:385-400, :1236-1251) fix the iteration order of small trees: a single leaf
yields its entries in source order.  The projected scans restate
builder.rs:2175-2305 over that order.
"""
import numpy as np
import pytest

import oracle


def test_iter_known_answers():
    # construction.rs:255-271: new_from_slice, f64 3-D
    t = oracle.OracleTree.build(np.array([[1.0, 2.0, 3.0], [4.0, 5.0, 6.0]]))
    items, pts = t.iter()
    assert items.tolist() == [0, 1]
    assert pts.tolist() == [[1.0, 2.0, 3.0], [4.0, 5.0, 6.0]]
    # construction.rs:385-400: new_from_entries, f32 2-D
    t = oracle.OracleTree.build(np.array([[0.0, 1.0], [2.0, 3.0]], np.float32),
                                np.array([42, 7], np.uint32))
    items, pts = t.iter()
    assert items.tolist() == [42, 7]
    assert pts.tolist() == [[0.0, 1.0], [2.0, 3.0]]
    # construction.rs:1236-1251 (before its replace_item): f64 2-D entries
    t = oracle.OracleTree.build(np.array([[1.0, 10.0], [2.0, 20.0], [3.0, 30.0]]),
                                np.array([20, 21, 22], np.uint32))
    items, pts = t.iter()
    assert items.tolist() == [20, 21, 22]
    assert pts.tolist() == [[1.0, 10.0], [2.0, 20.0], [3.0, 30.0]]


@pytest.mark.parametrize("dims", [1, 2, 3, 4])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_iter_is_a_permutation_in_leaf_order(dims, dtype):
    rng = np.random.default_rng(dims)
    P = rng.random((3000, dims)).astype(dtype)
    t = oracle.OracleTree.build(P)
    items, pts = t.iter()
    assert sorted(items.tolist()) == list(range(3000))
    assert np.array_equal(pts, P[items])
    lay = t.layout()
    assert int(lay.extents[:, 1].astype(np.int64).sum()) == 3000


def test_projected_scans_against_brute_force():
    rng = np.random.default_rng(5)
    P = (np.floor(rng.random((2000, 3)) * 8) / 8)  # many equal distances
    t = oracle.OracleTree.build(P)
    items, pts = t.iter()
    q = np.array([0.3, 0.55, 0.7])
    d = oracle.scan_dists(pts, q)
    dist, item, point, rank = oracle.projected_nearest_one(t, q)
    assert rank == int(np.nonzero(d == d.min())[0][0]) and item == items[rank]
    assert np.array_equal(point, pts[rank])
    dd, ii, pp, rr = oracle.projected_nearest(t, q, radius=0.05, sorted=False)
    assert np.all(np.diff(rr) > 0) and np.all(dd <= 0.05)  # iteration order
    dd, ii, pp, rr = oracle.projected_nearest(t, q, max_qty=40)
    assert len(dd) == 40 and np.all(np.diff(dd) >= 0)
    tie = dd[:-1] == dd[1:]
    assert np.all(rr[:-1][tie] < rr[1:][tie])  # equal distances in iteration order
    dd, ii, pp, rr = oracle.projected_best(t, q, 0.1, 5)
    assert np.all(np.diff(ii.astype(np.int64)) > 0) and np.all(dd <= 0.1)


def test_empty_tree_nearest_one():
    t = oracle.OracleTree.build(np.zeros((0, 2), np.float32))
    dist, item, point, rank = oracle.projected_nearest_one(t, np.zeros(2, np.float32))
    assert np.isinf(dist) and item == 0 and rank is None and point.tolist() == [0.0, 0.0]


def test_within_result_streaming_on_the_host():
    """QueryBuilder.visit/iter walk the CSR result of within().unsorted(): each
    query's hits in order, fields that a projection left out as None."""
    import kiddo_b200 as kb
    from kiddo_b200 import _capi as C
    res = kb.WithinResult(np.array([0, 2, 2, 3], np.uint64),
                          np.array([0.5, 0.25, 0.125], np.float32),
                          np.array([7, 3, 9], np.uint32), None)
    assert [(i, float(d), int(it), p) for i, d, it, p in res.iter()] == \
        [(0, 0.5, 7, None), (0, 0.25, 3, None), (2, 0.125, 9, None)]
    seen = []
    res.visit(lambda i, d, it, p: seen.append((i, int(it))))
    assert seen == [(0, 7), (0, 3), (2, 9)]

    b = kb.QueryBuilder.__new__(kb.QueryBuilder)
    b.__dict__.update(family=C.WITHIN_UNSORTED)
    b.execute_gpu = lambda: res
    assert len(list(b.iter())) == 3
    b.family = C.WITHIN
    with pytest.raises(TypeError):
        b.visit(print)


def test_projection_ordering_rules_on_the_host():
    """The orderings with_points applies to device results, run here on CPU
    tensors against numpy's lexsort: CSR rows by rank or (distance, rank),
    fixed rows by (distance, rank) with unused slots last."""
    import torch
    import kiddo_b200 as kb
    rng = np.random.default_rng(8)
    counts = rng.integers(0, 25, 60)
    off = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    n = int(off[-1])
    dist = np.floor(rng.random(n) * 6).astype(np.float32)  # many ties
    # ranks are uint32 held in int32: include some at 2^31 and above (negative as int32)
    ranks_u = rng.permutation(1 << 20)[:n].astype(np.uint32)
    ranks_u[::7] = rng.integers(1 << 31, (1 << 32) - 1, len(ranks_u[::7]), dtype=np.uint64)
    ranks = ranks_u.view(np.int32)
    rows = np.repeat(np.arange(60), counts)
    got = kb._csr_order(torch.from_numpy(off), torch.from_numpy(ranks)).numpy()
    assert np.array_equal(got, np.lexsort((ranks_u, rows)))
    got = kb._csr_order(torch.from_numpy(off), torch.from_numpy(ranks),
                        torch.from_numpy(dist)).numpy()
    assert np.array_equal(got, np.lexsort((ranks_u, dist, rows)))
    D = np.floor(rng.random((40, 12)) * 4).astype(np.float32)
    R = rng.integers(0, 1000, (40, 12)).astype(np.int32)
    D[:, 9:] = np.inf
    R[:, 9:] = -1  # unused slots: rank 0xFFFFFFFF
    got = kb._row_order(torch.from_numpy(D), torch.from_numpy(R)).numpy()
    key = R.astype(np.int64) % (1 << 32)
    for j in range(40):
        assert np.array_equal(got[j], np.lexsort((key[j], D[j])))


def test_nearest_one_projection_keeps_rows_without_hits():
    """with_points().nearest_one on a query with a NaN coordinate: its radius
    row is empty (NaN distances fail d <= r), and scan_projected_nearest_one
    (builder.rs:2175-2212) keeps the first entry in iteration order at its own
    NaN distance.  Empty rows in the middle and at the end, on CPU tensors."""
    import torch
    import kiddo_b200 as kb
    from kiddo_b200 import _capi as C

    class FakeTree:
        def iter(self, stream=None):
            return (torch.tensor([40, 41, 42], dtype=torch.int32),
                    torch.tensor([[0.5, 0.5], [0.1, 0.2], [0.9, 0.9]], dtype=torch.float32))

    class Res:
        pass

    r = Res()
    r.offsets = torch.tensor([0, 2, 2, 3, 3], dtype=torch.int64)  # rows 1 and 3 empty
    r.distances = torch.tensor([0.25, 0.25, 0.01], dtype=torch.float32)
    r.items = torch.tensor([42, 41, 40], dtype=torch.int32)
    ranks = torch.tensor([2, 1, 0], dtype=torch.int32)
    pts = torch.tensor([[0.9, 0.9], [0.1, 0.2], [0.5, 0.5]], dtype=torch.float32)
    q = torch.tensor([[0.4, 0.4], [float("nan"), 0.3], [0.5, 0.6], [0.2, float("nan")]],
                     dtype=torch.float32)
    out = kb._first_by_rank(r, ranks, pts, q, C.SQUARED_EUCLIDEAN, FakeTree(), None)
    assert out.items.tolist() == [41, 40, 40, 40]
    d = out.distances.numpy()
    assert d[0] == np.float32(0.25) and d[2] == np.float32(0.01)
    assert np.isnan(d[1]) and np.isnan(d[3])
    assert np.array_equal(out.points.numpy(), np.array([[0.1, 0.2], [0.5, 0.5], [0.5, 0.5],
                                                        [0.5, 0.5]], dtype=np.float32))
    # the NaN rows agree with the oracle's restatement of the scan
    import oracle
    P = np.array([[0.5, 0.5], [0.1, 0.2], [0.9, 0.9]], dtype=np.float32)
    o = oracle.OracleTree.build(P)
    items, ipts = o.iter()
    od, oi, op, orank = oracle.projected_nearest_one(o, q[1].numpy())
    assert orank == 0 and np.isnan(od) and oi == int(items[0])
