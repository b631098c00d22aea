"""Iteration order and point-projected queries (with_points) on the GPU,
against the oracle's restatement of the reference's scans
(src/kd_tree/iter.rs:64-90, src/kd_tree/query/builder.rs:2175-2305).

Everything here is bit-exact: items, ranks and stored coordinates are copied,
and distances are the reference's own float arithmetic.  The one place the
reference leaves the result open, the order of equal distances after
slice::sort_unstable and the choice among them at the max_qty cut, is pinned
here to iteration order, with the cut compared only below the cut distance.
"""
import zlib

import numpy as np
import pytest

import kiddo_b200 as kb
import oracle

pytestmark = pytest.mark.gpu

METRICS = {"sqeuclidean": kb.SquaredEuclidean, "manhattan": kb.Manhattan,
           "chebyshev": kb.Chebyshev, "minkowski3": kb.Minkowski(3)}

DATA = {
    "uniform": lambda rng, n, k, dt: rng.random((n, k)).astype(dt),
    "quantized": lambda rng, n, k, dt: (np.floor(rng.random((n, k)) * 12) / 12).astype(dt),
}


def _pair(P, items=None):
    t = kb.ImmutableKdTree.new_from_slice(P) if items is None else \
        kb.ImmutableKdTree.new_from_entries(items, P)
    return t, oracle.OracleTree.build(P, items)


def _np(x):
    return x.cpu().numpy()


@pytest.mark.parametrize("dims", [1, 2, 3, 4])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("n", [1, 33, 5000])
def test_iter_matches_oracle(dims, dtype, n):
    rng = np.random.default_rng(zlib.crc32(f"{dims}{n}".encode()))
    P = DATA["quantized"](rng, n, dims, dtype)
    t, o = _pair(P)
    oi, op = o.iter()
    gi, gp = t.to_gpu().iter()
    assert np.array_equal(_np(gi).view(np.uint32), oi)
    assert np.array_equal(_np(gp), op)


def test_iter_known_answers_and_device_build():
    import torch
    # KdTree::iter's documented answers (construction.rs:255-271, :385-400)
    t = kb.ImmutableKdTree.new_from_slice(np.array([[1.0, 2.0, 3.0], [4.0, 5.0, 6.0]]))
    gi, gp = t.to_gpu().iter()
    assert _np(gi).tolist() == [0, 1] and _np(gp).tolist() == [[1, 2, 3], [4, 5, 6]]
    t = kb.ImmutableKdTree.new_from_entries(np.array([42, 7], np.uint32),
                                            np.array([[0.0, 1.0], [2.0, 3.0]], np.float32))
    gi, gp = t.to_gpu().iter()
    assert _np(gi).tolist() == [42, 7] and _np(gp).tolist() == [[0, 1], [2, 3]]
    # a device-built tree iterates like the host-built one
    rng = np.random.default_rng(3)
    P = rng.random((20000, 3)).astype(np.float32)
    g = kb.GpuTree.build(torch.from_numpy(P).cuda())
    oi, op = oracle.OracleTree.build(P).iter()
    gi, gp = g.iter()
    assert np.array_equal(_np(gi).view(np.uint32), oi) and np.array_equal(_np(gp), op)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_project_ranks_and_points(dtype):
    import torch
    rng = np.random.default_rng(11)
    P = rng.random((7000, 3)).astype(dtype)
    items = rng.permutation(50000)[:7000].astype(np.uint32)  # sparse, distinct
    t, o = _pair(P, items)
    oi, op = o.iter()
    pos = {int(v): r for r, v in enumerate(oi)}
    ask = np.concatenate([items[rng.integers(0, 7000, 3000)],
                          np.array([0xFFFFFFFF, 50001], np.uint32)])
    for _ in range(2):  # the first call builds the table, the second reuses it
        r, p = t.to_gpu().project(torch.from_numpy(ask.view(np.int32)).cuda())
        want = np.array([pos.get(int(v), -1) for v in ask])
        assert np.array_equal(_np(r), want)
        wp = np.where((want >= 0)[:, None], op[np.maximum(want, 0)], 0)
        assert np.array_equal(_np(p), wp.astype(dtype))


def test_project_rejects_shared_items():
    import torch
    P = np.random.default_rng(2).random((100, 2))
    items = np.arange(100, dtype=np.uint32) // 2
    t = kb.ImmutableKdTree.new_from_entries(items, P)
    with pytest.raises(kb.KiddoGpuError):
        t.to_gpu().project(torch.zeros(4, dtype=torch.int32, device="cuda"))
    with pytest.raises(kb.KiddoGpuError):
        t.query(P[:3]).nearest_n(kb.SquaredEuclidean, 4).with_points().execute_gpu()


def test_periodic_queries_cannot_return_points():
    t = kb.ImmutableKdTree.new_from_slice(np.random.default_rng(0).random((50, 3)))
    with pytest.raises(TypeError):
        t.query(np.zeros((1, 3))).periodic_boundary_condition([1, 1, 1]).with_points()
    with pytest.raises(TypeError):
        t.query(np.zeros((1, 3))).with_points().periodic_boundary_condition([1, 1, 1])


@pytest.mark.parametrize("dims", [2, 3])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("metric", list(METRICS))
@pytest.mark.parametrize("data", list(DATA))
def test_with_points_families(dims, dtype, metric, data):
    import torch
    rng = np.random.default_rng(zlib.crc32(f"{dims}{metric}{data}".encode()))
    n = 6000
    P = DATA[data](rng, n, dims, dtype)
    Q = np.concatenate([DATA[data](rng, 150, dims, dtype), P[:50]])
    t, o = _pair(P)
    M = METRICS[metric]
    Qd = torch.from_numpy(Q).cuda()
    radius = {"sqeuclidean": 0.004, "manhattan": 0.09, "chebyshev": 0.04,
              "minkowski3": 0.0004}[metric]
    k = 12

    # nearest_one and approx: the first entry in iteration order at the least distance
    for approx in (False, True):
        b = t.query(Qd).nearest_one(M)
        g = (b.approx() if approx else b).with_points().execute_gpu()
        for j, q in enumerate(Q):
            d, it, p, r = oracle.projected_nearest_one(o, q, metric)
            assert _np(g.distances)[j] == d and int(_np(g.items)[j]) == it
            assert np.array_equal(_np(g.points)[j], p)

    # within().unsorted(): iteration order; within: distance, then iteration order
    for sorted_ in (False, True):
        b = t.query(Qd).within(M, radius)
        g = (b if sorted_ else b.unsorted()).with_points().execute_gpu()
        off = _np(g.offsets)
        for j, q in enumerate(Q):
            d, it, p, r = oracle.projected_nearest(o, q, metric, radius=radius, sorted=sorted_)
            a, e = off[j], off[j + 1]
            assert np.array_equal(_np(g.distances)[a:e], d)
            assert np.array_equal(_np(g.items)[a:e].view(np.uint32), it)
            assert np.array_equal(_np(g.points)[a:e], p)

    # nearest_n and nearest_n().within: distance order; the set below the cut
    # distance is fixed, the choice among entries at the cut distance is not
    for within in (False, True):
        b = t.query(Qd).nearest_n(M, k)
        if within:
            b = b.within(radius)
        g = b.with_points().execute_gpu()
        for j, q in enumerate(Q):
            d, it, p, r = oracle.projected_nearest(o, q, metric, radius=radius if within else None,
                                                   max_qty=k)
            c = int(_np(g.counts)[j])
            assert c == len(d)
            assert np.array_equal(_np(g.distances)[j, :c], d)
            below = d < d[-1] if c else np.zeros(0, bool)
            assert np.array_equal(_np(g.items)[j, :c].view(np.uint32)[below], it[below])
            assert np.array_equal(_np(g.points)[j, :c][below], p[below])
            # every returned point is the stored point of its item
            gi = _np(g.items)[j, :c].view(np.uint32)
            assert np.array_equal(_np(g.points)[j, :c], P[gi])

    # best_n_within: ascending item
    g = t.query(Qd).best_n_within(M, radius, 5).with_points().execute_gpu()
    for j, q in enumerate(Q):
        d, it, p, r = oracle.projected_best(o, q, radius, 5, metric)
        c = int(_np(g.counts)[j])
        assert c == len(d)
        assert np.array_equal(_np(g.items)[j, :c].view(np.uint32), it)
        assert np.array_equal(_np(g.distances)[j, :c], d)
        assert np.array_equal(_np(g.points)[j, :c], p)


def test_with_points_host_buffers_and_sparse_items():
    rng = np.random.default_rng(9)
    P = (np.floor(rng.random((4000, 3)) * 10) / 10).astype(np.float32)
    items = rng.permutation(1 << 30)[:4000].astype(np.uint32)
    t, o = _pair(P, items)
    Q = rng.random((100, 3)).astype(np.float32)
    g = t.query(Q).nearest_one(kb.SquaredEuclidean).with_points().execute_gpu()
    assert isinstance(g.points, np.ndarray) and g.items.dtype == np.uint32
    for j, q in enumerate(Q):
        d, it, p, r = oracle.projected_nearest_one(o, q)
        assert g.distances[j] == d and g.items[j] == it and np.array_equal(g.points[j], p)
    g = t.query(Q).within(kb.SquaredEuclidean, 0.01).unsorted().with_points().execute_gpu()
    for j, q in enumerate(Q):
        d, it, p, r = oracle.projected_nearest(o, q, radius=0.01, sorted=False)
        dj, ij, pj = g[j]
        assert np.array_equal(dj, d) and np.array_equal(ij, it) and np.array_equal(pj, p)


def test_item_and_distance_switches():
    rng = np.random.default_rng(4)
    P = rng.random((3000, 3)).astype(np.float32)
    t = kb.ImmutableKdTree.new_from_slice(P)
    Q = rng.random((64, 3)).astype(np.float32)
    full = t.query(Q).nearest_n(kb.SquaredEuclidean, 8).with_points().execute_gpu()
    g = t.query(Q).nearest_n(kb.SquaredEuclidean, 8).with_points().without_items() \
        .execute_gpu()
    assert g.items is None and np.array_equal(g.distances, full.distances)
    assert np.array_equal(g.points, full.points)
    g = t.query(Q).within(kb.SquaredEuclidean, 0.01).without_distances().execute_gpu()
    assert g.distances is None and g.items is not None
    g = t.query(Q).nearest_one(kb.SquaredEuclidean).with_points().without_points() \
        .without_distances().with_distances().execute_gpu()
    assert g.points is None and g.distances is not None
