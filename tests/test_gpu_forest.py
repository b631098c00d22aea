"""Batched queries over many trees (one persistent launch with a device work
queue) against the oracle tree each query names, bit for bit, for every
family, with one radius for the batch or one per query."""
import numpy as np
import pytest

import kiddo_b200 as kb
import oracle
from helpers import assert_same_csr, assert_same_fixed

pytestmark = pytest.mark.gpu


def _forest_data(rng, n_trees=9, dtype=np.float32):
    sizes = np.unique(np.exp(rng.uniform(np.log(20), np.log(60000), n_trees)).astype(int))
    pts = []
    for n in sizes:
        v = rng.normal(size=(n, 3))
        pts.append((v / np.linalg.norm(v, axis=1, keepdims=True)).astype(dtype))
    return pts


@pytest.mark.parametrize("engine", [None, "warp", "thread"])
@pytest.mark.parametrize("order", [None, True])
def test_forest_fixed_families_match_oracle(engine, order):
    """nearest_one, nearest_n(8) sorted and unsorted, nearest_n(8).within and
    best_n_within(5) over 9 trees of 20 to 60,000 points in one launch: each
    query's row against the oracle tree it names."""
    import torch
    rng = np.random.default_rng(8)
    pts = _forest_data(rng)
    items = [rng.permutation(len(p)).astype(np.uint32) for p in pts]
    trees = [kb.ImmutableKdTree.new_from_entries(it, p) for it, p in zip(items, pts)]
    oracles = [oracle.OracleTree.build(p, it) for it, p in zip(items, pts)]
    forest = kb.Forest(trees)
    nq = 12000
    tree_of = rng.integers(0, len(trees), nq).astype(np.int32)
    Q = rng.normal(size=(nq, 3))
    Q = (Q / np.linalg.norm(Q, axis=1, keepdims=True)).astype(np.float32)
    dq = torch.from_numpy(Q).cuda()
    dt = torch.from_numpy(tree_of).cuda()
    r = 4e-4
    cases = {
        "nn1": (lambda b: b.nearest_one(kb.SquaredEuclidean),
                lambda o, q: o.nearest_one(q) + (np.ones(len(q), np.uint32),)),
        "knn": (lambda b: b.nearest_n(kb.SquaredEuclidean, 8), lambda o, q: o.nearest_n(q, 8)),
        "knn_unsorted": (lambda b: b.nearest_n(kb.SquaredEuclidean, 8).unsorted(),
                         lambda o, q: o.nearest_n(q, 8, sorted=False)),
        "knn_within": (lambda b: b.nearest_n(kb.SquaredEuclidean, 8).within(r),
                       lambda o, q: o.nearest_n(q, 8, radius=r)),
        "best": (lambda b: b.best_n_within(kb.SquaredEuclidean, r, 5),
                 lambda o, q: o.best_n_within(q, r, 5)),
    }
    for fam, (make, ref) in cases.items():
        g = make(forest.query(dq, dt).with_engine(engine).with_spatial_order(order)).execute_gpu()
        gd = g.distances.cpu().numpy().reshape(nq, -1)
        gi = g.items.cpu().numpy().view(np.uint32).reshape(nq, -1)
        gc = np.ones(nq, np.uint32) if fam == "nn1" else g.counts.cpu().numpy()
        for t in range(len(trees)):
            sel = np.nonzero(tree_of == t)[0]
            if len(sel) == 0:
                continue
            od, oi, oc = ref(oracles[t], Q[sel])
            assert_same_fixed(gd[sel], gi[sel], gc[sel], np.asarray(od).reshape(len(sel), -1),
                              np.asarray(oi).reshape(len(sel), -1), oc, f"{fam} tree {t}")


@pytest.mark.parametrize("sorted_", [True, False])
def test_forest_radius_with_per_query_radii(sorted_):
    import torch
    rng = np.random.default_rng(9)
    pts = _forest_data(rng, n_trees=6)
    trees = [kb.ImmutableKdTree.new_from_slice(p) for p in pts]
    oracles = [oracle.OracleTree.build(p) for p in pts]
    forest = kb.Forest(trees)
    nq = 1500
    tree_of = rng.integers(0, len(trees), nq).astype(np.int32)
    Q = rng.normal(size=(nq, 3))
    Q = (Q / np.linalg.norm(Q, axis=1, keepdims=True)).astype(np.float32)
    chord = np.exp(rng.uniform(np.log(1e-3), np.log(0.2), nq))
    radii = (chord ** 2).astype(np.float32)  # SquaredEuclidean radius = chord^2
    b = forest.query(torch.from_numpy(Q).cuda(), torch.from_numpy(tree_of).cuda(),
                     torch.from_numpy(radii).cuda()).within(kb.SquaredEuclidean, 0.0)
    if not sorted_:
        b = b.unsorted()
    g = b.execute_gpu()
    off = g.offsets.cpu().numpy()
    gd = g.distances.cpu().numpy()
    gi = g.items.cpu().numpy().view(np.uint32)
    for j in range(nq):
        o_off, o_d, o_i = oracles[tree_of[j]].within(Q[j:j + 1], float(radii[j]), sorted=sorted_)
        a, e = int(off[j]), int(off[j + 1])
        assert e - a == int(o_off[1]), j
        assert np.array_equal(gd[a:e], o_d) and np.array_equal(gi[a:e], o_i), j


def test_forest_rejects_bad_ids_without_faulting():
    import torch
    rng = np.random.default_rng(10)
    trees = [kb.ImmutableKdTree.new_from_slice(rng.random((500, 3)).astype(np.float32))
             for _ in range(3)]
    forest = kb.Forest(trees)
    Q = rng.random((64, 3)).astype(np.float32)
    tree_of = np.full(64, 7, dtype=np.int32)  # names no tree: empty results
    g = forest.query(torch.from_numpy(Q).cuda(), torch.from_numpy(tree_of).cuda()).nearest_n(
        kb.SquaredEuclidean, 4).execute_gpu()
    assert int(g.counts.sum().item()) == 0


def test_captured_graph_replays_forest_queries():
    import torch
    rng = np.random.default_rng(11)
    pts = _forest_data(rng, n_trees=5)
    trees = [kb.ImmutableKdTree.new_from_slice(p) for p in pts]
    forest = kb.Forest(trees)
    nq = 4096
    Q = torch.from_numpy(rng.random((nq, 3)).astype(np.float32)).cuda()
    T = torch.from_numpy(rng.integers(0, 5, nq).astype(np.int32)).cuda()
    stream = torch.cuda.Stream()
    ref = forest.query(Q, T).nearest_n(kb.SquaredEuclidean, 8).on_stream(stream).execute_gpu()
    torch.cuda.synchronize()
    out = {}
    graph = kb.CapturedGraph(stream)
    with graph:
        out["r"] = forest.query(Q, T).nearest_n(kb.SquaredEuclidean, 8).on_stream(stream).execute_gpu()
    out["r"].distances.fill_(-1)
    graph.replay()
    stream.synchronize()
    assert torch.equal(out["r"].distances, ref.distances)
    assert torch.equal(out["r"].items, ref.items)
