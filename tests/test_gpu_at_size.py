"""Parity at the benchmark configurations' own sizes, on the paths the
benchmark times.

- The pipelined host-buffer path (2M-query chunks over three streams with
  eighth-length first and last chunks and slot reuse) on batches of several
  chunks, every row against the oracle.
- The nearest_one configuration in full: f64, 100,000 uniform points, 1,000,000
  uniform queries, every row, device and host buffers.
- The 16M-point configurations (f32 Gaussian mixture kNN16 and approx; f64
  periodic neighbour lists) and the 256-catalogue forest: the whole batch runs
  on the device in its default path (leaf-grouped order included), then
  100,000 seeded sampled rows are compared with the oracle.

The data comes from bench.py's own generators, so these are the arrays the
benchmark times.  Bit-exact throughout (integer and index work, and the
reference's own float arithmetic).
"""
import numpy as np
import pytest

import bench
import kiddo_b200 as kb
import oracle
from helpers import assert_same_csr, assert_same_fixed, gaussian_mixture

pytestmark = pytest.mark.gpu

SE = kb.SquaredEuclidean
CHUNK = 1 << 21  # the host pipeline's chunk (KGPU_HOST_CHUNK_LOG2)
SAMPLE = 100_000


def _oracle_of(tree):
    """The oracle over the product tree's own layout."""
    return oracle.OracleTree.from_layout(oracle.Layout(
        tree.dtype, tree.dims, tree.stems(), tree.leaf_bytes(), tree.leaf_extents(),
        tree.max_stem_level(), tree.size(), tree.max_leaf_len()))


def _pinned(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()


def _rows(x, rows):
    import torch
    r = torch.from_numpy(rows).to(x.device)
    return x.index_select(0, r).cpu().numpy()


def _sample(n, seed=2024):
    return np.sort(np.random.default_rng(seed).choice(n, size=min(SAMPLE, n), replace=False))


@pytest.mark.parametrize("nq", [CHUNK + 1000, 5_500_001])
def test_host_pipeline_multi_chunk(nq):
    """nq = 2M + 1000: two slots, three chunks (edge, middle, edge).
    nq = 5.5M: three slots, five chunks, slots 0 and 1 reused."""
    rng = np.random.default_rng(nq)
    P = gaussian_mixture(200_000, 256, 0.01, 0.2, rng)
    Q = _pinned(gaussian_mixture(nq, 256, 0.01, 0.2, rng))
    t = kb.ImmutableKdTree.new_from_slice(P)
    o = oracle.OracleTree.build(P)
    g = t.query(Q).nearest_n(SE, 16).execute_gpu()
    assert_same_fixed(g.distances, g.items, g.counts, *o.nearest_n(Q, 16), "host knn16")
    del g
    # rows whose query holds a NaN find no candidate (count 0): the pipeline
    # fills nearest_n's counts on the host and brings back the chunks with
    # short rows, here the first chunk and a later one
    Qn = Q.copy()
    Qn[[3, 17, nq - 5, nq // 2]] = np.nan
    g = t.query(Qn).nearest_n(SE, 16).execute_gpu()
    assert_same_fixed(g.distances, g.items, g.counts, *o.nearest_n(Qn, 16), "host knn16 nan rows")
    assert (g.counts == 0).sum() == 4
    del g, Qn
    g = t.query(Q).nearest_one(SE).execute_gpu()
    od, oi = o.nearest_one(Q)
    assert_same_fixed(g.distances, g.items, np.ones(nq), od, oi, np.ones(nq), "host nn1")
    g = t.query(Q).nearest_one(SE).approx().execute_gpu()
    od, oi = o.approx_nearest_one(Q)
    assert_same_fixed(g.distances, g.items, np.ones(nq), od, oi, np.ones(nq), "host approx")


def test_host_pipeline_periodic_multi_chunk():
    """The periodic neighbour-list family (nearest_n(32).within(0.01) in a
    unit box, f64) through the host pipeline: 5 chunks over 3 slots."""
    nq = 4 * CHUNK + 12_345
    P = bench.periodic_particles(100_000, np.random.default_rng(51), np.float64)
    Q = _pinned(bench.periodic_particles(nq, np.random.default_rng(52), np.float64))
    t = kb.ImmutableKdTree.new_from_slice(P)
    o = oracle.OracleTree.build(P)
    box = np.ones(3)
    g = (t.query(Q).periodic_boundary_condition(box).nearest_n(SE, 32)
         .within(bench.C5_RADIUS).execute_gpu())
    ref = o.periodic_nearest_n(Q, box, 32, radius=bench.C5_RADIUS)
    assert_same_fixed(g.distances, g.items, g.counts, *ref, "host periodic nn32")


def test_c1_nearest_one_full_size():
    """f64, 100,000 points U[0,1)^3 (seed 0), 1,000,000 queries (seed 1),
    nearest_one: every row, device buffers and pinned host buffers."""
    import torch
    P, Q = bench.make_data("c1_nn1", 0)
    assert P.shape == (100_000, 3) and Q.shape == (1_000_000, 3) and P.dtype == np.float64
    t = kb.ImmutableKdTree.new_from_slice(P)
    o = oracle.OracleTree.build(P)
    lay = o.layout()
    assert np.array_equal(t.stems(), lay.stems) and np.array_equal(t.leaf_bytes(), lay.leaf_bytes)
    od, oi = o.nearest_one(Q)
    g = t.query(torch.from_numpy(Q).cuda()).nearest_one(SE).execute_gpu()
    assert_same_fixed(g.distances.cpu().numpy(), g.items.cpu().numpy(), np.ones(len(Q)), od, oi,
                      np.ones(len(Q)), "c1 device")
    g = t.query(_pinned(Q)).nearest_one(SE).execute_gpu()
    assert_same_fixed(g.distances, g.items, np.ones(len(Q)), od, oi, np.ones(len(Q)), "c1 host")


@pytest.fixture(scope="module")
def c2():
    P, Q = bench.make_data("c2_knn16", 0)
    t = kb.ImmutableKdTree.new_from_slice(P)
    o = oracle.OracleTree.build(P)
    lay = o.layout()
    # the product builder and the oracle lay the 16M-point tree out byte for byte alike
    assert np.array_equal(t.stems(), lay.stems)
    assert np.array_equal(t.leaf_bytes(), lay.leaf_bytes)
    assert np.array_equal(t.leaf_extents(), lay.extents)
    return P, Q, t, o


def test_c2_knn16_full_batch_sampled(c2):
    """16M mixture points, all 16M queries in one call (leaf-grouped order on,
    as by default at this size), 100,000 sampled rows against the oracle."""
    import torch
    _, Q, t, o = c2
    rows = _sample(len(Q))
    g = t.query(torch.from_numpy(Q).cuda()).nearest_n(SE, 16).execute_gpu()
    assert_same_fixed(_rows(g.distances, rows), _rows(g.items, rows), _rows(g.counts, rows),
                      *o.nearest_n(Q[rows], 16), "c2 knn16 device")
    del g
    torch.cuda.empty_cache()
    # the end-to-end path: pinned host queries, 8 chunks over 3 slots
    h = t.query(_pinned(Q)).nearest_n(SE, 16).execute_gpu()
    assert_same_fixed(h.distances[rows], h.items[rows], h.counts[rows],
                      *o.nearest_n(Q[rows], 16), "c2 knn16 host")


def test_c2_approx_full_batch_sampled(c2):
    import torch
    _, Q, t, o = c2
    rows = _sample(len(Q), 7)
    g = t.query(torch.from_numpy(Q).cuda()).nearest_one(SE).approx().execute_gpu()
    od, oi = o.approx_nearest_one(Q[rows])
    assert_same_fixed(_rows(g.distances, rows), _rows(g.items, rows), np.ones(len(rows)), od, oi,
                      np.ones(len(rows)), "c2 approx")


def test_c5_periodic_full_batch_sampled():
    """16M f64 particles, every particle queries nearest_n(32).within(0.01)
    in the periodic unit box: the whole batch on the device, 100,000 sampled
    rows against the oracle."""
    import torch
    P, Q = bench.make_data("c5_periodic", 0)
    assert Q is P and P.shape == (16_000_000, 3)
    t = kb.ImmutableKdTree.new_from_slice(P)
    o = _oracle_of(t)
    box = np.ones(3)
    rows = _sample(len(Q), 11)
    g = (t.query(torch.from_numpy(Q).cuda()).periodic_boundary_condition(box).nearest_n(SE, 32)
         .within(bench.C5_RADIUS).execute_gpu())
    ref = o.periodic_nearest_n(Q[rows], box, 32, radius=bench.C5_RADIUS)
    assert_same_fixed(_rows(g.distances, rows), _rows(g.items, rows), _rows(g.counts, rows), *ref,
                      "c5 periodic nn32")
    del g
    torch.cuda.empty_cache()


def _csr_rows(res, rows):
    """(offsets, distances, items) of the chosen rows of a device CSR result."""
    import torch
    off = res.offsets.cpu().numpy().astype(np.int64)
    a, b = off[rows], off[rows + 1]
    lens = b - a
    idx = np.repeat(a - np.concatenate([[0], np.cumsum(lens)[:-1]]), lens) + np.arange(lens.sum())
    ti = torch.from_numpy(idx).to(res.distances.device)
    d = res.distances.index_select(0, ti).cpu().numpy() if len(idx) else np.zeros(0)
    i = res.items.index_select(0, ti).cpu().numpy().view(np.uint32) if len(idx) else np.zeros(0)
    return np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64), d, i


def test_c3_forest_full_batch_sampled():
    """The 256 catalogues (about 120M unit vectors, Pareto ranks as items) and
    64M queries with per-query radii: each family's batch in one forest call,
    then sampled rows of each against the oracle tree of the query's
    catalogue."""
    import torch
    pts, items, Q, tree_of, radii, family = bench.forest_workload(1.0)
    trees = [kb.ImmutableKdTree.new_from_entries(it, p) for it, p in zip(items, pts)]
    forest = kb.Forest(trees)
    oracles = [_oracle_of(t) for t in trees]
    del pts
    rng = np.random.default_rng(33)
    for fam in range(3):
        sel = np.nonzero(family == fam)[0]
        q, tof, rad = Q[sel], tree_of[sel], radii[sel]
        b = forest.query(torch.from_numpy(q).cuda(), torch.from_numpy(tof).cuda(),
                         torch.from_numpy(rad).cuda())
        if fam == 0:
            g = b.within(SE, 0.0).execute_gpu()
        elif fam == 1:
            g = b.within(SE, 0.0).unsorted().execute_gpu()
        else:
            g = b.best_n_within(SE, 0.0, 5).execute_gpu()
        rows = np.sort(rng.choice(len(sel), size=min(SAMPLE // 3, len(sel)), replace=False))
        if fam < 2:
            go, gd, gi = _csr_rows(g, rows)
        else:
            gd, gi, gc = _rows(g.distances, rows), _rows(g.items, rows), _rows(g.counts, rows)
        pos = 0
        for tr in np.unique(tof[rows]):
            r = rows[tof[rows] == tr]
            if fam < 2:
                oo, od, oi = oracles[tr].within(q[r], rad[r], sorted=(fam == 0))
                m = np.nonzero(tof[rows] == tr)[0]
                sub_off = go[m]
                lens = go[m + 1] - sub_off
                assert np.array_equal(lens.astype(np.int64), np.diff(oo).astype(np.int64)), \
                    f"family {fam} tree {tr}: hit counts differ"
                idx = np.concatenate([np.arange(a, a + n) for a, n in
                                      zip(sub_off.astype(np.int64), lens.astype(np.int64))]) \
                    if lens.sum() else np.zeros(0, np.int64)
                assert_same_csr((oo, gd[idx], gi[idx]), (oo, od, oi), f"fam {fam} tree {tr}")
            else:
                m = tof[rows] == tr
                assert_same_fixed(gd[m], gi[m], gc[m], *oracles[tr].best_n_within(q[r], rad[r], 5),
                                  f"best_n tree {tr}")
            pos += len(r)
        assert pos == len(rows)
        del g
        torch.cuda.empty_cache()
