"""Bit-exact parity of the CUDA engine with the CPU oracle, through the C ABI.

Every case builds one tree, uploads the same layout to the GPU and to the
oracle, and compares distances and items bit for bit (integer index work and
the reference's own float arithmetic: no tolerance).
"""
import zlib

import numpy as np
import pytest

import kiddo_b200 as kb
import oracle
from helpers import assert_same_csr, assert_same_fixed, gaussian_mixture, load_kats

pytestmark = pytest.mark.gpu


def _pair(P, items=None):
    t = kb.ImmutableKdTree.new_from_slice(P) if items is None else \
        kb.ImmutableKdTree.new_from_entries(items, P)
    o = oracle.OracleTree.build(P, items)
    return t, o


def _metric(m):
    return {"sqeuclidean": kb.SquaredEuclidean, "manhattan": kb.Manhattan,
            "chebyshev": kb.Chebyshev, "minkowski3": kb.Minkowski(3),
            "minkowski4": kb.Minkowski(4)}[m]


DATASETS = {
    "uniform": lambda rng, n, k, dt: rng.random((n, k)).astype(dt),
    "quantized": lambda rng, n, k, dt: (np.floor(rng.random((n, k)) * 16) / 16).astype(dt),
    "clustered": lambda rng, n, k, dt: (rng.random((8, k))[rng.integers(0, 8, n)]
                                        + rng.normal(0, 0.002, (n, k))).astype(dt),
}


ENGINES = [None, "warp", "thread"]


@pytest.mark.parametrize("engine", ENGINES)
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("dims", [2, 3])
@pytest.mark.parametrize("metric", ["sqeuclidean", "manhattan", "chebyshev",
                                    "minkowski3", "minkowski4"])
@pytest.mark.parametrize("data", ["uniform", "quantized", "clustered"])
def test_fixed_families(dtype, dims, metric, data, engine):
    rng = np.random.default_rng(zlib.crc32(f"{dims}{metric}{data}".encode()))
    n = 20000
    P = DATASETS[data](rng, n, dims, dtype)
    Q = np.concatenate([DATASETS[data](rng, 1500, dims, dtype), P[:200]])  # on-point queries
    t, o = _pair(P)
    M = _metric(metric)
    # nearest_one
    g = t.query(Q).with_engine(engine).nearest_one(M).execute_gpu()
    od, oi = o.nearest_one(Q, metric=metric)
    assert_same_fixed(g.distances, g.items, np.ones(len(Q)), od, oi, np.ones(len(Q)), "nearest_one")
    # approx
    g = t.query(Q).with_engine(engine).nearest_one(M).approx().execute_gpu()
    od, oi = o.approx_nearest_one(Q, metric=metric)
    assert_same_fixed(g.distances, g.items, np.ones(len(Q)), od, oi, np.ones(len(Q)), "approx")
    # nearest_n, sorted and unsorted, and .within
    r = {"sqeuclidean": 0.001, "manhattan": 0.03, "chebyshev": 0.015, "minkowski3": 3e-5,
         "minkowski4": 1e-6}[metric]
    for k in (1, 5, 16, 32):
        g = t.query(Q).with_engine(engine).nearest_n(M, k).execute_gpu()
        assert_same_fixed(g.distances, g.items, g.counts, *o.nearest_n(Q, k, metric=metric),
                          f"nearest_n({k})")
        g = t.query(Q).with_engine(engine).nearest_n(M, k).unsorted().execute_gpu()
        assert_same_fixed(g.distances, g.items, g.counts,
                          *o.nearest_n(Q, k, metric=metric, sorted=False), f"unsorted({k})")
        for excl in (False, True):
            b = t.query(Q).with_engine(engine).nearest_n(M, k).within(r)
            if excl:
                b = b.exclusive_boundaries()
            g = b.execute_gpu()
            assert_same_fixed(g.distances, g.items, g.counts,
                              *o.nearest_n(Q, k, radius=r, metric=metric, exclusive=excl),
                              f"nearest_n({k}).within excl={excl}")
    # best_n_within
    for excl in (False, True):
        b = t.query(Q).with_engine(engine).best_n_within(M, r, 5)
        if excl:
            b = b.exclusive_boundaries()
        g = b.execute_gpu()
        assert_same_fixed(g.distances, g.items, g.counts,
                          *o.best_n_within(Q, r, 5, metric=metric, exclusive=excl), "best_n")


@pytest.mark.parametrize("engine", ENGINES)
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("metric", ["sqeuclidean", "manhattan", "chebyshev",
                                    "minkowski3", "minkowski4"])
@pytest.mark.parametrize("data", ["uniform", "quantized"])
def test_within_families(dtype, metric, data, engine):
    rng = np.random.default_rng(11)
    P = DATASETS[data](rng, 30000, 3, dtype)
    Q = DATASETS[data](rng, 2000, 3, dtype)
    t, o = _pair(P)
    M = _metric(metric)
    # radii giving 0 .. ~7000 hits per query, so every segment-sort path runs
    # (one warp <= 32, shared memory <= 4096, global memory above)
    cases = {"sqeuclidean": ((1e-5, 2000), (3e-4, 2000), (4e-3, 2000), (0.15, 120)),
             "manhattan": ((0.005, 2000), (0.04, 2000), (0.2, 2000), (0.6, 120)),
             "chebyshev": ((0.003, 2000), (0.03, 2000), (0.1, 2000), (0.3, 120)),
             "minkowski3": ((3e-8, 2000), (5e-6, 2000), (2.5e-4, 2000), (0.06, 120)),
             "minkowski4": ((1e-10, 2000), (8e-8, 2000), (1.6e-5, 2000), (0.023, 120))}[metric]
    for r, nq in cases:
        Qr = Q[:nq]
        for excl in (False, True):
            for sorted_ in (True, False):
                b = t.query(Qr).with_engine(engine).within(M, r)
                if not sorted_:
                    b = b.unsorted()
                if excl:
                    b = b.exclusive_boundaries()
                g = b.execute_gpu()
                ref = o.within(Qr, r, metric=metric, exclusive=excl, sorted=sorted_)
                assert_same_csr((g.offsets, g.distances, g.items), ref,
                                f"within r={r} excl={excl} sorted={sorted_}")


@pytest.mark.parametrize("engine", ENGINES)
@pytest.mark.parametrize("n", [0, 1, 2, 31, 32, 33, 47, 64, 65, 1000])
def test_small_and_ragged_trees(n, engine):
    rng = np.random.default_rng(n)
    P = rng.random((n, 3))
    Q = rng.random((300, 3))
    t, o = _pair(P)
    g = t.query(Q).with_engine(engine).nearest_one(kb.SquaredEuclidean).execute_gpu()
    od, oi = o.nearest_one(Q)
    assert_same_fixed(g.distances, g.items, np.ones(300), od, oi, np.ones(300), "nn1")
    g = t.query(Q).with_engine(engine).nearest_n(kb.SquaredEuclidean, 7).execute_gpu()
    assert_same_fixed(g.distances, g.items, g.counts, *o.nearest_n(Q, 7), "nn7")
    g = t.query(Q).with_engine(engine).nearest_one(kb.SquaredEuclidean).approx().execute_gpu()
    od, oi = o.approx_nearest_one(Q)
    assert_same_fixed(g.distances, g.items, np.ones(300), od, oi, np.ones(300), "approx")
    g = t.query(Q).with_engine(engine).within(kb.SquaredEuclidean, 0.05).execute_gpu()
    assert_same_csr((g.offsets, g.distances, g.items), o.within(Q, 0.05), "within")


@pytest.mark.parametrize("engine", ENGINES)
def test_duplicate_heavy_tree(engine):
    """Unsplittable chunks (construction.rs:1137-1150) give long and empty leaves."""
    rng = np.random.default_rng(3)
    P = np.concatenate([np.zeros((900, 3)), np.repeat(rng.random((20, 3)), 40, axis=0),
                        rng.random((3000, 3))])
    Q = np.concatenate([rng.random((500, 3)), P[::50]])
    t, o = _pair(P)
    assert t.max_leaf_len() >= 900
    g = t.query(Q).with_engine(engine).nearest_one(kb.SquaredEuclidean).execute_gpu()
    od, oi = o.nearest_one(Q)
    assert_same_fixed(g.distances, g.items, np.ones(len(Q)), od, oi, np.ones(len(Q)), "nn1")
    for k in (3, 32):
        g = t.query(Q).with_engine(engine).nearest_n(kb.SquaredEuclidean, k).execute_gpu()
        assert_same_fixed(g.distances, g.items, g.counts, *o.nearest_n(Q, k), f"nn{k}")
    g = t.query(Q).with_engine(engine).within(kb.SquaredEuclidean, 0.01).execute_gpu()
    assert_same_csr((g.offsets, g.distances, g.items), o.within(Q, 0.01), "within")


@pytest.mark.parametrize("engine", ENGINES)
def test_explicit_items_best_n(engine):
    rng = np.random.default_rng(5)
    P = rng.random((50000, 3)).astype(np.float32)
    items = rng.permutation(50000).astype(np.uint32)
    Q = rng.random((3000, 3)).astype(np.float32)
    t, o = _pair(P, items)
    for r in (1e-4, 1e-3):
        g = t.query(Q).with_engine(engine).best_n_within(kb.SquaredEuclidean, r, 5).execute_gpu()
        assert_same_fixed(g.distances, g.items, g.counts, *o.best_n_within(Q, r, 5), "best_n")


@pytest.mark.parametrize("engine", ENGINES)
def test_gaussian_mixture_knn16(engine):
    """Medium case with the C2 shape (f32 mixture, dense clumps, in-leaf ties)."""
    rng = np.random.default_rng(2)
    P = gaussian_mixture(1_000_000, 1024, 0.005, 0.2, rng)
    Q = gaussian_mixture(50_000, 1024, 0.005, 0.2, rng)
    t, o = _pair(P)
    g = t.query(Q).with_engine(engine).nearest_n(kb.SquaredEuclidean, 16).execute_gpu()
    assert_same_fixed(g.distances, g.items, g.counts, *o.nearest_n(Q, 16), "gm knn16")
    g = t.query(Q).with_engine(engine).nearest_one(kb.SquaredEuclidean).approx().execute_gpu()
    od, oi = o.approx_nearest_one(Q)
    assert_same_fixed(g.distances, g.items, np.ones(len(Q)), od, oi, np.ones(len(Q)), "gm approx")


def test_device_buffers_match_host_buffers():
    import torch
    rng = np.random.default_rng(9)
    P = rng.random((100000, 3)).astype(np.float32)
    Q = rng.random((20000, 3)).astype(np.float32)
    t = kb.ImmutableKdTree.new_from_slice(P)
    h = t.query(Q).nearest_n(kb.SquaredEuclidean, 16).execute_gpu()
    dq = torch.from_numpy(Q).cuda()
    d = t.query(dq).nearest_n(kb.SquaredEuclidean, 16).execute_gpu()
    torch.cuda.synchronize()
    assert np.array_equal(d.distances.cpu().numpy(), h.distances)
    assert np.array_equal(d.items.cpu().numpy().view(np.uint32), h.items)
    # host buffers fill nearest_n's counts as min(k, size) on the host and
    # copy back only chunks with shorter rows (NaN queries find nothing)
    assert np.array_equal(d.counts.cpu().numpy().view(np.uint32), h.counts)
    Qn = Q.copy()
    Qn[::997] = np.nan
    hn = t.query(Qn).nearest_n(kb.SquaredEuclidean, 16).execute_gpu()
    dn = t.query(torch.from_numpy(Qn).cuda()).nearest_n(kb.SquaredEuclidean, 16).execute_gpu()
    assert np.array_equal(dn.counts.cpu().numpy().view(np.uint32), hn.counts)
    assert np.all(hn.counts[::997] == 0) and (hn.counts == 16).sum() == len(Q) - len(Q[::997])
    hw = t.query(Q).within(kb.SquaredEuclidean, 1e-4).execute_gpu()
    dw = t.query(dq).within(kb.SquaredEuclidean, 1e-4).execute_gpu()
    assert np.array_equal(dw.offsets.cpu().numpy().astype(np.uint64), hw.offsets)
    assert np.array_equal(dw.distances.cpu().numpy(), hw.distances)


def test_known_answers_on_gpu():
    for kat in load_kats():
        if "box" in kat:
            continue  # periodic KATs run in test_gpu_periodic
        P = kat["np_points"]
        t = kb.ImmutableKdTree.new_from_slice(P) if kat["np_items"] is None else \
            kb.ImmutableKdTree.new_from_entries(kat["np_items"], P)
        o = oracle.OracleTree.build(P, kat["np_items"])
        for chk in kat["checks"]:
            q = np.asarray([chk["query"]], dtype=P.dtype)
            M = _metric(chk.get("metric", "sqeuclidean"))
            fam = chk["family"]
            if fam == "nearest_one":
                g = t.query(q).nearest_one(M).execute_gpu()
                items = g.items.tolist()
            elif fam == "nearest_n":
                g = t.query(q).nearest_n(M, chk["k"]).execute_gpu()
                items = g.items[0, :g.counts[0]].tolist()
                if "expect_dists" in chk:
                    assert g.distances[0, :g.counts[0]].tolist() == chk["expect_dists"]
            else:
                b = t.query(q).within(M, chk["radius"])
                if chk.get("exclusive"):
                    b = b.exclusive_boundaries()
                g = b.execute_gpu()
                items = g.items.tolist()
                ref = o.within(q, chk["radius"], metric=chk.get("metric", "sqeuclidean"),
                               exclusive=chk.get("exclusive", False))
                assert_same_csr((g.offsets, g.distances, g.items), ref, kat["name"])
            if "expect_items" in chk:
                assert items == chk["expect_items"], kat["name"]
            if "expect_first_item" in chk:
                assert items[0] == chk["expect_first_item"], kat["name"]
            if "expect_item_set" in chk:
                assert sorted(items) == chk["expect_item_set"], kat["name"]


def test_engines_report_identical_traversal_counters():
    """Both kernels walk exactly the reference's traversal: equal stem, leaf and
    point counts (exact_query_stats.rs:23-60) for every query family."""
    rng = np.random.default_rng(21)
    P = rng.random((40000, 3)).astype(np.float32)
    Q = rng.random((5000, 3)).astype(np.float32)
    t = kb.ImmutableKdTree.new_from_slice(P)
    o = oracle.OracleTree.build(P)
    for fam in ("nn1", "approx", "knn", "best", "within"):
        stats = []
        for engine in ("warp", "thread"):
            b = t.query(Q).with_engine(engine)
            if fam == "nn1":
                b = b.nearest_one(kb.SquaredEuclidean)
            elif fam == "approx":
                b = b.nearest_one(kb.SquaredEuclidean).approx()
            elif fam == "knn":
                b = b.nearest_n(kb.SquaredEuclidean, 16)
            elif fam == "best":
                b = b.best_n_within(kb.SquaredEuclidean, 1e-3, 5)
            else:
                b = b.within(kb.SquaredEuclidean, 1e-3)
            stats.append(b.traversal_stats())
        assert np.array_equal(stats[0], stats[1]), fam
        if fam == "knn":
            _, _, _, ost = o.nearest_n(Q, 16, stats=True)
            assert np.array_equal(stats[0], ost)


@pytest.mark.parametrize("engine", ["warp", "thread"])
def test_spatial_order_gives_identical_results(engine):
    rng = np.random.default_rng(31)
    P = gaussian_mixture(200_000, 64, 0.01, 0.2, rng)
    Q = gaussian_mixture(30_000, 64, 0.01, 0.2, rng)
    t, o = _pair(P)
    g = t.query(Q).with_engine(engine).with_spatial_order().nearest_n(kb.SquaredEuclidean, 16).execute_gpu()
    assert_same_fixed(g.distances, g.items, g.counts, *o.nearest_n(Q, 16), "ordered knn16")
    g = t.query(Q).with_engine(engine).with_spatial_order().nearest_one(kb.SquaredEuclidean).execute_gpu()
    od, oi = o.nearest_one(Q)
    assert_same_fixed(g.distances, g.items, np.ones(len(Q)), od, oi, np.ones(len(Q)), "ordered nn1")
    g = t.query(Q).with_engine(engine).with_spatial_order().within(kb.SquaredEuclidean, 1e-4).execute_gpu()
    assert_same_csr((g.offsets, g.distances, g.items), o.within(Q, 1e-4), "ordered within")


def test_autotuner_caches_a_choice_and_keeps_results(tmp_path, monkeypatch):
    import torch
    monkeypatch.setenv("KIDDO_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    rng = np.random.default_rng(41)
    P = rng.random((300_000, 3)).astype(np.float32)
    Q = torch.from_numpy(rng.random((100_000, 3)).astype(np.float32)).cuda()
    t = kb.ImmutableKdTree.new_from_slice(P)
    plain = t.query(Q).nearest_n(kb.SquaredEuclidean, 16).execute_gpu()
    b = t.query(Q).nearest_n(kb.SquaredEuclidean, 16).autotuned()
    assert b.engine in ("warp", "thread", "coop")
    tuned = b.execute_gpu()
    assert torch.equal(plain.distances, tuned.distances) and torch.equal(plain.items, tuned.items)
    import json
    db = json.loads((tmp_path / "tune.json").read_text())
    entry = next(iter(db.values()))
    assert len(db) == 1 and {"engine", "spatial_order", "refill", "chunk"} <= set(entry)
    # stage 1 covers 3 engines x 2 orders, then 4 refill and 4 chunk settings
    assert len(entry["ms"]) >= 6 + 4
    # a second builder of the same kind takes the cached choice
    b2 = t.query(Q).nearest_n(kb.SquaredEuclidean, 16).autotuned(tune_if_missing=False)
    assert (b2.engine, b2.refill, b2.chunk) == (entry["engine"], entry["refill"], entry["chunk"])


@pytest.mark.parametrize("engine", ["thread", "coop", "warp"])
def test_launch_knobs_keep_results(engine):
    """The refill threshold and the chunk size change only the schedule."""
    import torch
    rng = np.random.default_rng(43)
    P = gaussian_mixture(200_000, 64, 0.01, 0.2, rng)
    Q = torch.from_numpy(gaussian_mixture(100_000, 64, 0.01, 0.2, rng)).cuda()
    t, o = _pair(P)
    ref = o.nearest_n(Q.cpu().numpy(), 16)
    for refill, chunk in ((1, 32), (8, 256), (32, 1024), (None, 128)):
        g = (t.query(Q).with_engine(engine).with_tuning(refill, chunk)
             .nearest_n(kb.SquaredEuclidean, 16).execute_gpu())
        assert_same_fixed(g.distances.cpu().numpy(), g.items.cpu().numpy(), g.counts.cpu().numpy(),
                          *ref, f"refill={refill} chunk={chunk}")
        g = (t.query(Q).with_engine(engine).with_tuning(refill, chunk)
             .within(kb.SquaredEuclidean, 1e-4).execute_gpu())
        assert_same_csr((g.offsets.cpu().numpy(), g.distances.cpu().numpy(),
                         g.items.cpu().numpy()), o.within(Q.cpu().numpy(), 1e-4), "within")
