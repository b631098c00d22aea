"""Pin the CPU oracle: the reference's literal known-answer tests and its own
brute-force parity rules (tests/kd_tree_fuzz_v6.rs:244-340, 682-734, 960-1029)."""
import json
import os

import numpy as np
import pytest

import oracle
from helpers import brute_dists, compare_nearest_n_reference_rule, load_kats, ulps_apart

KATS = load_kats()


def run_check(tree, kat, chk):
    q = np.asarray([chk["query"]], dtype=kat["np_points"].dtype)
    fam = chk["family"]
    metric = chk.get("metric", "sqeuclidean")
    if fam == "nearest_one":
        d, i = tree.nearest_one(q, metric=metric)
        return d, i
    if fam == "nearest_n":
        d, i, c = tree.nearest_n(q, chk["k"], radius=chk.get("radius", np.inf), metric=metric)
        return d[0, :c[0]], i[0, :c[0]]
    if fam in ("within", "within_brute"):
        off, d, i = tree.within(q, chk["radius"], metric=metric, exclusive=chk.get("exclusive", False))
        return d, i
    if fam == "periodic_nearest_one":
        d, i = tree.periodic_nearest_one(q, kat["box"], metric=metric)
        return d, i
    if fam == "periodic_nearest_n":
        d, i, c = tree.periodic_nearest_n(q, kat["box"], chk["k"], radius=chk.get("radius", np.inf),
                                          metric=metric)
        return d[0, :c[0]], i[0, :c[0]]
    raise AssertionError(fam)


def verify(kat, chk, d, i):
    d = np.asarray(d)
    i = np.asarray(i)
    if "expect_items" in chk:
        assert i.tolist() == chk["expect_items"], (kat["name"], chk)
    if "expect_dists" in chk:
        assert d.tolist() == chk["expect_dists"]
    if "expect_first_item" in chk:
        assert int(i[0]) == chk["expect_first_item"]
    if "expect_len" in chk:
        assert len(i) == chk["expect_len"]
    if "expect_item_set" in chk:
        assert sorted(i.tolist()) == chk["expect_item_set"]
    if chk.get("expect_dist_is_manual_sq"):
        pts = kat["np_points"]
        qq = np.asarray(chk["query"])
        for dd, ii in zip(d, i):
            manual = (qq[0] - pts[ii][0]) ** 2 + (qq[1] - pts[ii][1]) ** 2
            assert dd == manual
    if chk["family"] == "within_brute":
        pts = kat["np_points"]
        bd = brute_dists(pts, chk["query"], chk["metric"])
        sel = np.nonzero(bd <= np.asarray(chk["radius"], dtype=pts.dtype))[0]
        exp = sorted(zip(bd[sel].tolist(), sel.tolist()))
        got = sorted(zip(d.tolist(), i.tolist()))
        assert got == exp


@pytest.mark.parametrize("kat", KATS, ids=[k["name"] for k in KATS])
def test_oracle_known_answers(kat):
    t = oracle.OracleTree.build(kat["np_points"], kat["np_items"])
    for chk in kat["checks"]:
        d, i = run_check(t, kat, chk)
        verify(kat, chk, d, i)


def test_metric_known_answers():
    """The reference's metric unit tests (dist/mod.rs:1436-1490): point
    distances and the rectangle update of each metric, f64 3-D."""
    a, b = [1.0, 2.0, 3.0], [4.0, 2.0, -1.0]
    assert oracle.metric_f64x3("sqeuclidean", a, b, 0, [0, 0, 0], 0, 0)[0] == 25.0
    assert oracle.metric_f64x3("manhattan", a, b, 0, [0, 0, 0], 0, 0)[0] == 7.0
    assert oracle.metric_f64x3("manhattan", a, b, 7.0, [0.0, 2.0, 5.0], 1, 4.0)[1] == 9.0
    assert oracle.metric_f64x3("chebyshev", a, [4.0, 2.5, -1.0], 0, [0, 0, 0], 0, 0)[0] == 4.0
    # Chebyshev re-scans every offset, the changed axis taking its new one
    assert oracle.metric_f64x3("chebyshev", a, b, 5.0, [0.0, 2.0, 5.0], 2, 1.0)[1] == 2.0
    assert oracle.metric_f64x3("chebyshev", a, b, 5.0, [0.0, 2.0, 5.0], 0, 6.0)[1] == 6.0
    # a NaN component is not greater than the accumulator, so it is passed over
    assert oracle.metric_f64x3("chebyshev", [np.nan, 2.0, 3.0], b, 0, [0, 0, 0], 0, 0)[0] == 4.0
    # Minkowski<3>: sum of |dx|^3 (dist/mod.rs:1497-1507)
    assert oracle.metric_f64x3("minkowski3", a, [4.0, 2.5, -1.0], 0, [0, 0, 0], 0, 0)[0] == 91.125
    assert oracle.metric_f64x3("minkowski4", a, [4.0, 2.5, -1.0], 0, [0, 0, 0], 0, 0)[0] == \
        81.0 + 0.0625 + 256.0


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("metric", ["sqeuclidean", "manhattan", "chebyshev", "minkowski3",
                                    "minkowski4"])
@pytest.mark.parametrize("n", [1, 31, 33, 1000, 20000])
def test_oracle_vs_brute_force(dtype, metric, n):
    rng = np.random.default_rng(n)
    P = rng.random((n, 3)).astype(dtype)
    Q = rng.random((60, 3)).astype(dtype)
    t = oracle.OracleTree.build(P)
    d1, i1 = t.nearest_one(Q, metric=metric)
    k = 8
    dn, inn, cn = t.nearest_n(Q, k, metric=metric)
    r = np.asarray({"sqeuclidean": 0.02, "manhattan": 0.2, "chebyshev": 0.08,
                    "minkowski3": 0.002, "minkowski4": 0.0002}[metric], dtype=dtype)
    off, dw, iw = t.within(Q, float(r), metric=metric)
    bd_, bi_, bc_ = t.best_n_within(Q, float(r), 5, metric=metric)
    for j in range(len(Q)):
        bd = brute_dists(P, Q[j], metric)
        # nearest_one: any member of the tied best set (fuzz_v6.rs:682-734)
        assert d1[j] == bd.min()
        assert bd[i1[j]] == bd.min()
        order = np.lexsort((np.arange(n), bd))
        kk = min(k, n)
        compare_nearest_n_reference_rule(dn[j, :cn[j]], inn[j, :cn[j]], bd[order[:kk]],
                                         order[:kk], k)
        sel = np.nonzero(bd <= r)[0]
        a, b = int(off[j]), int(off[j + 1])
        assert sorted(iw[a:b].tolist()) == sorted(sel.tolist())
        assert np.all(np.diff(dw[a:b]) >= 0)
        # best_n: within-set sorted by item, truncated (fuzz_v6.rs:1020-1029)
        exp_best = sorted(sel.tolist())[:5]
        assert bi_[j, :bc_[j]].tolist() == exp_best


@pytest.mark.parametrize("k", [33, 100, 256])
def test_oracle_large_k_vs_brute_force(k):
    """nearest_n beyond the fixed-size lists (ThresholdVec up to 192, BinaryHeap
    above): the k smallest by the reference's brute-force rule
    (tests/kd_tree_fuzz_v6.rs:272-340)."""
    rng = np.random.default_rng(k)
    P = rng.random((20000, 3))
    Q = rng.random((40, 3))
    t = oracle.OracleTree.build(P)
    dn, inn, cn = t.nearest_n(Q, k)
    for j in range(len(Q)):
        bd = brute_dists(P, Q[j])
        order = np.lexsort((np.arange(len(P)), bd))
        compare_nearest_n_reference_rule(dn[j, :cn[j]], inn[j, :cn[j]], bd[order[:k]],
                                         order[:k], k)
    # best_n_within: the within-set sorted by item, truncated (fuzz_v6.rs:1020-1029)
    bd_, bi_, bc_ = t.best_n_within(Q, 0.01, k)
    for j in range(len(Q)):
        sel = np.nonzero(brute_dists(P, Q[j]) <= 0.01)[0]
        assert bi_[j, :bc_[j]].tolist() == sorted(sel.tolist())[:k]


def test_oracle_periodic_vs_brute_force():
    rng = np.random.default_rng(7)
    P = rng.random((5000, 3))
    Q = np.concatenate([rng.random((50, 3)), rng.random((50, 3)) * 0.02,
                        1 - rng.random((50, 3)) * 0.02])
    box = np.ones(3)
    t = oracle.OracleTree.build(P)
    d, i = t.periodic_nearest_one(Q, box)
    dn, inn, cn = t.periodic_nearest_n(Q, box, 32, radius=0.01)
    for j in range(len(Q)):
        delta = np.abs(P - Q[j])
        delta = np.where(box - delta < delta, box - delta, delta)
        bd = ((delta[:, 0] ** 2 + delta[:, 1] ** 2) + delta[:, 2] ** 2)
        # the image queries measure (p - (q +/- L))^2 with q +/- L rounded, the
        # brute force the min-image delta: equal within the reference's
        # REL_EPS_F64 = 1e-12 (kd_tree/query/nearest_one.rs tests)
        assert abs(d[j] - bd.min()) <= 1e-12 * bd.min()
        sel = np.sort(bd[bd <= 0.01])[:32]
        assert np.array_equal(np.sort(dn[j, :cn[j]]), sel)


# ---------------------------------------------------------------------------
# Donnelly stem strategy (stem_strategy/donnelly/core.rs)
# ---------------------------------------------------------------------------
def test_donnelly_index_math_matches_reference_cases():
    """The reference's own DonnellyCore::<3> cases (core.rs tests, extracted by
    tests/golden/make_golden.py): stem index after a path, and both children
    of the node a path reaches."""
    kats = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "kats.json")))
    for c in kats["donnelly_paths"]:
        idx, _ = oracle.donnelly_path(c["bh"], c["path"])
        assert idx == c["stem_idx"], c
    for c in kats["donnelly_children"]:
        _, ch = oracle.donnelly_path(c["bh"], c["path"])
        assert list(ch) == c["children"], c


@pytest.mark.parametrize("bh", [3, 4])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_donnelly_tree_matches_brute_force_and_eytzinger(bh, dtype):
    """A Donnelly<bh> tree answers every family like brute force and like the
    Eytzinger tree of the same points (equal-distance groups as multisets, the
    reference's fuzz rule kd_tree_fuzz_v6.rs:244-340)."""
    rng = np.random.default_rng(100 + bh)
    for n in (1, 31, 33, 100, 2000, 7000):
        P = rng.random((n, 3)).astype(dtype)
        Q = np.concatenate([rng.random((300, 3)).astype(dtype), P[:50]])
        don = oracle.OracleTree.build(P, block_height=bh)
        eyt = oracle.OracleTree.build(P)
        lay = don.layout()
        assert lay.block_height == bh
        dd, di = don.nearest_one(Q)
        ed, ei = eyt.nearest_one(Q)
        assert np.array_equal(dd, ed)
        bd = ((Q[:, None, :].astype(np.float64) - P[None, :, :]) ** 2).sum(-1)
        assert np.allclose(dd, bd.min(1), rtol=1e-5, atol=1e-12)
        for k in (1, 5, 16):
            d1, i1, c1 = don.nearest_n(Q, k)
            d2, i2, c2 = eyt.nearest_n(Q, k)
            assert np.array_equal(d1, d2) and np.array_equal(c1, c2)
            for a, b, dist in zip(i1, i2, d1):
                # items may differ only inside equal-distance groups
                for v in np.unique(dist):
                    m = dist == v
                    assert sorted(a[m]) == sorted(b[m])
        r = 0.05 if dtype == np.float32 else 0.05
        o1, wd1, wi1 = don.within(Q, r)
        o2, wd2, wi2 = eyt.within(Q, r)
        assert np.array_equal(o1, o2)
        for j in range(len(Q)):
            s1 = sorted(zip(wd1[o1[j]:o1[j + 1]].tolist(), wi1[o1[j]:o1[j + 1]].tolist()))
            s2 = sorted(zip(wd2[o2[j]:o2[j + 1]].tolist(), wi2[o2[j]:o2[j + 1]].tolist()))
            assert s1 == s2
        b1 = don.best_n_within(Q, r, 4)
        b2 = eyt.best_n_within(Q, r, 4)
        assert np.array_equal(b1[1], b2[1]) and np.array_equal(b1[2], b2[2])
        a1 = don.approx_nearest_one(Q)[0]
        assert np.all(a1 >= dd)


def test_timing_build_matches_the_checker():
    """The timed CPU baseline (the oracle's source at -O3 -march=native, built
    on this host) answers the benchmarked families bit for bit like the -O2
    checker, and builds the same tree; a mismatch would mean the timed code is
    not the checked code."""
    T = oracle.timing_lib()
    rng = np.random.default_rng(77)
    for dtype in (np.float32, np.float64):
        P = np.concatenate([rng.random((30_000, 3)),
                            np.floor(rng.random((5_000, 3)) * 8) / 8]).astype(dtype)
        Q = np.concatenate([rng.random((4_000, 3)), P[:500]]).astype(dtype)
        a = oracle.OracleTree.build(P)
        b = oracle.OracleTree.build(P, L=T)
        la, lb = a.layout(), b.layout()
        assert np.array_equal(la.stems, lb.stems) and np.array_equal(la.leaf_bytes, lb.leaf_bytes)
        for x, y in ((a.nearest_one(Q), b.nearest_one(Q)),
                     (a.approx_nearest_one(Q), b.approx_nearest_one(Q)),
                     (a.nearest_n(Q, 16), b.nearest_n(Q, 16)),
                     (a.periodic_nearest_n(Q, np.ones(3), 32, radius=0.01),
                      b.periodic_nearest_n(Q, np.ones(3), 32, radius=0.01)),
                     (a.best_n_within(Q, 1e-3, 5), b.best_n_within(Q, 1e-3, 5)),
                     (a.within(Q, 1e-3), b.within(Q, 1e-3))):
            for u, v in zip(x, y):
                assert np.array_equal(u, v)


@pytest.mark.parametrize("metric", ["sqeuclidean", "manhattan", "chebyshev", "minkowski3",
                                    "minkowski4"])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_periodic_families_match_min_image_brute_force(metric, dtype):
    """periodic.rs is generic over the metric: the plural families scan leaves
    with combine_component over min-image components (periodic.rs:272-284,
    357-400), so their results equal a brute-force min-image scan; nearest_one
    (home query plus shifted images, :156-214) agrees up to the rounding of
    the shifted query."""
    rng = np.random.default_rng(len(metric) + (dtype == np.float64))
    P = rng.random((3000, 3)).astype(dtype)
    Q = np.concatenate([rng.random((150, 3)), rng.random((40, 3)) * 0.01,
                        1 - rng.random((40, 3)) * 0.01]).astype(dtype)
    box = np.ones(3, dtype)
    o = oracle.OracleTree.build(P)

    def min_image(q):
        acc = np.zeros(len(P), dtype)
        for d in range(3):
            delta = np.abs((q[d] - P[:, d]).astype(dtype))
            w = (box[d] - delta).astype(dtype)
            m = np.where(w < delta, w, delta)
            if metric == "chebyshev":
                acc = np.where(m > acc, m, acc).astype(dtype)
            elif metric == "sqeuclidean":
                acc = (acc + m * m).astype(dtype)
            elif metric == "manhattan":
                acc = (acc + m).astype(dtype)
            else:
                x2 = (m * m).astype(dtype)
                acc = (acc + ((m * x2) if metric == "minkowski3" else (x2 * x2))).astype(dtype)
        return acc

    d, i, c = o.periodic_nearest_n(Q, box, 10, metric=metric)
    nd, ni = o.periodic_nearest_one(Q, box, metric=metric)
    r = {"chebyshev": 0.05, "minkowski3": 1e-4, "minkowski4": 1e-5, "sqeuclidean": 2e-3,
         "manhattan": 0.08}[metric]
    off, wd, wi = o.periodic_within(Q, box, r, metric=metric)
    for j, q in enumerate(Q):
        bd = min_image(q)
        assert np.array_equal(np.sort(bd)[:10], d[j])
        assert abs(float(nd[j]) - float(bd.min())) <= 1e-5 * float(bd.min()) + 1e-7
        assert set(wi[off[j]:off[j + 1]].tolist()) == set(np.nonzero(bd <= r)[0].tolist())
