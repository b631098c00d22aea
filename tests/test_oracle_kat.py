"""Pin the CPU oracle: the reference's literal known-answer tests and its own
brute-force parity rules (tests/kd_tree_fuzz_v6.rs:244-340, 682-734, 960-1029)."""
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


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("metric", ["sqeuclidean", "manhattan"])
@pytest.mark.parametrize("n", [1, 31, 33, 1000, 20000])
def test_oracle_vs_brute_force(dtype, metric, n):
    rng = np.random.default_rng(n)
    P = rng.random((n, 3)).astype(dtype)
    Q = rng.random((60, 3)).astype(dtype)
    t = oracle.OracleTree.build(P)
    d1, i1 = t.nearest_one(Q, metric=metric)
    k = 8
    dn, inn, cn = t.nearest_n(Q, k, metric=metric)
    r = np.asarray(0.02 if metric == "sqeuclidean" else 0.2, dtype=dtype)
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
