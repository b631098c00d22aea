"""The exactness claim behind the periodic fast path, checked on the CPU with
the oracle alone: for every row whose plain list keeps clear of the box's
faces (the test k_periodic_needed applies on the device, restated here in
the tree's own arithmetic), the reference's periodic walk
(kd_tree/query/periodic.rs:455-619, as the oracle restates it) returns the
plain walk's row, bit for bit: same items, same distances, same order."""
import numpy as np
import pytest

import oracle

METRICS = {"sqeuclidean": lambda x: x * x, "manhattan": np.abs, "chebyshev": np.abs,
           "minkowski3": lambda x: x * (x * x)}


def _clear_rows(Q, d, c, k, radius, box, metric, dtype):
    """k_periodic_needed's test: every axis's face, less 8 ulps of the box,
    is positive, and its metric term, shrunk by 1e-5, is above the row's
    bound (its k-th distance, or the radius while the list is not full)."""
    ulps = dtype(8.0 / (8388608.0 if dtype == np.float32 else 4503599627370496.0))
    shrink = dtype(1.0 - 1e-5)
    bound = np.where(c >= k, d[:, k - 1], dtype(radius)).astype(dtype)
    clear = np.ones(len(Q), dtype=bool)
    with np.errstate(invalid="ignore"):
        for a in range(Q.shape[1]):
            q = Q[:, a]
            up = (box[a] - q).astype(dtype)
            face = (np.minimum(q, up) - (box[a] * ulps).astype(dtype)).astype(dtype)
            term = METRICS[metric](face).astype(dtype)
            clear &= (face > 0) & ((term * shrink).astype(dtype) > bound)
    return clear


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("metric", sorted(METRICS))
def test_clear_rows_of_the_plain_walk_equal_the_periodic_walk(dtype, metric):
    rng = np.random.default_rng(len(metric) + (dtype == np.float64))
    n = 30_000
    c = rng.random((64, 3))
    P = np.concatenate([(c[rng.integers(0, 64, n // 2)] + rng.normal(0, 0.01, (n // 2, 3))) % 1.0,
                        rng.random((n - n // 2, 3))]).astype(dtype)
    P[P >= 1.0] = 0.0
    Q = np.concatenate([rng.random((4000, 3)), rng.random((500, 3)) * 0.02,
                        1.0 - rng.random((500, 3)) * 0.02]).astype(dtype)
    box = np.ones(3, dtype=dtype)
    o = oracle.OracleTree.build(P)
    for k, radius in ((16, np.inf), (32, np.inf), (32, 0.004 if metric != "minkowski3" else 1e-7)):
        pd, pi, pc = o.nearest_n(Q, k, radius=radius, metric=metric)
        wd, wi, wc = o.periodic_nearest_n(Q, box, k, radius=radius, metric=metric)
        clear = _clear_rows(Q, pd, pc, k, radius, box, metric, dtype)
        assert clear.sum() > 500                  # many rows take the plain walk
        assert (~clear).sum() > 0                 # and some do not
        assert np.array_equal(pc[clear], wc[clear])
        assert np.array_equal(pd[clear], wd[clear])
        assert np.array_equal(pi[clear], wi[clear])
        if radius == np.inf:
            # the rows the test keeps for the periodic walk include rows the
            # plain walk gets wrong (so the test is not vacuous)
            assert not np.array_equal(pi[~clear], wi[~clear])
