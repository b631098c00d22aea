"""Trees uploaded straight from rkyv archives (kgpu_tree_create_from_archive)
answer like the oracle over the same layout, and read back the archived
bytes.  The archives come from the oracle's restatement of kiddo's
`rkyv::to_bytes` (oracle/rkyv_archive.py); parity against an archive written
by the Rust crate itself is unpinned (no Rust toolchain here)."""
import numpy as np
import pytest

import kiddo_b200 as kb
import oracle
from helpers import assert_same_csr, assert_same_fixed, gaussian_mixture
from kiddo_b200 import _capi as C
from oracle import rkyv_archive as ra

pytestmark = pytest.mark.gpu
SE = kb.SquaredEuclidean


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("dims", [2, 3])
@pytest.mark.parametrize("bh", [0, 4])
@pytest.mark.parametrize("width", [4, 8])
def test_archive_upload_matches_the_oracle(dtype, dims, bh, width, tmp_path):
    rng = np.random.default_rng(dims * 7 + bh + width)
    P = np.concatenate([rng.random((30_000, dims)),
                        np.floor(rng.random((5_000, dims)) * 8) / 8]).astype(dtype)
    Q = np.concatenate([rng.random((3_000, dims)), P[:300]]).astype(dtype)
    o = oracle.OracleTree.build(P, block_height=bh)
    lay = o.layout()
    path = tmp_path / "tree.rkyv"
    path.write_bytes(ra.write_layout(lay, width))
    g = kb.GpuTree.from_archive(str(path), dtype, dims, block_height=bh, pointer_width=width)
    stems, lb, ex = g.read_layout()
    assert np.array_equal(stems, lay.stems) and np.array_equal(lb, lay.leaf_bytes)
    assert np.array_equal(ex, lay.extents)
    r = g.query(Q).nearest_one(SE).execute_gpu()
    od, oi = o.nearest_one(Q)
    assert_same_fixed(r.distances, r.items, np.ones(len(Q)), od, oi, np.ones(len(Q)), "nn1")
    r = g.query(Q).nearest_n(SE, 16).execute_gpu()
    assert_same_fixed(r.distances, r.items, r.counts, *o.nearest_n(Q, 16), "knn16")
    r = g.query(Q).within(SE, 1e-3).execute_gpu()
    assert_same_csr((r.offsets, r.distances, r.items), o.within(Q, 1e-3), "within")


def test_archive_upload_from_bytes_and_the_c2_shape():
    rng = np.random.default_rng(3)
    P = gaussian_mixture(500_000, 256, 0.005, 0.2, rng)
    Q = gaussian_mixture(40_000, 256, 0.005, 0.2, rng)
    o = oracle.OracleTree.build(P)
    b = ra.write_layout(o.layout(), 4, "pristine")
    g = kb.GpuTree.from_archive(b, np.float32, 3)
    r = g.query(Q).nearest_n(SE, 16).execute_gpu()
    assert_same_fixed(r.distances, r.items, r.counts, *o.nearest_n(Q, 16), "knn16")
    r = g.query(Q).nearest_one(SE).approx().execute_gpu()
    od, oi = o.approx_nearest_one(Q)
    assert_same_fixed(r.distances, r.items, np.ones(len(Q)), od, oi, np.ones(len(Q)), "approx")


@pytest.mark.parametrize("width", [4, 8])
def test_archive_of_a_mutable_tree(width):
    """A MutableKdTree archive (hard buckets, Mapped resolution with its
    leaf_idx_map) uploads in place and answers like the oracle."""
    rng = np.random.default_rng(width)
    P = rng.random((30_000, 3))
    Q = rng.random((2_000, 3))
    o = oracle.OracleTree.build_mutable(P)
    b = ra.write_layout(o.layout(), width)
    info = kb.GpuTree.inspect_archive(b, np.float64, 3, pointer_width=width)
    assert info["resolution"] == C.RES_MAPPED and info["map_len"] == o.leaf_map()[0].size
    g = kb.GpuTree.from_archive(b, np.float64, 3, pointer_width=width)
    r = g.query(Q).nearest_n(SE, 10).execute_gpu()
    assert_same_fixed(r.distances, r.items, r.counts, *o.nearest_n(Q, 10), "knn10")
    r = g.query(Q).within(SE, 5e-4).execute_gpu()
    assert_same_csr((r.offsets, r.distances, r.items), o.within(Q, 5e-4), "within")
