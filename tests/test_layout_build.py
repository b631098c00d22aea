"""The product's host construction (kgpu_layout_build) writes exactly the
bytes of the oracle's restatement of the reference construction."""
import numpy as np
import pytest

import kiddo_b200 as kb
import oracle


def same_layout(P, items=None):
    t = kb.ImmutableKdTree.new_from_slice(P) if items is None else \
        kb.ImmutableKdTree.new_from_entries(items, P)
    o = oracle.OracleTree.build(P, items).layout()
    assert t.max_stem_level() == o.max_stem_level
    assert t.max_leaf_len() == o.max_leaf_len
    assert t.size() == o.size
    assert np.array_equal(t.stems().view(np.uint8), o.stems.view(np.uint8))
    assert np.array_equal(t.leaf_extents(), o.extents)
    assert np.array_equal(t.leaf_bytes(), o.leaf_bytes)
    return t, o


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("dims", [1, 2, 3, 4])
@pytest.mark.parametrize("n", [0, 1, 5, 32, 33, 64, 65, 100, 1000, 100_000])
def test_uniform_layouts(dtype, dims, n):
    P = np.random.default_rng(n * 7 + dims).random((n, dims)).astype(dtype)
    same_layout(P)


def test_config1_shape():
    """100,000 f64 points -> stems_depth 12, 4,096 leaves, 8,192 stems (construction.rs:423-469)."""
    P = np.random.default_rng(0).random((100_000, 3))
    t, _ = same_layout(P)
    assert t.leaf_count() == 4096 and t.max_stem_level() == 11 and t.stems().size == 8192


@pytest.mark.parametrize("case", ["all_same", "repeated", "quantized", "axis_degenerate", "grid"])
def test_adversarial_layouts(case):
    """Adversarial layouts of tests/kd_tree_fuzz_v6.rs:3240-4117."""
    rng = np.random.default_rng(1)
    if case == "all_same":
        P = np.full((1000, 3), 0.5)
    elif case == "repeated":
        P = np.repeat(rng.random((50, 3)), 20, axis=0)
    elif case == "quantized":
        P = np.round(rng.random((20000, 3)) * 8) / 8
    elif case == "axis_degenerate":
        P = rng.random((20000, 3))
        P[:, 1] = 0.25
    else:
        g = np.linspace(0, 1, 30)
        P = np.stack(np.meshgrid(g, g, g), -1).reshape(-1, 3)
    same_layout(P)


def test_explicit_items():
    rng = np.random.default_rng(2)
    P = rng.random((5000, 3)).astype(np.float32)
    items = rng.permutation(5000).astype(np.uint32) * 3 + 7
    same_layout(P, items)


@pytest.mark.parametrize("bh", [3, 4])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("n", [0, 1, 33, 64, 65, 1000, 5000, 100_000])
def test_donnelly_layouts(bh, dtype, n):
    """Donnelly<bh> stems (stem_strategy/donnelly/core.rs, construction.rs:431-469):
    the product builder writes the oracle's bytes, padding levels included."""
    P = np.random.default_rng(n * 3 + bh).random((n, 3)).astype(dtype)
    t = kb.ImmutableKdTree.new_from_slice(P, block_height=bh)
    o = oracle.OracleTree.build(P, block_height=bh).layout()
    assert t.block_height() == bh and o.block_height == bh
    assert t.max_stem_level() == o.max_stem_level
    assert t.max_leaf_len() == o.max_leaf_len
    assert np.array_equal(t.stems().view(np.uint8), o.stems.view(np.uint8))
    assert np.array_equal(t.leaf_extents(), o.extents)
    assert np.array_equal(t.leaf_bytes(), o.leaf_bytes)
    if o.max_stem_level >= 0:
        assert (o.max_stem_level + 1) % bh == 0


def test_donnelly_rejects_other_block_heights():
    P = np.random.default_rng(0).random((100, 3))
    for bh in (1, 2, 5):
        with pytest.raises(Exception):
            kb.ImmutableKdTree.new_from_slice(P, block_height=bh)
