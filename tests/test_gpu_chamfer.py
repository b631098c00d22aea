"""Chamfer forward + adjoint on the GPU against the FP64 CPU gradient and f64
central differences (h = 1e-6), neighbour sets fixed by the forward pass."""
import numpy as np
import pytest

import kiddo_b200 as kb
from kiddo_b200.chamfer import chamfer_backward, chamfer_forward
from oracle import chamfer_ref as ref

pytestmark = pytest.mark.gpu

SIGMA = 0.01


def cloud(rng, n, kind):
    """Noisy plane or sphere, N(0, 0.001) jitter, random orientation."""
    if kind == "plane":
        p = np.c_[rng.uniform(-0.05, 0.05, (n, 2)), np.zeros(n)]
    else:
        v = rng.normal(size=(n, 3))
        p = 0.05 * v / np.linalg.norm(v, axis=1, keepdims=True)
    q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
    return (p @ q + rng.normal(0, 0.001, (n, 3)) + 0.5).astype(np.float32)


@pytest.mark.parametrize("k", [1, 8])
@pytest.mark.parametrize("kind", ["plane", "sphere"])
def test_chamfer_gradient_vs_fp64(k, kind):
    import torch
    rng = np.random.default_rng(k * 7 + len(kind))
    src = cloud(rng, 10_000, kind)
    tgt = cloud(rng, 40_000, kind)
    tree = kb.ImmutableKdTree.new_from_slice(tgt)
    ds, dt = torch.from_numpy(src).cuda(), torch.from_numpy(tgt).cuda()
    loss, ctx = chamfer_forward(tree, ds, dt, k, SIGMA)
    g_src, g_tgt = chamfer_backward(ctx)
    items = ctx.items.cpu().numpy().view(np.uint32)
    counts = ctx.counts.cpu().numpy()
    l64 = ref.loss(src, tgt, items, counts, k, SIGMA)
    assert abs(float(loss) - l64) <= 1e-5 * abs(l64)
    r_src, r_tgt = ref.gradient(src, tgt, items, counts, k, SIGMA)
    gs, gt = g_src.cpu().numpy(), g_tgt.cpu().numpy()
    # relative error of the gradient vectors (f32 engine vs FP64 oracle)
    e_src = np.linalg.norm(gs - r_src) / np.linalg.norm(r_src)
    e_tgt = np.linalg.norm(gt - r_tgt) / np.linalg.norm(r_tgt)
    print(f"chamfer k={k} {kind}: loss rel err {abs(float(loss) - l64) / abs(l64):.2e}, "
          f"grad rel err src {e_src:.2e} tgt {e_tgt:.2e}")
    assert e_src <= 1e-5 and e_tgt <= 1e-5
    # f64 central differences on 1,000 sampled coordinates away from ties
    picks = rng.choice(len(src), 500, replace=False)
    for i in picks[:500]:
        a = int(rng.integers(0, 3))
        fd = ref.central_difference(src, tgt, items, counts, k, SIGMA, "src", i, a)
        assert abs(fd - r_src[i, a]) <= 1e-6 * max(1.0, abs(r_src[i, a])) + 1e-7
        # per coordinate: relative to max(|fd|, 5% of the largest component),
        # since f32 rounding of tiny components is absolute, not relative
        assert abs(gs[i, a] - fd) <= 1e-5 * max(abs(fd), np.abs(r_src).max() * 0.05)
    used = np.unique(items[:, :1][counts > 0])
    for m in rng.choice(used, 500, replace=len(used) < 500):
        a = int(rng.integers(0, 3))
        fd = ref.central_difference(src, tgt, items, counts, k, SIGMA, "tgt", m, a)
        assert abs(gt[m, a] - fd) <= 1e-5 * max(abs(fd), np.abs(r_tgt).max() * 0.05)


def test_chamfer_backward_is_deterministic_and_recompute_matches():
    import torch
    rng = np.random.default_rng(5)
    src, tgt = cloud(rng, 20_000, "sphere"), cloud(rng, 80_000, "sphere")
    tree = kb.ImmutableKdTree.new_from_slice(tgt)
    ds, dt = torch.from_numpy(src).cuda(), torch.from_numpy(tgt).cuda()
    _, ctx = chamfer_forward(tree, ds, dt, 8, SIGMA)
    a = chamfer_backward(ctx)
    b = chamfer_backward(ctx)
    c = chamfer_backward(ctx, recompute=True)
    for x, y in ((a, b), (a, c)):
        assert torch.equal(x[0], y[0]) and torch.equal(x[1], y[1])


def test_batched_cloud_pairs_match_single_pairs():
    import torch
    rng = np.random.default_rng(6)
    pairs = [(cloud(rng, n, kind), cloud(rng, 4 * n, kind))
             for n, kind in ((3000, "plane"), (5000, "sphere"), (2000, "sphere"))]
    trees = [kb.ImmutableKdTree.new_from_slice(t) for _, t in pairs]
    forest = kb.Forest(trees)
    src = np.concatenate([s for s, _ in pairs])
    tgt = np.concatenate([t for _, t in pairs])
    tree_of = np.concatenate([np.full(len(s), p, np.int32) for p, (s, _) in enumerate(pairs)])
    base = np.cumsum([0] + [len(t) for _, t in pairs[:-1]]).astype(np.uint64)
    ds, dt = torch.from_numpy(src).cuda(), torch.from_numpy(tgt).cuda()
    loss, ctx = chamfer_forward(forest, ds, dt, 8, SIGMA, torch.from_numpy(tree_of).cuda(),
                                torch.from_numpy(base.astype(np.int64)).cuda())
    gs, gt = chamfer_backward(ctx)
    off_s = 0
    for p, (s, t) in enumerate(pairs):
        l1, c1 = chamfer_forward(trees[p], torch.from_numpy(s).cuda(), torch.from_numpy(t).cuda(),
                                 8, SIGMA)
        g1s, g1t = chamfer_backward(c1)
        assert torch.equal(gs[off_s:off_s + len(s)], g1s)
        o = int(base[p])
        assert torch.equal(gt[o:o + len(t)], g1t)
        off_s += len(s)


def test_autograd_function():
    import torch
    from kiddo_b200.chamfer import ChamferLoss
    rng = np.random.default_rng(7)
    src, tgt = cloud(rng, 4000, "plane"), cloud(rng, 16000, "plane")
    tree = kb.ImmutableKdTree.new_from_slice(tgt)
    ds = torch.from_numpy(src).cuda().requires_grad_(True)
    dt = torch.from_numpy(tgt).cuda().requires_grad_(True)
    (2.0 * ChamferLoss.apply(ds, dt, tree, 8, SIGMA)).backward()
    _, ctx = chamfer_forward(tree, ds.detach(), dt.detach(), 8, SIGMA)
    gs, gt = chamfer_backward(ctx, 2.0)
    assert torch.equal(ds.grad, gs) and torch.equal(dt.grad, gt)
