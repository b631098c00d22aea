"""Chamfer/ICP-style neighbour loss on the GPU, with its adjoint.

    loss, ctx = chamfer_forward(target, src, k=8, sigma=0.01)   # nearest_n + loss
    g_src, g_tgt = chamfer_backward(ctx)                         # dL/dsrc, dL/dtgt

``target`` is an ImmutableKdTree (or GpuTree) built with new_from_slice on the
target points (so items are target rows) or a Forest of such trees for a batch
of cloud pairs (then ``tree_of`` names each source's pair).  The neighbour
indices are those of the forward pass; ``recompute=True`` in the backward
recomputes them with the same deterministic nearest_n instead of keeping them.
``ChamferLoss`` wraps both as a torch.autograd.Function.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional

from . import _capi as C


@dataclass
class ChamferContext:
    target: object
    src: object
    tgt_points: object
    k: int
    sigma: float
    tree_of: Optional[object]
    tgt_base: Optional[object]
    dists: object
    items: object
    counts: object


def _vp(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _knn(target, src, k, tree_of):
    from . import Forest, SquaredEuclidean
    if isinstance(target, Forest):
        b = target.query(src, tree_of)
    else:
        b = target.query(src)
    return b.with_spatial_order().nearest_n(SquaredEuclidean, k).execute_gpu()


def chamfer_forward(target, src, tgt_points, k, sigma, tree_of=None, tgt_base=None):
    """Loss (0-d CUDA tensor) and the context for the backward pass."""
    import torch
    if src.dtype != torch.float32 or src.shape[1] != 3:
        raise TypeError("Chamfer takes float32 [n, 3] CUDA tensors")
    r = _knn(target, src, k, tree_of)
    loss = torch.empty((), dtype=torch.float32, device=src.device)
    st = ctypes.c_void_p(torch.cuda.current_stream(src.device).cuda_stream)
    C.check(C.lib().kgpu_chamfer_loss(_vp(r.distances), _vp(r.counts), src.shape[0], k,
                                      float(sigma), None, _vp(loss), st))
    ctx = ChamferContext(target, src, tgt_points, k, sigma, tree_of, tgt_base, r.distances,
                         r.items, r.counts)
    return loss, ctx


def chamfer_backward(ctx: ChamferContext, grad_scale: float = 1.0, recompute: bool = False):
    import torch
    items, counts = ctx.items, ctx.counts
    if recompute:
        r = _knn(ctx.target, ctx.src, ctx.k, ctx.tree_of)
        items, counts = r.items, r.counts
    g_src = torch.empty_like(ctx.src)
    g_tgt = torch.empty_like(ctx.tgt_points)
    st = ctypes.c_void_p(torch.cuda.current_stream(ctx.src.device).cuda_stream)
    C.check(C.lib().kgpu_chamfer_backward(
        _vp(ctx.src), ctx.src.shape[0], _vp(ctx.tgt_points), ctx.tgt_points.shape[0], _vp(items),
        _vp(counts), ctx.k, _vp(ctx.tree_of), _vp(ctx.tgt_base), float(ctx.sigma),
        float(grad_scale), _vp(g_src), _vp(g_tgt), st))
    return g_src, g_tgt


def chamfer_step_sharded(target, src_shard, tgt_points, k, sigma, tree_of=None, tgt_base=None,
                         recompute=False):
    """One Chamfer forward + backward with the source points sharded over the
    ranks of the process group (each rank holds every target tree and its own
    slice of sources).  The loss and the target gradient are sums over all
    sources, so their per-rank partials are combined with
    ``multi.fixed_order_sum`` (gathered, added in rank order): the same bits on
    every rank and every run.  The source gradient is per source and stays on
    its rank.  Returns (loss, grad of this rank's sources, grad of targets)."""
    from . import multi
    loss, ctx = chamfer_forward(target, src_shard, tgt_points, k, sigma, tree_of, tgt_base)
    g_src, g_tgt = chamfer_backward(ctx, recompute=recompute)
    return multi.fixed_order_sum(loss), g_src, multi.fixed_order_sum(g_tgt)


def _autograd_function():
    import torch

    class ChamferLoss(torch.autograd.Function):
        """loss = ChamferLoss.apply(src, tgt_points, target_tree, k, sigma)"""

        @staticmethod
        def forward(fctx, src, tgt_points, target, k, sigma):
            loss, c = chamfer_forward(target, src.detach().contiguous(),
                                      tgt_points.detach().contiguous(), k, sigma)
            fctx.c = c
            return loss

        @staticmethod
        def backward(fctx, grad_out):
            g_src, g_tgt = chamfer_backward(fctx.c, float(grad_out.item()))
            return g_src, g_tgt, None, None, None

    return ChamferLoss


def __getattr__(name):
    if name == "ChamferLoss":
        return _autograd_function()
    raise AttributeError(name)
