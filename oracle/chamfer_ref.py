"""FP64 CPU reference for the Chamfer neighbour loss and its gradient.

TEST INFRASTRUCTURE (checker only).  The reference library has no Chamfer
loss; this restates the loss the engine defines (kiddo_b200/csrc/kgpu_chamfer.cu)
in float64 with the neighbour sets held fixed:
    L = sum_i sum_j phi(d_ij),  d_ij = |t_m - s_i|^2,  phi(d) = d exp(-d / (2 sigma^2)).
"""
from __future__ import annotations

import numpy as np


def _pairs(items, counts, k, tree_of=None, tgt_base=None):
    n = counts.shape[0]
    rows = np.repeat(np.arange(n), k)
    ranks = np.tile(np.arange(k), n)
    valid = ranks < np.repeat(counts.astype(np.int64), k)
    m = items.reshape(-1).astype(np.int64)
    if tree_of is not None:
        m = m + tgt_base[tree_of[rows]].astype(np.int64)
    return rows[valid], m[valid]


def loss(src, tgt, items, counts, k, sigma, tree_of=None, tgt_base=None):
    i, m = _pairs(items, counts, k, tree_of, tgt_base)
    s = src.astype(np.float64)[i]
    t = tgt.astype(np.float64)[m]
    d = ((t - s) ** 2).sum(1)
    return float((d * np.exp(-d / (2 * sigma * sigma))).sum())


def gradient(src, tgt, items, counts, k, sigma, tree_of=None, tgt_base=None):
    i, m = _pairs(items, counts, k, tree_of, tgt_base)
    s = src.astype(np.float64)[i]
    t = tgt.astype(np.float64)[m]
    diff = s - t
    d = (diff ** 2).sum(1)
    a = 1.0 / (2 * sigma * sigma)
    w = (np.exp(-d * a) * (1 - d * a) * 2.0)[:, None] * diff
    g_src = np.zeros((src.shape[0], 3))
    g_tgt = np.zeros((tgt.shape[0], 3))
    np.add.at(g_src, i, w)
    np.add.at(g_tgt, m, -w)
    return g_src, g_tgt


def central_difference(src, tgt, items, counts, k, sigma, which, index, axis, h=1e-6,
                       tree_of=None, tgt_base=None):
    """d L / d (which[index, axis]) by f64 central differences, neighbours fixed."""
    s = src.astype(np.float64).copy()
    t = tgt.astype(np.float64).copy()
    arr = s if which == "src" else t
    x0 = arr[index, axis]
    arr[index, axis] = x0 + h
    lp = loss(s, t, items, counts, k, sigma, tree_of, tgt_base)
    arr[index, axis] = x0 - h
    lm = loss(s, t, items, counts, k, sigma, tree_of, tgt_base)
    return (lp - lm) / (2 * h)
