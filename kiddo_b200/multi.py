"""Multi-GPU plumbing: one process per GPU.

Queries are independent (the reference parallelises them with a rayon par_iter over
`.execute()`, benches/query.rs:36-52), so a batch shards with no data-path
collective:

* one tree: every rank holds a replica and answers a contiguous query range
  (``shard_range``);
* many trees: every tree has one owner rank (``partition_trees``, balanced by
  points x queries) that holds it and answers its queries;
* sums that span ranks (a Chamfer loss, the target-point gradient when sources
  are sharded) are combined by ``fixed_order_sum``: gathered, then added in
  rank order, so every rank gets the same bits on every run.

The other collectives are the timing barrier, the max-over-ranks reduction of
elapsed times and optional result gathering on rank 0.
"""
from __future__ import annotations

import datetime
import os


def init_process_group(backend: str, timeout_s: float = 120.0):
    import torch.distributed as dist
    if not dist.is_initialized():
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=timeout_s))


def world():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


def shard_range(n: int, rank: int, world_size: int):
    """Contiguous [begin, end) slice of n queries for `rank`; sizes differ by <= 1."""
    base, extra = divmod(n, world_size)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def barrier():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.barrier()


def max_over_ranks(value: float) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    dev = torch.device("cuda", torch.cuda.current_device()) \
        if dist.get_backend() == "nccl" else torch.device("cpu")
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_to_rank0(arr):
    """Concatenate per-rank numpy arrays on rank 0 (in rank order)."""
    import numpy as np
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return arr
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, arr)
    return np.concatenate(out) if dist.get_rank() == 0 else None


def partition_trees(weights, world_size: int):
    """Owner rank of each tree: longest-first greedy on `weights` (for
    example points x queries of each tree), each tree to the least-loaded rank,
    ties to the lower tree index and the lower rank.  Every rank computes the
    same map from the same weights."""
    n = len(weights)
    order = sorted(range(n), key=lambda i: (-float(weights[i]), i))
    load = [0.0] * world_size
    owner = [0] * n
    for i in order:
        r = min(range(world_size), key=lambda j: (load[j], j))
        owner[i] = r
        load[r] += float(weights[i])
    return owner


def fixed_order_sum(t):
    """Elementwise sum of tensor `t` over the ranks, added in rank order
    0, 1, ..., N-1 on every rank (all-gather, then a fixed sequence of adds),
    so the result does not depend on the collective's reduction order."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return t.clone()
    parts = [t.new_empty(t.shape) for _ in range(dist.get_world_size())]
    dist.all_gather(parts, t.contiguous())
    acc = parts[0].clone()
    for p in parts[1:]:
        acc += p
    return acc
