"""Multi-GPU plumbing: one process per GPU, each holding a replica of the tree.

Queries are independent (the reference parallelises them with a rayon par_iter over
`.execute()`, benches/query.rs:36-52), so a batch shards by contiguous query
ranges with no data-path collective.  The only collectives are the timing
barrier and the max-over-ranks reduction of elapsed times, and optional result
gathering for callers that want every rank's answers on rank 0.
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
