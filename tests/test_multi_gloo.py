"""Host logic of the multi-GPU path (replicas + query shards) on CPU ranks
with the gloo backend, world size 2."""
import os

import numpy as np
import pytest
import torch.multiprocessing as mp

from kiddo_b200.multi import shard_range


def test_shard_range_covers_exactly():
    for n in (0, 1, 7, 1000, 16_000_001):
        for w in (1, 2, 3, 8):
            spans = [shard_range(n, r, w) for r in range(w)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            for (a, b), (c, d) in zip(spans, spans[1:]):
                assert b == c
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    import torch.distributed as dist
    from kiddo_b200 import multi
    multi.init_process_group("gloo", timeout_s=60)
    # each rank answers its shard with the oracle; rank 0 gathers in rank order
    import oracle
    rng = np.random.default_rng(0)
    P = rng.random((5000, 3))
    Q = rng.random((1001, 3))
    a, b = shard_range(len(Q), rank, world)
    t = oracle.OracleTree.build(P)
    d, i = t.nearest_one(Q[a:b])
    got = multi.gather_to_rank0(i)
    mx = multi.max_over_ranks(float(rank + 1))
    if rank == 0:
        full_d, full_i = t.nearest_one(Q)
        out.put((bool(np.array_equal(got, full_i)), mx))
    multi.barrier()
    dist.destroy_process_group()


def test_two_rank_gloo_shards_match_single_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 1000)
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    ok, mx = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
    assert ok and mx == 2.0
    assert all(p.exitcode == 0 for p in procs)


def test_partition_trees_is_balanced_and_deterministic():
    from kiddo_b200.multi import partition_trees
    rng = np.random.default_rng(4)
    w = (np.exp(rng.uniform(np.log(1e4), np.log(4e6), 256)) *
         rng.dirichlet(np.full(256, 0.5)) * 64e6)
    for ws in (1, 2, 4, 8):
        owner = partition_trees(w, ws)
        assert owner == partition_trees(list(w), ws)
        load = np.zeros(ws)
        for i, r in enumerate(owner):
            load[r] += w[i]
        # greedy longest-first: no rank exceeds the mean by more than the largest tree
        assert load.max() - load.sum() / ws <= w.max() + 1e-6


def _sum_worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    import torch
    import torch.distributed as dist
    from kiddo_b200 import multi
    multi.init_process_group("gloo", timeout_s=60)
    g = torch.Generator().manual_seed(100 + rank)
    part = torch.randn(10007, 3, generator=g, dtype=torch.float32)
    s1 = multi.fixed_order_sum(part)
    s2 = multi.fixed_order_sum(part)
    parts = [torch.randn(10007, 3, generator=torch.Generator().manual_seed(100 + r),
                         dtype=torch.float32) for r in range(world)]
    ref = parts[0].clone()
    for p in parts[1:]:
        ref += p
    out.put((rank, bool(torch.equal(s1, s2)), bool(torch.equal(s1, ref)),
             s1.view(torch.int32).sum().item()))
    multi.barrier()
    dist.destroy_process_group()


def test_fixed_order_sum_same_bits_on_every_rank():
    """The cross-rank sum is the rank-order sum on every rank (what the sharded
    Chamfer loss and target gradient use)."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29600 + (os.getpid() % 1000)
    procs = [ctx.Process(target=_sum_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=120)
    assert all(r[1] and r[2] for r in res)
    assert res[0][3] == res[1][3]
    assert all(p.exitcode == 0 for p in procs)
