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
