"""The multi-GPU plumbing on CPU: two gloo ranks shard a batch by contiguous
ranges, each solves its share (the CPU checker stands in for a GPU), and the
reassembled result equals the single-process solve; timings reduce by max."""
import os

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import load_pkg

D = load_pkg("distributed")


def test_shard_range_covers_batch():
    for batch in (0, 1, 7, 64, 1001):
        for world in (1, 2, 3, 8):
            spans = [D.shard_range(batch, world, r) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == batch
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        D.shard_range(10, 2, 2)


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle.oracle import Oracle
        O = Oracle("port")
        rng = np.random.default_rng(0)
        batch, n = 37, 9
        A = rng.standard_normal((batch, n, n)) + n * np.eye(n)
        B = rng.standard_normal((batch, n, 2))
        s, e = D.shard_range(batch, world, rank)
        LU, piv, X, info = O.gesv(A[s:e], B[s:e], "scalar")
        Xall = D.gather_shards(torch.from_numpy(X), batch, world).numpy()
        pall = D.gather_shards(torch.from_numpy(piv), batch, world).numpy()
        mx = D.max_over_ranks(10.0 + rank)
        if rank == 0:
            LU0, piv0, X0, info0 = O.gesv(A, B, "scalar")
            q.put((np.array_equal(Xall.view(np.uint64), X0.view(np.uint64)), np.array_equal(pall, piv0), mx))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_reassemble():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    same_x, same_piv, mx = q.get(timeout=10)
    assert same_x and same_piv and mx == 11.0
