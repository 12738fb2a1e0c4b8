"""Replica layout: sharding arithmetic, and the end-of-run collectives over a
2-rank gloo process group on CPU (no GPU needed)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from nebula_b200 import replicas


def test_shard_covers_everything_once():
    for n in (0, 1, 7, 100, 1001):
        for world in (1, 2, 3, 8):
            parts = [replicas.shard(n, r, world) for r in range(world)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(parts, parts[1:]))
            sizes = [b - a for a, b in parts]
            assert max(sizes) - min(sizes) <= 1


def test_replica_seeds_distinct():
    seeds = {replicas.replica_seed(1234, r) for r in range(64)}
    assert len(seeds) == 64


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t = replicas.max_over_ranks(10.0 + rank, dist)
        a, b = replicas.sum_tallies([np.full((4, 4), rank + 1, np.uint32), np.arange(3.0) * rank], dist)
        out[rank] = (t, float(a.sum()), b.tolist())
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_collectives_over_gloo_two_ranks():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(100)
        assert p.exitcode == 0
    for r in range(2):
        t, s, b = out[r]
        assert t == 11.0
        assert s == 16 * 3
        assert b == [0.0, 1.0, 2.0]
