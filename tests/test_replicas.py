"""Multi-rank host logic on CPU: world_size 2 over gloo (127.0.0.1)."""

from __future__ import annotations

import os
import socket

import pytest

from lithofem_b200 import replicas


def test_shard_covers_every_item_once():
    for n in (1, 5, 16):
        for world in (1, 2, 3, 8):
            got = sorted(i for r in range(world) for i in replicas.shard(n, r, world))
            assert got == list(range(n))
    with pytest.raises(ValueError):
        replicas.shard(4, 2, 2)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        mine = replicas.shard(16, rank, world)
        units = sum(100 + i for i in mine)
        ms = 1.0 + rank                      # rank 1 is the slower one
        total = replicas.sum_over_ranks(units, dist)
        slowest = replicas.max_over_ranks(ms, dist)
        import torch
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        q.put((rank, total, slowest, gathered))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_units_and_time():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want_total = float(sum(100 + i for i in range(16)))
    for rank, total, slowest, gathered in res:
        assert total == want_total and slowest == 2.0
        assert sorted(i for part in gathered for i in part) == list(range(16))
        assert set(gathered[0]).isdisjoint(gathered[1])
