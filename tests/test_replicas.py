"""Replica sharding across ranks (world size 2, gloo on CPU)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from mixedprecisionfaracoustic_b200.replicas import max_over_ranks, my_shots, shard


def test_shard_partition_balanced():
    costs = [7, 3, 9, 1, 4, 4, 8, 2, 6, 5]
    for w in (1, 2, 3, 4):
        parts = shard(costs, w)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs)
    with pytest.raises(ValueError):
        shard(costs, 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    costs = [5, 1, 9, 3, 3, 7, 2]
    mine = my_shots(costs, rank, world)
    t = max_over_ranks(float(10 * rank + sum(costs[i] for i in mine)))
    q.put((rank, mine, t))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_disjoint_cover_and_max():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, s0, t0), (r1, s1, t1) = res
    assert sorted(s0 + s1) == list(range(7)) and not set(s0) & set(s1)
    costs = [5, 1, 9, 3, 3, 7, 2]
    expect = max(0 + sum(costs[i] for i in s0), 10 + sum(costs[i] for i in s1))
    assert t0 == t1 == expect
