"""Clip sharding and the multi-process reductions, on CPU with the gloo backend
(world size 2): balanced disjoint shards, gradient all-reduce, kernel-set
broadcast."""
import os
import socket

import pytest

import shard


def test_partition_balanced_and_disjoint():
    sizes = [512 * 512] * 128 + [1024 * 1024] * 192 + [2048 * 2048] * 64
    for world in (1, 2, 4, 8):
        parts = shard.partition(sizes, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(sizes)))
        loads = [sum(sizes[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(sizes)


def test_partition_rejects_bad_world():
    with pytest.raises(ValueError):
        shard.partition([1, 2], 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path[:0] = [os.path.join(os.path.dirname(here), "k-litho_b200")]
    import datetime

    import torch
    import torch.distributed as dist

    import shard as sh
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    sizes = [100, 300, 200, 400, 50]
    mine = sh.shard_for_rank(sizes, rank, world)
    # each rank's "source gradient" is the sum of its clip indices + 1
    g = torch.zeros(9)
    for i in mine:
        g += float(i + 1)
    sh.allreduce_source_gradient(g)
    k = torch.arange(6, dtype=torch.float32) if rank == 0 else torch.zeros(6)
    sh.broadcast_kernels(k, src=0)
    q.put((rank, mine, g.tolist(), k.tolist()))
    dist.barrier()
    dist.destroy_process_group()


def test_gloo_two_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res.sort()
    shards = [r[1] for r in res]
    assert sorted(shards[0] + shards[1]) == [0, 1, 2, 3, 4]
    total = sum(i + 1 for i in range(5))
    for _, _, g, k in res:
        assert all(abs(v - total) < 1e-6 for v in g)
        assert k == [0.0, 1.0, 2.0, 3.0, 4.0, 5.0]
