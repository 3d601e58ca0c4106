"""Work partition across ranks, on CPU with gloo (world size 2)."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from flow_anizotropy_b200.parallel import gather_results, max_over_ranks, shard_ids


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    ids = list(range(11))
    mine = shard_ids(ids, rank, world)
    local = {i: i * i for i in mine}             # stand-in for a per-sample result row
    merged = gather_results(local)
    worst = max_over_ranks(10.0 + rank)
    q.put((rank, mine, sorted(merged.items()), worst))
    dist.barrier()
    dist.destroy_process_group()


def test_shard_rule():
    ids = list(range(10))
    parts = [shard_ids(ids, r, 3) for r in range(3)]
    assert sorted(sum(parts, [])) == ids
    assert all(i % 3 == r for r, p in enumerate(parts) for i in p)


def test_two_ranks_partition_and_max():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    mine0, mine1 = out[0][1], out[1][1]
    assert not set(mine0) & set(mine1) and sorted(mine0 + mine1) == list(range(11))
    assert out[0][2] == out[1][2] == [(i, i * i) for i in range(11)]
    assert out[0][3] == out[1][3] == 11.0
