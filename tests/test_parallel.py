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


def _tensor_rows(ids):
    """Tensor rows of seeded structures: three solves each (the CPU oracle
    stands in for the device solver here, where no GPU is present), then the
    host tensor assembly of the drop-in."""
    from flow_anizotropy_b200 import structures as st
    from flow_anizotropy_b200 import tensor
    from oracle import oracle as O
    F = 1e-6
    mu = (1.0 / 3.0) * (1.0 - 0.5)
    prm = dict(eps=1e-6, lag=100, hold=2, min_steps=200, max_steps=1500, avg_steps=20)
    rows = {}
    for i in ids:
        s = st.sphere_packing((8, 10, 12), 2.5, 0.6, seed=100 + i, percolate=(True, True, True))
        runs = [O.solve3d(s, f, **prm) for f in ([F, 0, 0], [0, F, 0], [0, 0, F])]
        T = tensor.assemble3([r["q"] for r in runs], mu, F)
        rows[i] = (tuple(r["steps"] for r in runs), tuple(map(float, sum(T.K, []))))
    return rows


def _tensor_worker(rank, world, port, q):
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    mine = shard_ids(list(range(5)), rank, world)
    merged = gather_results(_tensor_rows(mine))
    q.put((rank, mine, sorted(merged.items())))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_shard_tensor_solves():
    """Two ranks split five structures by the reference driver's shard rule,
    each solves its own tensors with no collective in the data path, and the
    gathered rows equal a single process's rows exactly."""
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_tensor_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=300) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0][1] == [0, 2, 4] and out[1][1] == [1, 3]
    alone = sorted(_tensor_rows(range(5)).items())
    assert out[0][2] == out[1][2] == alone
