"""Multi-GPU plumbing: the solve is data parallel at structure granularity.

Every (structure, direction) solve is independent (LMB3d/lbm3d-perm.cpp:518-520),
so N GPUs split the structures, one process per GPU, with no collective in
the data path.  This module holds the partition rule and the two scalar
collectives the benchmark needs (a barrier and a max over ranks of the
device time), over torch.distributed (NCCL on GPUs, gloo for CPU tests).
"""
from __future__ import annotations

import os


def shard_ids(ids, rank: int, world: int):
    """The reference driver's --shard I/N rule: sample_id % N == I
    (scripts/solve_permeability3d.py:185-193)."""
    return [i for i in ids if int(i) % world == rank]


def env_rank():
    """(rank, world, local_rank) from the torchrun environment (1 process: 0, 1, 0)."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def max_over_ranks(value: float, device=None) -> float:
    """Max of a scalar over all ranks (identity without a process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64,
                     device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_results(local: dict) -> dict:
    """Union of per-rank {sample_id: row} dicts on every rank."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return dict(local)
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, local)
    merged = {}
    for d in out:
        merged.update(d)
    return merged
