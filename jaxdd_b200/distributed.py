"""Several GPUs, one process each: the devices split into contiguous shards, each rank solving
its own with no collective on the data path, the curves gathered afterwards.

jaxdd splits a batch across accelerators the same way (`devices`, batch.py:1050-1101: a
shard of devices per accelerator, no communication during the solve, the results gathered).
Here each rank is a process with its own GPU (`torch.distributed`, NCCL between GPUs, gloo on
the CPU); `solve_batch` returns every rank the whole batch's curves in the caller's order.
"""

from __future__ import annotations

import numpy as np

from .batch import prepare
from .batch import solve_batch as _solve_batch


def shard(n: int, rank: int, world: int) -> slice:
    """The devices of `rank`: contiguous, the first `n % world` ranks one more."""
    if not 0 <= rank < world:
        raise ValueError(f"rank {rank} of {world}")
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return slice(start, start + base + (1 if rank < extra else 0))


def _group_info(group):
    import torch.distributed as dist
    return dist.get_rank(group), dist.get_world_size(group)


def solve_batch(devices, voltages, group=None, solve=None, **kwargs):
    """`jaxdd_b200.solve_batch` over the process group: each rank solves its shard of `devices`
    (built `Device`s, the same list on every rank) and every rank gets `(J, converged,
    iterations)` of all of them, in the order of `devices`. `solve(batch, voltages, **kwargs)`
    replaces the GPU solve of one shard (the default is `jaxdd_b200.solve_batch`)."""
    import torch.distributed as dist
    rank, world = _group_info(group)
    devices = list(devices)
    part = devices[shard(len(devices), rank, world)]
    nv = len(np.atleast_1d(voltages))
    if part:
        J, ok, its = (solve or _solve_batch)(prepare(part), voltages, **kwargs)
    else:
        J, ok, its = np.zeros((0, nv)), np.zeros((0, nv), bool), np.zeros((0, nv), int)
    pieces = [None] * world
    dist.all_gather_object(pieces, (rank, np.asarray(J), np.asarray(ok), np.asarray(its)),
                           group=group)
    pieces.sort(key=lambda p: p[0])
    return (np.concatenate([p[1] for p in pieces]), np.concatenate([p[2] for p in pieces]),
            np.concatenate([p[3] for p in pieces]))


def max_over_ranks(value: float, group=None, device=None) -> float:
    """The largest `value` of all ranks (the time a step took on the slowest GPU)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
