"""Multi-GPU tracing by replication: one process per GPU, electrons sharded
across ranks, no communication while tracing.

Every electron is independent (traceon/tracing.py:210-245 traces them one by
one), so N GPUs trace N disjoint shards of the beam with their own copy of
the field; the only collectives are the final gather of the per-electron
results and the max-over-ranks of the timings.  Works with any
torch.distributed backend (NCCL on GPUs, gloo in the CPU tests).
"""
from __future__ import annotations

import numpy as np


def shard(n: int, rank: int, world: int) -> slice:
    """Contiguous block of [0, n) owned by `rank` (sizes differ by at most 1)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError('bad rank / world size')
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return slice(lo, lo + base + (1 if rank < extra else 0))


def gather_shards(local, n: int, group=None):
    """All-gather per-electron rows (first dimension = this rank's shard of
    n) into the full (n, ...) array on every rank.  `local` is a torch
    tensor; shards of unequal size are padded for the collective."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    sizes = [shard(n, r, world).stop - shard(n, r, world).start for r in range(world)]
    width = max(sizes)
    pad = torch.zeros((width,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[:local.shape[0]] = local
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    return torch.cat([p[:s] for p, s in zip(parts, sizes)], dim=0)


def max_over_ranks(value: float, device=None, group=None) -> float:
    """The largest value over all ranks (job time = slowest rank)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def trace_sharded(trace_fn, start, qm, group=None):
    """Runs trace_fn(start_shard, qm_shard) -> (n_shard, k) tensor on this
    rank's shard of the electrons and gathers the full (n, k) result."""
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    n = start.shape[0]
    sl = shard(n, rank, world)
    local = trace_fn(start[sl].contiguous(), qm[sl].contiguous())
    return gather_shards(local, n, group)
