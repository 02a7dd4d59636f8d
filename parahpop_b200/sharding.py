"""Object sharding for one process per GPU.

Objects are independent, so a batch shards into contiguous object ranges
with no data-path collective; ranks exchange only the final states (to
assemble results) and their timings (the job time is the maximum over ranks).
"""
from __future__ import annotations

import numpy as np


def shard_bounds(n: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous [lo, hi) range of rank `rank` out of `world` for n objects;
    sizes differ by at most one."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("bad rank / world")
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def gather_states(local_epochs, local_states, n: int, group=None):
    """Assemble every rank's (epochs, n_local x 6 states) into full arrays on
    every rank (torch.distributed all_gather of padded blocks)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    lo, hi = shard_bounds(n, rank, world)
    width = -(-n // world)
    block = torch.zeros(width, 7, dtype=torch.float64)
    block[: hi - lo, 0] = torch.as_tensor(np.asarray(local_epochs, dtype=np.float64))
    block[: hi - lo, 1:] = torch.as_tensor(np.asarray(local_states, dtype=np.float64).reshape(-1, 6))
    out = [torch.zeros_like(block) for _ in range(world)]
    dist.all_gather(out, block, group=group)
    epochs = np.zeros(n)
    states = np.zeros((n, 6))
    for r in range(world):
        a, b = shard_bounds(n, r, world)
        epochs[a:b] = out[r][: b - a, 0].numpy()
        states[a:b] = out[r][: b - a, 1:].numpy()
    return epochs, states


def max_over_ranks(value: float, group=None) -> float:
    """Maximum of a per-rank scalar (the job's device time)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
