"""Multi-GPU by replicas: the path shards by domain, never inside one.

Every configuration fits one B200, so N GPUs run N independent sets of
domains with no data-path collective: one process per GPU
(torch.distributed, NCCL on GPUs, gloo for CPU tests), a barrier around the
timed region and a MAX of the per-rank times.  Batched and served domains are
routed to ranks by longest-processing-time-first on their cell-steps.
"""
from __future__ import annotations

import os


def rank_env():
    """(rank, world_size, local_rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def assign(costs, world: int):
    """Greedy LPT: returns owner[i] in [0, world) for each cost, so the
    largest load is within 4/3 of optimal; deterministic (ties by index)."""
    owner = [0] * len(costs)
    load = [0.0] * world
    for i in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        r = min(range(world), key=lambda q: (load[q], q))
        owner[i] = r
        load[r] += costs[i]
    return owner


def my_share(costs, world: int, rank: int):
    owner = assign(costs, world)
    return [i for i, r in enumerate(owner) if r == rank]


def max_over_ranks(x: float, device=None) -> float:
    """MAX of a per-rank scalar over the default process group (identity
    when no group is initialised)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()


def aggregate_rate(cells_per_rank: float, steps: int, world: int, max_seconds: float) -> float:
    """Whole-job GCell-updates/s: all ranks' updates over the slowest rank."""
    return cells_per_rank * steps * world / max_seconds / 1e9
