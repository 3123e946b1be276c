"""Independent replicas across ranks.

The hot path does not shard in this build: one grid lives on one GPU and N GPUs
run N independent solves (bench replicas, or the requests of the serving
queue).  No data-path collective exists; the only communication is the timing
reduction (max over ranks) and the work assignment below.
"""
from __future__ import annotations


def assign(items, rank: int, world: int):
    """Round-robin share of a request list for one rank."""
    return list(items)[rank::world]


def max_over_ranks(x: float, device=None) -> float:
    """The slowest rank's value (torch.distributed, any backend)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, device=None) -> float:
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
