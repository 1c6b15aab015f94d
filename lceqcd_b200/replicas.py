"""Replica placement for multi-GPU runs.

The Monte Carlo path does not shard inside one lattice (every pass is a
stencil with a grid-wide dependency), so multi-GPU runs place independent
chains (or independent configurations for gauge fixing) on different GPUs,
one process per GPU, with no collective on the data path.  Chains of uneven
volume are balanced greedily by site count (largest first onto the least
loaded rank), which keeps the slowest rank within one chain of the mean.
"""
from __future__ import annotations


def assign_chains(volumes, world_size: int):
    """Return, for each rank, the list of chain indices it runs."""
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    load = [0] * world_size
    out = [[] for _ in range(world_size)]
    for i in sorted(range(len(volumes)), key=lambda k: (-volumes[k], k)):
        r = min(range(world_size), key=lambda q: (load[q], q))
        out[r].append(i)
        load[r] += volumes[i]
    for lst in out:
        lst.sort()
    return out


def rank_loads(volumes, world_size: int):
    return [sum(volumes[i] for i in idx) for idx in assign_chains(volumes, world_size)]


def max_over_ranks(value: float) -> float:
    """Max of a float over the default process group (timing is the max over
    ranks); identity without an initialised group."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
