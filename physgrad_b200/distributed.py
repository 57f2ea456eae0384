"""Multi-GPU host logic for the MPM step: one process per GPU.

A single scene's step does not shard (no domain decomposition on this path),
so N GPUs run either independent replicas of one workload (weak scaling) or
disjoint shards of a batch of scenes (no exchange between ranks: scenes are
independent).  The only collective is the reduction of the timing: the
whole-job time is the maximum of the ranks' device times.
"""
from __future__ import annotations

from typing import List, Sequence


def shard_scenes(counts: Sequence[int], world: int, rank: int) -> List[int]:
    """Scene indices of ``rank``: greedy longest-processing-time assignment by
    particle count (deterministic: ties broken by scene index, then rank)."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("need 0 <= rank < world")
    load = [0] * world
    owner = [0] * len(counts)
    for s in sorted(range(len(counts)), key=lambda i: (-int(counts[i]), i)):
        r = min(range(world), key=lambda k: (load[k], k))
        owner[s] = r
        load[r] += int(counts[s])
    return [s for s in range(len(counts)) if owner[s] == rank]


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of ``value`` over the default process group (identity without
    one).  Works with NCCL (pass the rank's CUDA device) and gloo (CPU)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
