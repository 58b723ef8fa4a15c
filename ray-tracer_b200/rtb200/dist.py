"""Multi-GPU plumbing for the hot path: one process per GPU, no data-path collective.

The path shards by independent units: a batch of scenes is split into per-rank scene lists
(balanced by triangle count), each rank builds and renders its own, and the only collectives
are the timing reduction (max over ranks) and, where a caller wants every image on one rank,
a gather. Works with any torch.distributed backend (nccl on GPUs, gloo in the CPU tests).
"""
from __future__ import annotations


def shard_scenes(weights, rank: int, world: int) -> list[int]:
    """Scene indices for `rank`: longest-processing-time assignment of the scenes (by weight,
    e.g. triangle count; ties by index) to the least-loaded rank, so every rank gets a
    deterministic, disjoint share and the shares cover all scenes."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    order = sorted(range(len(weights)), key=lambda i: (-float(weights[i]), i))
    load = [0.0] * world
    owner = [0] * len(weights)
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += float(weights[i])
    return [i for i in range(len(weights)) if owner[i] == rank]


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """The maximum of `value` over all ranks (the whole job's time); identity without dist."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_to_rank0(obj, dist=None):
    """Every rank's `obj` on rank 0 (a list in rank order), None elsewhere."""
    if dist is None:
        return [obj]
    out = [None] * dist.get_world_size() if dist.get_rank() == 0 else None
    dist.gather_object(obj, out, dst=0)
    return out
