"""One process per GPU: how independent work is split over ranks and how the
ranks' timings combine.

The nonbonded path has no exchange step between GPUs: every rank evaluates
whole systems of its own (its own replica of the box, seeded with seed +
rank, or its share of a batch of independent boxes), so the data path needs
no collective.  The only cross-rank traffic is bookkeeping: a barrier before
a timed region, the largest step time over ranks (the job is as slow as its
slowest rank) and the sum of the units (pairs) all ranks processed.  These
helpers take the tensor device from the caller, so they run on NCCL with
CUDA tensors on GPUs and on gloo with CPU tensors in tests.
"""
from __future__ import annotations


def rank_seed(seed: int, rank: int) -> int:
    """Seed of a rank's own replica of a generated system."""
    return int(seed) + int(rank)


def shard_sizes(sizes, world: int) -> list[list[int]]:
    """Split independent boxes of the given atom counts over `world` ranks so
    that the largest rank total is small: longest first, each to the rank
    with the fewest atoms so far (ties to the lowest rank).  Returns each
    rank's box indices in ascending order; every box goes to exactly one
    rank, and a rank may get none when there are fewer boxes than ranks."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i))
    load = [0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += int(sizes[i])
    return [sorted(o) for o in out]


def max_over_ranks(values, device="cpu") -> list[float]:
    """Element-wise maximum of per-rank values (all ranks get it)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def sum_over_ranks(values, device="cpu") -> list[float]:
    """Element-wise sum of per-rank values (all ranks get it)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return [float(v) for v in t.tolist()]


def job_rate(units: float, ms: float, device="cpu") -> tuple[float, float, float]:
    """(units of all ranks, slowest rank's ms, whole-job units per second)
    from this rank's units processed per step and its ms per step."""
    total = sum_over_ranks([units], device)[0]
    slow = max_over_ranks([ms], device)[0]
    return total, slow, total / (slow * 1e-3)
