"""Multi-GPU plumbing for independent stripes: one process per GPU, stripes
partitioned across ranks with no data-path collective (every stripe is
encoded or decoded entirely on its owner's GPU).  The only collectives are
host-side bookkeeping: the max of a per-rank time and the AND of per-rank
success flags.  Works with any torch.distributed backend (NCCL between GPUs,
gloo on CPU for tests)."""
from __future__ import annotations

import os
from typing import List, Sequence, Tuple


def world_info() -> Tuple[int, int, int]:
    """(world_size, rank, local_rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard_range(n: int, rank: int, world: int) -> Tuple[int, int]:
    """Contiguous block [lo, hi) of n units owned by `rank` (sizes differ by at most one)."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("rank out of range")
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def shard_by_bytes(sizes: Sequence[int], world: int) -> List[Tuple[int, int]]:
    """Split units with the given byte sizes into `world` contiguous ranges of
    about equal bytes (a unit is never split): range r starts at the first
    unit whose byte prefix reaches r/world of the total."""
    if world <= 0:
        raise ValueError("world must be positive")
    total = sum(sizes)
    bounds, prefix, r = [0], 0, 1
    for i, s in enumerate(sizes):
        while r < world and prefix * world >= total * r:
            bounds.append(i)
            r += 1
        prefix += s
    while r < world:
        bounds.append(len(sizes))
        r += 1
    bounds.append(len(sizes))
    return [(bounds[q], bounds[q + 1]) for q in range(world)]


def _device_for(dist):
    import torch

    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def max_over_ranks(value: float) -> float:
    """Max of a per-rank value (e.g. a step time) over all ranks."""
    import torch
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return value
    t = torch.tensor([value], dtype=torch.float64, device=_device_for(dist))
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def all_ranks_ok(ok: bool) -> bool:
    """True when every rank reports success."""
    import torch
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return ok
    t = torch.tensor([1 if ok else 0], dtype=torch.int32, device=_device_for(dist))
    dist.all_reduce(t, op=dist.ReduceOp.MIN)
    return bool(t.item())
