"""Multi-GPU plumbing: independent replicas.

Every programmable bootstrap is independent and the reference has no
collective, so N GPUs run N replicas: each process (one per GPU) holds its
own copy of the keys and bootstraps its own share of the ciphertexts.
torch.distributed is used only to split work, align the timed region and
take the maximum time over ranks; no ciphertext data crosses GPUs.
"""
from __future__ import annotations

import os
from dataclasses import dataclass


@dataclass(frozen=True)
class Rank:
    rank: int
    world: int
    local_rank: int

    @staticmethod
    def from_env() -> "Rank":
        return Rank(int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
                    int(os.environ.get("LOCAL_RANK", "0")))


def shard(batch: int, rank: int, world: int) -> range:
    """Contiguous share of `batch` ciphertexts for `rank`: shares differ by
    at most one and cover [0, batch) exactly once."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world {world}")
    base, extra = divmod(batch, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """The maximum of `value` over all ranks (the whole-job time of a
    replicated step); the value itself without a process group."""
    if dist is None or not dist.is_initialized():
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def total_over_ranks(value: float, dist=None, device=None) -> float:
    """The sum of `value` over all ranks (units processed by the job)."""
    if dist is None or not dist.is_initialized():
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
