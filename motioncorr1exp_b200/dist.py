"""Replica parallelism: one process per GPU, each aligning its own movies.

The drift-correction path has no exchange step (a movie fits one GPU), so
multi-GPU runs shard whole movies across ranks and combine only timing and
counts: ``shard`` assigns movie indices round-robin, ``max_over_ranks`` /
``sum_over_ranks`` reduce host scalars over the default process group (NCCL
on GPUs, gloo on CPU).  Nothing on the data path is communicated.
"""
from __future__ import annotations

import os


def world() -> tuple[int, int, int]:
    """(rank, world size, local rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard(n_items: int, rank: int, world_size: int) -> list[int]:
    """Movie indices this rank processes (round-robin, disjoint, covering)."""
    if world_size < 1 or not 0 <= rank < world_size:
        raise ValueError(f"bad rank {rank} of {world_size}")
    return list(range(rank, n_items, world_size))


def _reduce(value: float, op: str) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    backend = dist.get_backend()
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=getattr(dist.ReduceOp, op))
    return float(t.item())


def max_over_ranks(value: float) -> float:
    return _reduce(value, "MAX")


def sum_over_ranks(value: float) -> float:
    return _reduce(value, "SUM")
