"""Case sharding across GPUs: one process per GPU, independent cases, no data-path collective.

Two ways to hand cases to ranks. A batch workload (the 512-case sweep) is weakly scaled: rank r
solves its own full batch, drawn from the same distribution with seed base + r, so the work per
GPU is fixed as GPUs are added. A stream of requests is split: case i goes to rank
i mod world_size. The only collectives are the ones that combine measurements: the sum of
converged cases, the max over ranks of the timed duration, and the gathered per-case latencies.
They run on any torch.distributed backend (NCCL with CUDA tensors on GPUs, gloo with CPU
tensors in the tests).
"""
from __future__ import annotations

from typing import Iterable, List


def stream_index(rank: int, world_size: int, k: int) -> int:
    """Global index of this rank's k-th case."""
    if not 0 <= rank < world_size:
        raise ValueError(f"rank {rank} outside world of {world_size}")
    return rank + world_size * k


def batch_seed(rank: int, world_size: int, base: int) -> int:
    """Seed of rank `rank`'s own batch under weak scaling (rank 0 keeps the base seed)."""
    if not 0 <= rank < world_size:
        raise ValueError(f"rank {rank} outside world of {world_size}")
    return base + rank


def shard(rank: int, world_size: int, n_total: int) -> List[int]:
    """The indices of the first n_total stream cases that belong to this rank."""
    return list(range(rank, n_total, world_size))


def _device(dist):
    import torch
    return torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")


def reduce_sum(x: float) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device(dist))
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def reduce_max(x: float) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device(dist))
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather(values: Iterable) -> list:
    import torch.distributed as dist
    vals = list(values)
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return vals
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, vals)
    return [v for part in out for v in part]
