"""Several GPUs as replicas: independent systems or solve requests are sharded over ranks (one
process per GPU), each rank solves its share with no collective on the data path, and only
timings and counts are combined (max / sum over ranks).

Every north-star system fits one B200, so nothing here splits a single system; a row-sharded
solve with halo exchanges is not built.  The process group is torch.distributed over NCCL on
GPUs (gloo on CPU hosts), rendezvous from the usual RANK / WORLD_SIZE / MASTER_ADDR /
MASTER_PORT environment (torchrun).
"""
from __future__ import annotations

import os
from datetime import timedelta


def env() -> tuple[int, int, int]:
    """(world size, rank, local rank) from the launcher's environment (1, 0, 0 without one)."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str | None = None, timeout_s: float = 120.0, device=None):
    """Joins the process group when WORLD_SIZE > 1 (a short timeout, so ranks that wait for a
    missing peer end with an error).  Returns (world size, rank, local rank)."""
    import torch
    import torch.distributed as dist
    ws, rank, local = env()
    if ws > 1 and not dist.is_initialized():
        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        kw = {"timeout": timedelta(seconds=timeout_s)}
        if backend == "nccl" and device is not None:
            kw["device_id"] = device
        dist.init_process_group(backend, **kw)
    return ws, rank, local


def _reduce(value: float, op) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(value: float) -> float:
    import torch.distributed as dist
    return _reduce(value, dist.ReduceOp.MAX)


def sum_over_ranks(value: float) -> float:
    import torch.distributed as dist
    return _reduce(value, dist.ReduceOp.SUM)


def barrier() -> None:
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()


def shard(sizes, world_size: int) -> list[list[int]]:
    """Assigns item indices to ranks, largest first to the least-loaded rank (longest-processing-
    time), so every rank gets about the same number of rows.  Deterministic; every index appears
    exactly once; within a rank the original order is kept."""
    loads = [0] * world_size
    owner = [0] * len(sizes)
    for i in sorted(range(len(sizes)), key=lambda k: (-sizes[k], k)):
        r = min(range(world_size), key=lambda q: (loads[q], q))
        owner[i] = r
        loads[r] += sizes[i]
    return [[i for i in range(len(sizes)) if owner[i] == r] for r in range(world_size)]


def my_share(items, sizes, rank: int, world_size: int) -> list:
    """The items this rank solves (see shard)."""
    return [items[i] for i in shard(list(sizes), world_size)[rank]]


def finish() -> None:
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.destroy_process_group()
