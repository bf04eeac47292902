"""Multi-process plumbing: one process per GPU, torch.distributed for the
barrier and the max-over-ranks timing, and the sharding of independent work.

The single-grid MHD step does not shard without a halo exchange, so several
GPUs run replicas (one mesh per rank) or split an ensemble of independent
members; no collective sits on the data path.  Works with the "nccl" backend
on GPUs and "gloo" on CPU (the tests use gloo, world size 2).
"""
from __future__ import annotations

import datetime
import os

import torch
import torch.distributed as dist


def env():
    """(rank, world_size, local_rank) from the torchrun environment (defaults: 0, 1, 0)."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str | None = None, timeout_s: float = 300.0) -> bool:
    """Joins the process group when WORLD_SIZE > 1; returns True if it did."""
    rank, world, local = env()
    if world <= 1 or dist.is_initialized():
        return dist.is_initialized()
    if backend is None:
        backend = "nccl" if torch.cuda.is_available() else "gloo"
    kw = {}
    if backend == "nccl":
        kw["device_id"] = torch.device("cuda", local)
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
    return True


def _device():
    if dist.is_initialized() and dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def barrier() -> None:
    if dist.is_initialized():
        dist.barrier()


def max_over_ranks(x: float) -> float:
    """The maximum of x over all ranks (x itself on one rank)."""
    if not dist.is_initialized():
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float) -> float:
    if not dist.is_initialized():
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def shard(costs, rank: int, world: int) -> list[int]:
    """Indices of the items rank `rank` owns: greedy longest-first assignment of
    items with the given costs (e.g. cell counts) to `world` ranks, so the
    largest per-rank load is within one item of the balanced share.  The same
    on every rank (deterministic, ties broken by index)."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    owner = [0] * len(costs)
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += costs[i]
    return [i for i in range(len(costs)) if owner[i] == rank]


def destroy() -> None:
    if dist.is_initialized():
        dist.destroy_process_group()
