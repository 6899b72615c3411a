"""Multi-GPU plumbing: replicas only.

The sampling path shards by independent unit (chain, disorder sample,
serving request) with no exchange on the data path, so N GPUs run N
independent replicas, one process per GPU (``torch.distributed``: NCCL
between GPUs, gloo on CPU for tests).  The only collectives are a barrier
around timed regions, a max over ranks of the elapsed time, and one gather
of per-rank summaries at the end.  critmc's counterpart is its process pool
over independent tasks (src/critmc/runner.py:154-223).
"""

from __future__ import annotations

import os
from datetime import timedelta

import torch
import torch.distributed as dist


def rank_env() -> tuple[int, int, int]:
    """(rank, world size, local rank) from the launcher's environment (1 process if unset)."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str, device=None, timeout_s: float = 120.0) -> None:
    """Join the process group when there is more than one rank (short timeout: a lost rank errors out)."""
    _, world, _ = rank_env()
    if world > 1 and not dist.is_initialized():
        kw = {"device_id": device} if backend == "nccl" and device is not None else {}
        dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s), **kw)


def shard(units, rank: int, world: int) -> list:
    """The units of one rank: every world-th unit from ``rank`` (each unit on exactly one rank)."""
    return list(units)[rank::world]


def barrier(device=None) -> None:
    if device is not None and torch.device(device).type == "cuda":
        torch.cuda.synchronize(device)
    if dist.is_initialized():
        dist.barrier()


def max_over_ranks(x: float, device="cpu") -> float:
    """Largest value over ranks (device times: the job ends when the slowest rank ends)."""
    if not dist.is_initialized():
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, device="cpu") -> float:
    if not dist.is_initialized():
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def gather_to_root(obj) -> list | None:
    """Every rank's object on rank 0 (None elsewhere); the one gather at the end of a run."""
    if not dist.is_initialized():
        return [obj]
    out = [None] * dist.get_world_size() if dist.get_rank() == 0 else None
    dist.gather_object(obj, out, dst=0)
    return out


def finish() -> None:
    if dist.is_initialized():
        dist.destroy_process_group()
