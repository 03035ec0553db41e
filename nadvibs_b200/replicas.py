"""Replica bookkeeping for multi-GPU runs of the Lanczos stage.

The stage does not shard (one system per GPU), so N GPUs run N independent replicas: one
process per GPU, each with its own handle.  The process group is used only to align the
timed regions (barrier) and to take the slowest rank's time (all-reduce MAX); the
aggregate rate is N * steps / max_time.  NCCL on GPUs, gloo on CPU (tests).
"""
from __future__ import annotations

import os
from datetime import timedelta

import torch
import torch.distributed as dist


def env() -> tuple[int, int, int]:
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str | None = None, timeout_s: int = 120) -> tuple[int, int, int]:
    rank, world, local = env()
    if world > 1 and not dist.is_initialized():
        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))
    return rank, world, local


def _device():
    if dist.is_initialized() and dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def barrier() -> None:
    if dist.is_initialized():
        dist.barrier()


def max_over_ranks(x: float) -> float:
    if not dist.is_initialized():
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(steps: int, seconds_local: float) -> float:
    """Whole-job steps/s: every rank ran `steps`, the job took the slowest rank's time."""
    world = dist.get_world_size() if dist.is_initialized() else 1
    return world * steps / max_over_ranks(seconds_local)


def shutdown() -> None:
    if dist.is_initialized():
        dist.destroy_process_group()
