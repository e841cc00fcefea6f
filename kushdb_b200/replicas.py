"""Multi-GPU replicas: one process per GPU, each holding its own copy of the
tables and running the same queries; no collective is on the data path
(KushDB runs one query in one process; a query here fits one GPU).  The
process group only brackets timed regions and takes the slowest rank's
time, so whole-job throughput = work of all ranks / max time.

Works with NCCL on GPUs and with gloo on CPU (the multi-process tests)."""

from __future__ import annotations

import datetime
import os
from typing import Optional, Tuple


def rank_info() -> Tuple[int, int, int]:
    """(rank, world size, local rank) from the launcher's environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: int = 300):
    """The process group when more than one rank runs, else None."""
    _, world, _ = rank_info()
    if world <= 1:
        return None
    import torch.distributed as dist
    if not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def barrier(dist) -> None:
    if dist is not None:
        dist.barrier()


def max_over_ranks(value: float, dist, device: Optional[str] = None) -> float:
    """The largest `value` over all ranks (every rank gets it)."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: float, steps: int, world: int, max_ms: float) -> float:
    """Units per second of the whole job: every rank's units over the
    slowest rank's time."""
    return units_per_rank * steps * world / (max_ms / 1e3)


def share(n: int, rank: int, world: int) -> Tuple[int, int]:
    """[begin, end) of rank's contiguous share of n items (sizes differ by at
    most one)."""
    return n * rank // world, n * (rank + 1) // world


def finish(dist) -> None:
    if dist is not None and dist.is_initialized():
        dist.destroy_process_group()
