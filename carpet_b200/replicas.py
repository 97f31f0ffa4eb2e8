"""One process per GPU running independent replicas of the workload.

The transfer path has no exchange step on one GPU (every grid function of a
hierarchy is resident on its own device), so ``bench.py --gpus N`` runs N
independent hierarchies, one per rank, with no data-path collective.  This
module holds the rank plumbing: process-group set-up with a short timeout,
the barrier around the timed region, the maximum of the per-rank times, and
the whole-job throughput computed from it.
"""
from __future__ import annotations

import datetime
import os


def world():
    """(world size, rank) from the launcher's environment"""
    return int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0"))


def init(backend: str = "nccl", timeout_s: int = 120):
    import torch.distributed as dist
    if not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))


def active() -> bool:
    import torch.distributed as dist
    return dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1


def barrier():
    import torch.distributed as dist
    if active():
        dist.barrier()


def max_over_ranks(x: float, device="cuda") -> float:
    """the largest value of x over all ranks (the timed region of the slowest)"""
    if not active():
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(units_per_rank: float, world_size: int, max_ms: float) -> float:
    """units per second of the whole job: every rank's units over the slowest
    rank's time"""
    return units_per_rank * world_size / (max_ms * 1e-3)


def finish():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.destroy_process_group()
