"""Multi-process plumbing for the benchmark: one process per GPU, torch.distributed for the barrier
and the max-over-ranks timing only (the element path has no data exchange between ranks)."""
from __future__ import annotations

import datetime
import os


def world():
    return int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0"))


def init(backend="nccl", timeout_s=120):
    import torch.distributed as dist
    ws, rank, _ = world()
    if ws > 1 and not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return ws, rank


def barrier():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.barrier()


def max_over_ranks(x: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(units_per_rank: float, seconds_per_rank: float, device=None) -> tuple[float, float]:
    """Whole-job rate: units processed by all ranks / the slowest rank's time."""
    import torch.distributed as dist
    ws = dist.get_world_size() if (dist.is_available() and dist.is_initialized()) else 1
    t = max_over_ranks(seconds_per_rank, device)
    return ws * units_per_rank / t, t


def finalize():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.barrier()
        dist.destroy_process_group()
