"""Replicas across GPUs: one process per GPU, each running an independent
simulation (its own screens, seeded by rank); no collective on the data path.
The only collectives are for timing: a barrier around the timed region and
the maximum of the ranks' times, so that the job's throughput is the units
of all ranks over the slowest rank's time.

The frame of a WFS does not exchange data with any other (the reference runs
whole WFS per GPU with replicated screens, cuda/sim/cudata.cu:404-470), so
the path shards as independent replicas.  NCCL carries the timing
collectives on GPUs; gloo carries them on the CPU (tests).
"""
from __future__ import annotations

import datetime
import os
from typing import Optional, Sequence, Tuple


def init(backend: Optional[str] = None, timeout_s: float = 300.0) -> Tuple[int, int, int]:
    """(world size, rank, local rank) from the torchrun environment; joins the
    process group when there is more than one rank (nccl by default)."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import torch.distributed as dist
        if not dist.is_initialized():
            dist.init_process_group(backend or "nccl", timeout=datetime.timedelta(seconds=timeout_s))
    return ws, rank, local


def _tensor(x: float, device):
    import torch
    return torch.tensor([x], dtype=torch.float64, device=device if device is not None else "cpu")


def max_over_ranks(x: float, ws: int, device=None) -> float:
    """The largest x over all ranks (every rank gets it)."""
    if ws == 1:
        return x
    import torch.distributed as dist
    t = _tensor(x, device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, ws: int, device=None) -> float:
    if ws == 1:
        return x
    import torch.distributed as dist
    t = _tensor(x, device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(ws: int, device=None):
    """All ranks reach this point (and, on a GPU, their queued work is done)."""
    if ws == 1:
        return
    import torch
    import torch.distributed as dist
    if device is not None and getattr(device, "type", "cpu") == "cuda":
        dist.barrier(device_ids=[device.index])
        torch.cuda.synchronize(device)
    else:
        dist.barrier()


def job_value(units_per_step: float, steps: int, ws: int, max_seconds: float) -> float:
    """Throughput of the whole job: every rank's units over the slowest rank's time."""
    return units_per_step * steps * ws / max_seconds


def shard(items: Sequence, rank: int, ws: int) -> list:
    """The items a rank takes when a list of independent units is split
    across replicas (round robin)."""
    return [x for i, x in enumerate(items) if i % ws == rank]


def finish(ws: int):
    if ws > 1:
        import torch.distributed as dist
        if dist.is_initialized():
            dist.destroy_process_group()
