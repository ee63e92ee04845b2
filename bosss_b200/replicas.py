"""Independent replicas, one process per GPU.

A solve of one system has no exchange step when every GPU holds its own system, so N GPUs run N independent
replicas (the batch of independent XDG problems splits the same way).  The only collectives are outside the data
path: a barrier around the timed region and a max over ranks of the measured times.  The reference distributes
one system over MPI ranks instead (BlockMsrMatrix.cs:226-260 row partitioning, halo exchange :3033-3070); that
partitioned form is not built here.
"""
from __future__ import annotations

import datetime
import os


def world() -> tuple[int, int, int]:
    """(world size, rank, local rank) from the torchrun environment; (1, 0, 0) without one."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: int = 600) -> tuple[int, int, int]:
    ws, rank, local = world()
    if ws > 1:
        import torch.distributed as dist
        if not dist.is_initialized():
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return ws, rank, local


def _device(backend_device):
    import torch
    import torch.distributed as dist
    if backend_device is not None:
        return backend_device
    return torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")


def max_over_ranks(v: float, ws: int, device=None) -> float:
    """Largest value over all ranks (every rank must call it, in the same order)."""
    if ws == 1:
        return float(v)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v)], dtype=torch.float64, device=_device(device))
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(v: float, ws: int, device=None) -> float:
    if ws == 1:
        return float(v)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v)], dtype=torch.float64, device=_device(device))
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(ws: int):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def shard(n_items: int, ws: int, rank: int) -> range:
    """Contiguous share of n_items for this rank (sizes differ by at most one)."""
    q, r = divmod(n_items, ws)
    lo = rank * q + min(rank, r)
    return range(lo, lo + q + (1 if rank < r else 0))


def aggregate(units: float, seconds: float, ws: int, device=None) -> dict:
    """Whole-job throughput of independent replicas: all ranks' units over the slowest rank's time."""
    total = sum_over_ranks(units, ws, device)
    t = max_over_ranks(seconds, ws, device)
    return {"units": total, "seconds": t, "per_s": total / t if t > 0 else None}


def finalize(ws: int):
    if ws > 1:
        import torch.distributed as dist
        if dist.is_initialized():
            dist.destroy_process_group()
