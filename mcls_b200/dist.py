"""Process-group plumbing for multi-GPU runs (one process per GPU).

torch.distributed carries the collectives: NCCL between GPUs, gloo between
CPU processes (the tests).  Reductions go through tensors on the device the
backend expects.
"""
from __future__ import annotations

import datetime
import os


def init(backend: str | None = None, timeout_s: int = 300):
    """(world, rank, local_rank, group module or None) from the torchrun
    environment; one process per GPU with NCCL unless `backend` says gloo."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world <= 1:
        return world, rank, local, None
    import torch
    import torch.distributed as dist

    backend = backend or "nccl"
    if backend == "nccl":
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=timeout_s),
                                device_id=torch.device("cuda", local))
    else:
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return world, rank, local, dist


def _device(pg):
    return "cuda" if pg.get_backend() == "nccl" else "cpu"


def barrier(pg):
    if pg is None:
        return
    pg.barrier()
    if _device(pg) == "cuda":
        import torch

        torch.cuda.synchronize()


def _reduce(pg, v, op):
    if pg is None:
        return v
    import torch

    t = torch.tensor([float(v)], dtype=torch.float64, device=_device(pg))
    pg.all_reduce(t, op=op)
    return float(t.item())


def allmax(pg, v):
    """Largest v over the ranks (device timings: the job time is the slowest rank's)."""
    return v if pg is None else _reduce(pg, v, pg.ReduceOp.MAX)


def allsum(pg, v):
    return v if pg is None else _reduce(pg, v, pg.ReduceOp.SUM)
