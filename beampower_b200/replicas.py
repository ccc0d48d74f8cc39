"""Multi-GPU runs as independent replicas.

The beamforming hot path has no cross-GPU exchange in this package (sources
are independent and the benchmark is quoted on one GPU): N processes, one per
GPU, each run the whole workload.  What is shared is only the measurement: a barrier before
and after the timed region, the slowest rank's time (max over ranks), and the
whole-job rate = N x work / that time.  These helpers work with any
torch.distributed backend (NCCL on GPUs, gloo on CPU for tests).
"""
from __future__ import annotations

import os


def world():
    """(rank, world_size, local_rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def max_over_ranks(value: float, device=None) -> float:
    """The maximum of `value` over all ranks (identity without a process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64,
                     device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(device=None):
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        if device is not None and getattr(device, "type", "cpu") == "cuda":
            dist.barrier(device_ids=[device.index])
        else:
            dist.barrier()


def whole_job_rate(work_per_rank: float, elapsed_s: float, device=None):
    """(rate, slowest elapsed): every rank processed `work_per_rank` units in
    its own `elapsed_s`; the job rate counts all ranks' work over the slowest
    rank's time (weak scaling)."""
    import torch.distributed as dist
    n = dist.get_world_size() if dist.is_available() and dist.is_initialized() else 1
    slowest = max_over_ranks(elapsed_s, device)
    return n * work_per_rank / slowest, slowest
