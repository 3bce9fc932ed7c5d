"""Multi-GPU bookkeeping for replica (weak-scaling) runs.

The receive path has no exchange step: every rank beamforms its own frames on its own GPU and nothing
crosses between GPUs on the data path. Timing follows the job, not a rank: each rank times its region
on its device (CUDA events), the job's time is the maximum over ranks, and the job's rate counts the
units of all ranks. The only collective is this reduction of one number per rank (NCCL on GPUs, gloo
in the CPU tests).
"""
from __future__ import annotations

from typing import Tuple

import torch
import torch.distributed as dist


def world_size() -> int:
    return dist.get_world_size() if dist.is_available() and dist.is_initialized() else 1


def max_over_ranks(local_ms: float, device="cpu") -> float:
    """The maximum of `local_ms` over all ranks of the default process group (local_ms when alone)."""
    t = torch.tensor([float(local_ms)], dtype=torch.float64, device=device)
    if world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank_step: float, steps: int, local_ms: float, device="cpu") -> Tuple[float, float]:
    """(units per second of the whole job, job time in ms): all ranks' units over the slowest rank's
    time for `steps` steps."""
    ms = max_over_ranks(local_ms, device)
    return units_per_rank_step * steps * world_size() / (ms / 1e3), ms
