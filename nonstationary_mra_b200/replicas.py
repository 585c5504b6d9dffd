"""Replica bookkeeping for `bench.py --gpus N` (one process per GPU, each
rank evaluating its own copy of the workload; no data-path collective).

Every rank times its own steps on its device; the job's time is the maximum
over ranks and the job's throughput counts the steps of all ranks."""
from __future__ import annotations

from typing import Sequence


def max_over_ranks(values: Sequence[float], device: str = "cpu") -> list:
    """Element-wise maximum of `values` across the ranks of the default process
    group (identity when torch.distributed is not initialised)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def job_throughput(steps_per_rank: int, world: int, ms_max: float) -> float:
    """Steps per second of the whole job: all ranks' steps over the slowest rank's time."""
    return world * steps_per_rank / (ms_max * 1e-3)
