"""Multi-GPU replicas: one process per GPU, each running its own independent
circuit(s) on its own state (the path has no state exchange), combined as

    value = (units processed by all ranks) / (max over ranks of the device time)

The only collectives are a barrier around the timed region and one MAX
all-reduce of the elapsed time; they run over whatever process group is
initialised (NCCL on GPUs, gloo in the CPU tests).
"""
from __future__ import annotations

import datetime
import os


def world() -> tuple[int, int, int]:
    """(rank, local_rank, world_size) from the launcher's environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")),
            int(os.environ.get("WORLD_SIZE", "1")))


def init(backend: str, timeout_s: float = 300.0):
    """Initialise the default process group when WORLD_SIZE > 1 (env:// rendezvous)."""
    import torch.distributed as dist
    rank, _, size = world()
    if size > 1 and not dist.is_initialized():
        dist.init_process_group(backend, init_method="env://", rank=rank, world_size=size,
                                timeout=datetime.timedelta(seconds=timeout_s))
    return size


def barrier():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.barrier()


def max_over_ranks(x: float, device=None) -> float:
    """MAX of a per-rank float over all ranks (identity without a process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(units_per_rank: float, elapsed_s_local: float, device=None) -> tuple[float, float]:
    """(whole-job rate, max elapsed seconds): every rank processed units_per_rank."""
    import torch.distributed as dist
    size = dist.get_world_size() if (dist.is_available() and dist.is_initialized()) else 1
    t = max_over_ranks(elapsed_s_local, device)
    return units_per_rank * size / t, t


def shutdown():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.barrier()
        dist.destroy_process_group()
