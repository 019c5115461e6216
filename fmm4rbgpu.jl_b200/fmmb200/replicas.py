"""Rank plumbing for replicated field evaluations (one beam per GPU rank).

The field evaluation of one beam runs on one GPU; ``bench.py --gpus N`` under
torchrun runs N independent beams (weak scaling) and reports the aggregate rate
over the slowest rank.  No collective touches the data path: only a barrier
around the timed region and a max-reduction of the per-rank times.
"""
from __future__ import annotations

import datetime
import os


def env_ranks():
    """(world, rank, local_rank) from the torchrun environment (1, 0, 0 by default)."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str, local_rank: int, timeout_s: int = 600):
    """Initialise the default process group when WORLD_SIZE > 1 (nccl binds the rank's GPU)."""
    import torch
    import torch.distributed as dist

    kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
    if backend == "nccl":
        torch.cuda.set_device(local_rank)
        kw["device_id"] = torch.device("cuda", local_rank)
    dist.init_process_group(backend, **kw)


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(world: int, value: float, device=None) -> float:
    """The maximum of a per-rank float over all ranks (the slowest rank's time)."""
    if world == 1:
        return float(value)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(world: int, units_per_rank: int, ms_max: float) -> float:
    """Whole-job units per second: every rank processed units_per_rank in ms_max (max over ranks)."""
    return world * units_per_rank / (ms_max * 1e-3)
