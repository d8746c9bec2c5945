"""Host-side plumbing for runs with one process per GPU (torchrun).

Batched QAOA / VQE instances are independent units: rank r of N takes units
r, r + N, r + 2N, ... of the same seeded list, with no collective on the data
path.  The only collectives are a barrier around timed regions and a MAX of
the per-rank device time, so a whole-job rate is units / max time.
"""
from __future__ import annotations

import datetime
import os


def world():
    """(world size, rank, local rank) from the torchrun environment (1, 0, 0 alone)."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard(units, rank: int, world_size: int):
    """This rank's units: every world_size-th, starting at rank."""
    if world_size < 1 or not 0 <= rank < world_size:
        raise ValueError(f"rank {rank} outside world of {world_size}")
    return units[rank::world_size]


def init(backend: str, timeout_s: float = 120.0):
    import torch.distributed as tdist
    tdist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return tdist


def _device():
    import torch
    import torch.distributed as tdist
    if tdist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def max_over_ranks(x: float) -> float:
    """MAX of a per-rank scalar over the process group (identity when not distributed)."""
    import torch
    import torch.distributed as tdist
    if not (tdist.is_available() and tdist.is_initialized()) or tdist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
    return float(t.item())


def barrier():
    import torch.distributed as tdist
    if tdist.is_available() and tdist.is_initialized() and tdist.get_world_size() > 1:
        tdist.barrier()


def whole_job_rate(units_total: int, per_rank_ms: float) -> float:
    """Units per second of the whole job: all units / the slowest rank's time."""
    return units_total / (max_over_ranks(per_rank_ms) / 1e3)
