"""Process-group helpers for replica runs (one process per GPU; gloo on CPU in tests).

The DF path is single-GPU; with N processes every rank runs an independent
replica and the only collectives are a barrier around the timed region and a
max over ranks of the measured time.
"""

from __future__ import annotations

import torch
import torch.distributed as dist


def world() -> tuple[int, int]:
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


def _device_for_backend() -> torch.device:
    if dist.is_initialized() and dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def barrier() -> None:
    if dist.is_available() and dist.is_initialized():
        dist.barrier()


def max_over_ranks(x: float) -> float:
    """Maximum of a per-rank scalar (timing is reported as the slowest rank)."""
    r, n = world()
    if n == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device_for_backend())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
