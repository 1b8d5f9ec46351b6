"""Multi-GPU runs of a path that does not shard: one independent replica per
rank (one process per GPU).  Only the plumbing lives here -- the barrier around
a timed region and the max over ranks of a per-rank time -- so the same code
runs with NCCL on GPUs and with gloo on CPU (tests)."""
from __future__ import annotations

import torch
import torch.distributed as dist


def world():
    if dist.is_available() and dist.is_initialized():
        return dist.get_world_size(), dist.get_rank()
    return 1, 0


def barrier():
    if world()[0] > 1:
        dist.barrier()


def max_over_ranks(value: float, device=None) -> float:
    """Max of a per-rank scalar over all ranks (every rank gets the result)."""
    if world()[0] == 1:
        return float(value)
    if device is None:
        device = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
