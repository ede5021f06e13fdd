"""Process-group helpers of the multi-GPU runs (one process per GPU).

The stepper's work shards into independent fields (replicas, ensemble members), so the
only cross-rank traffic is a barrier and a few scalars: the max of the ranks' device
times and sums of counters.  Works with NCCL (CUDA tensors) and gloo (CPU tensors).
"""
from __future__ import annotations

import datetime
import os

import torch


def env_world():
    """(world_size, rank, local_rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend, timeout_s=300):
    import torch.distributed as dist
    if not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))


def _device():
    import torch.distributed as dist
    return torch.device("cuda") if dist.get_backend() == "nccl" else torch.device("cpu")


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def reduce_scalars(world, values, op="max"):
    """All-reduce a list of floats across ranks (max or sum)."""
    if world == 1:
        return [float(v) for v in values]
    import torch.distributed as dist
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return [float(v) for v in t.cpu().tolist()]


def shutdown(world):
    if world > 1:
        import torch.distributed as dist
        if dist.is_initialized():
            dist.destroy_process_group()
