"""Replicas across GPUs: one process per GPU, each running its own scene (or
batch, or trajectory), with no data-path collective. The single-scene
pipeline does not shard (a slab decomposition with halo exchange is the
next step of the multi-GPU row); what crosses ranks is only the timing and
the aggregate:

* every rank times its own steps on its own stream;
* the job's time is the maximum over ranks (all_reduce MAX);
* the job's throughput is the units all ranks processed divided by that time.

torch.distributed is the plumbing: NCCL between GPUs, gloo on CPU (tests).
"""
from __future__ import annotations

import os


def world():
    """(rank, world size, local rank) from the launcher's environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def _dist():
    import torch.distributed as dist
    return dist if dist.is_available() and dist.is_initialized() else None


def _device():
    import torch
    dist = _dist()
    if dist is not None and dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def barrier():
    dist = _dist()
    if dist is not None and dist.get_world_size() > 1:
        dist.barrier()


def max_over_ranks(*values: float) -> list:
    """Each value's maximum over all ranks (one all_reduce)."""
    import torch
    dist = _dist()
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=_device())
    if dist is not None and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.cpu()]


def sum_over_ranks(*values: float) -> list:
    import torch
    dist = _dist()
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=_device())
    if dist is not None and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return [float(x) for x in t.cpu()]


def job_throughput(local_units: float, local_ms: float) -> tuple:
    """(units of all ranks per second over the slowest rank's time, that time in ms)."""
    units = sum_over_ranks(local_units)[0]
    ms = max_over_ranks(local_ms)[0]
    return units / (ms / 1e3), ms
