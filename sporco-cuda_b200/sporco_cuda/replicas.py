"""Independent replicas of a solve on several GPUs, one process per GPU.

The ADMM iteration has no data-path collective: an image (or a batch of
images) is solved entirely on one GPU, so N GPUs run N independent solves
(weak scaling).  The ranks only agree on measurements: the job's time is the
slowest rank's time, counts are summed.  These helpers work with any
``torch.distributed`` backend (NCCL between GPUs, gloo on the host), and
with no process group at all (one process).
"""

from __future__ import annotations

import torch

__all__ = ["world", "max_over_ranks", "sum_over_ranks", "job_rate", "shard"]


def _dist():
    import torch.distributed as dist
    return dist if dist.is_available() and dist.is_initialized() else None


def world():
    """(rank, world size) of the current process group, (0, 1) without one."""
    d = _dist()
    return (d.get_rank(), d.get_world_size()) if d else (0, 1)


def _reduce(x, op, device):
    d = _dist()
    if d is None:
        return float(x)
    if device is None:
        device = torch.device("cuda", torch.cuda.current_device()) \
            if d.get_backend() == "nccl" else torch.device("cpu")
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    d.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(x, device=None):
    """The largest value of x over the ranks (every rank gets it)."""
    import torch.distributed as dist
    return _reduce(x, dist.ReduceOp.MAX, device)


def sum_over_ranks(x, device=None):
    """The sum of x over the ranks (every rank gets it)."""
    import torch.distributed as dist
    return _reduce(x, dist.ReduceOp.SUM, device)


def job_rate(units, ms, device=None):
    """Whole-job throughput: the units all ranks processed divided by the
    slowest rank's time (ms), in units per second."""
    total = sum_over_ranks(units, device)
    slowest = max_over_ranks(ms, device)
    return total / (slowest / 1e3)


def shard(items, rank=None, world_size=None):
    """The items rank `rank` of `world_size` solves: a round-robin split that
    gives every item to exactly one rank."""
    if rank is None or world_size is None:
        rank, world_size = world()
    return list(items)[rank::world_size]
