"""Multi-GPU as independent replicas: one process per GPU, each running its
own fit jobs (scenes are independent, so the data path has no collective).

The process group is used only for the job split, the barrier around the
timed region and the max-over-ranks time -- ``nccl`` on GPUs, ``gloo`` in
the CPU tests.  Every rank calls the collectives below in the same order.
"""
import datetime
import os

import torch
import torch.distributed as dist


def world():
    return int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0"))


def init(backend="nccl", timeout_s=120):
    """Join the process group described by the torchrun environment (a short
    timeout, so that ranks waiting for a dead peer end with an error)."""
    n, _ = world()
    if n > 1 and not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return world()


def shard(n_items, rank, world_size):
    """Round-robin split of item indices 0..n-1."""
    return list(range(rank, n_items, world_size))


def shard_by_cost(costs, rank, world_size):
    """Longest-processing-time-first split: items sorted by decreasing cost
    (ties by index) go to the least-loaded rank (ties by rank).  Deterministic,
    so every rank computes the same assignment without communication."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world_size
    owner = [0] * len(costs)
    for i in order:
        r = min(range(world_size), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += costs[i]
    return [i for i in range(len(costs)) if owner[i] == rank]


def _reduce(x, op):
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(x):
    return _reduce(x, dist.ReduceOp.MAX)


def sum_over_ranks(x):
    return _reduce(x, dist.ReduceOp.SUM)


def barrier():
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        if dist.get_backend() == "nccl":
            dist.barrier(device_ids=[torch.cuda.current_device()])
        else:
            dist.barrier()


def finish():
    if dist.is_available() and dist.is_initialized():
        dist.destroy_process_group()
