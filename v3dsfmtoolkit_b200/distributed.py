"""Multi-process plumbing for running independent bundle adjustments on several GPUs.

One process per GPU (torchrun).  A single bundle adjustment does not shard in this library:
N GPUs run N independent problems (replicas) or split a batch of independent problems
(triplets, submodels) into contiguous shards.  There is no collective on the data path; the
only communication is the barrier around the timed region and the reduction of the timing
(max over ranks) and of the work counts (sum over ranks).
"""
from __future__ import annotations

import datetime
import os


def env_rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def shard_range(n_items: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous shard [lo, hi) of n_items for rank; sizes differ by at most one."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("bad rank / world size")
    base, extra = divmod(n_items, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def init(backend: str, timeout_s: float = 300.0):
    """Initialises the process group from the torchrun environment (MASTER_ADDR/PORT, RANK,
    WORLD_SIZE); returns torch.distributed, or None for a single process."""
    rank, world, _ = env_rank()
    if world <= 1:
        return None
    import torch.distributed as dist
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def reduce_scalar(dist, value: float, op: str, device=None) -> float:
    """max / sum of a scalar over all ranks (identity without a process group)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def gather_shards(dist, local: list) -> list:
    """The per-rank result lists of a sharded job, concatenated in rank order (every rank gets the
    whole list; with contiguous shards from shard_range this is the job's order).  Host objects
    over the process group (gloo or NCCL); the identity without a process group."""
    if dist is None:
        return list(local)
    parts = [None] * dist.get_world_size()
    dist.all_gather_object(parts, list(local))
    return [x for part in parts for x in part]
