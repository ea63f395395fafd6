"""One process per GPU: frames are independent, so N GPUs run N replicas.

Each reference frame (and each fusion volume) is a complete unit of work with
no exchange between units, so a batch of frames is sharded by index across
ranks and there is no data-path collective.  The only collectives are the
timing ones: a barrier around the timed region and a max over ranks of the
device-measured time.
"""
from __future__ import annotations

import os


def world():
    """(rank, world_size, local_rank) from the torchrun environment (1 process if unset)."""
    rank = int(os.environ.get("RANK", "0"))
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", str(rank)))
    return rank, ws, local


def shard(n_items: int, rank: int, world_size: int) -> range:
    """Contiguous block of item indices owned by `rank` (sizes differ by at most one)."""
    base, extra = divmod(n_items, world_size)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def init(backend: str):
    """Initialise torch.distributed when launched with more than one rank."""
    import datetime

    import torch.distributed as dist
    rank, ws, _ = world()
    if ws > 1 and not dist.is_initialized():
        dist.init_process_group(backend=backend, rank=rank, world_size=ws,
                                timeout=datetime.timedelta(seconds=120))
    return rank, ws


def max_over_ranks(value: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.barrier()


def finish():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.destroy_process_group()
