"""Replica parallelism: independent lattices, one process per GPU.

The flow step has no data exchange between independent relaxations, so the
multi-GPU form is a partition of lattices (or of a batch of instances) over ranks
with no collective on the data path.  The only collectives are host-side
bookkeeping: the max-over-ranks of a measured time and the gather of per-rank
results.  Works with any torch.distributed backend (NCCL on GPUs, gloo on CPU).
"""
from __future__ import annotations

import datetime
import os

import torch
import torch.distributed as dist


def env_rank():
    """(rank, world_size, local_rank) from the torchrun environment (defaults: single process)."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str, timeout_s: float = 300.0, device=None):
    """Initialise the default process group from the environment (idempotent)."""
    rank, world, _ = env_rank()
    if world > 1 and not dist.is_initialized():
        kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
        if device is not None and backend == "nccl":
            kw["device_id"] = device
        dist.init_process_group(backend, **kw)
    return rank, world


def shard(n_items: int, rank: int, world: int) -> range:
    """Contiguous block of items owned by `rank`; blocks differ in size by at most one."""
    if n_items < 0 or world < 1 or not (0 <= rank < world):
        raise ValueError("bad shard arguments")
    base, extra = divmod(n_items, world)
    lo = rank * base + min(rank, extra)
    return range(lo, lo + base + (1 if rank < extra else 0))


def replica_seed(base_seed: int, rank: int) -> int:
    """Seed of rank `rank`'s lattice: distinct per rank, reproducible."""
    return int(base_seed) + 1000 * int(rank)


def _reduce(x: float, op, device=None) -> float:
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    if device is None:
        device = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(x: float, device=None) -> float:
    return _reduce(x, dist.ReduceOp.MAX, device)


def sum_over_ranks(x: float, device=None) -> float:
    return _reduce(x, dist.ReduceOp.SUM, device)


def barrier():
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()
