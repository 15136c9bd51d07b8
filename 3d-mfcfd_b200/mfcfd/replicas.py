"""Multi-GPU runs as independent replicas.

The LU-SGS sweeps visit points in one global order (the alias breadth-first
order, implicit_forward_and_reverse_sweeps.f90:26-84), so one cloud does not
shard without changing the algorithm.  N GPUs therefore run N independent
solves, one process per GPU, with no collective on the data path; the only
collectives are a barrier around the timed region and a max of the ranks'
device times.
"""
from __future__ import annotations

import datetime
import os


def env():
    """(rank, world_size, local_rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str, timeout_s: float = 300.0):
    """Join the process group when world_size > 1 (MASTER_ADDR/PORT from env)."""
    import torch.distributed as dist
    rank, world, _ = env()
    if world > 1 and not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return rank, world


def barrier():
    import torch.distributed as dist
    if dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()


def max_over_ranks(value: float, device="cpu") -> float:
    """Max of a per-rank scalar (device times are reported as the slowest rank)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    if dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_seed(base_seed: int, rank: int) -> int:
    """Each rank solves its own seeded cloud."""
    return base_seed + rank


def throughput(points_per_rank: int, steps: int, seconds_max: float, world: int) -> float:
    """Whole-job point-iterations per second: all ranks' points over the slowest rank's time."""
    return world * points_per_rank * steps / seconds_max


def finalize():
    import torch.distributed as dist
    if dist.is_initialized():
        dist.destroy_process_group()
