"""Multi-GPU plumbing of the benchmark: independent replicas.

Cells are independent, so N GPUs run N replicas of the solve on disjoint
seeded cell sets with no collective on the data path (weak scaling).  The
only cross-rank steps are the barrier around the timed region, the
max-over-ranks of its device time and the sum over ranks of the cells that
finished.  One process per GPU; NCCL on GPUs, gloo
for the CPU tests of this logic.
"""
from __future__ import annotations

import os
from datetime import timedelta

SEED_STRIDE = 7919  # rank r uses seed base + SEED_STRIDE * r


def init(backend: str = "nccl", timeout_s: float = 300.0):
    """(world, rank, local_rank) from the torchrun environment; joins the
    process group when world > 1 (rendezvous at MASTER_ADDR/MASTER_PORT)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist

        if backend == "nccl":
            import torch

            # each rank owns its GPU before NCCL binds a communicator to it
            torch.cuda.set_device(local)
        if not dist.is_initialized():
            dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))
    return world, rank, local


def rank_seed(base: int, rank: int) -> int:
    return base + SEED_STRIDE * rank


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, world: int) -> float:
    """Sum of a per-rank count (successful cell-steps) over the job."""
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(world: int) -> None:
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def aggregate_throughput(cells_per_rank: int, steps: int, world: int, max_seconds: float) -> float:
    """Whole-job cell-steps/s: every rank's cells over the slowest rank's time."""
    return world * cells_per_rank * steps / max_seconds


def finalize(world: int) -> None:
    if world > 1:
        import torch.distributed as dist

        if dist.is_initialized():
            dist.destroy_process_group()
