"""Replica parallelism: one independent scenario per rank, no collective on
the data path.

A scenario does not shard without an all-to-all transpose every half-step
(consecutive half-steps sweep orthogonal directions), and the reference runs
on one GPU only, so N GPUs run N replicas: rank r solves its own seeded
scenario (weak scaling). The only collectives are for timing: a barrier
around the timed region and the maximum of the ranks' device times. Every
rank takes the same collective steps in the same order.

The process group gets a short timeout so that ranks waiting for a rank that
failed end with an error instead of hanging.
"""
from __future__ import annotations

import os
from datetime import timedelta

DEFAULT_TIMEOUT_S = 120


def env_ranks():
    """(rank, local_rank, world_size) from the launcher's environment."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", str(rank)))
    return rank, local, ws


def init(backend: str = "nccl", timeout_s: float = DEFAULT_TIMEOUT_S):
    """Join the process group when WORLD_SIZE > 1. With nccl, rank r uses
    cuda:LOCAL_RANK. Returns (rank, local_rank, world_size)."""
    rank, local, ws = env_ranks()
    if ws > 1:
        import torch
        import torch.distributed as dist
        kw = {}
        if backend == "nccl":
            torch.cuda.set_device(local)
            kw["device_id"] = torch.device("cuda", local)
        dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s), **kw)
    return rank, local, ws


def _device():
    import torch.distributed as dist
    import torch
    if dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def max_over_ranks(x: float, ws: int) -> float:
    """Maximum of a per-rank scalar (the timed region's device time)."""
    if ws == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, ws: int) -> float:
    """Sum of a per-rank scalar (units processed by all replicas)."""
    if ws == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(ws: int):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def finish(ws: int):
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def replica_seed(base: int, rank: int) -> int:
    """Seed of rank r's scenario: replicas solve different scenarios."""
    return int(base) + 7919 * int(rank)
