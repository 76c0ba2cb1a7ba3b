"""Replica plumbing for N GPUs of one node (weak scaling).

The path does not shard a single solve across GPUs here: every rank (one process per GPU)
advances its own independent batch of cases, seeded by its rank, and no collective touches
the data path. The only collectives are around the timed region: a barrier before and after,
the maximum of the per-rank device times and the sum of the per-rank cell counts, so that the
whole-job throughput is (sum of cells x steps) / (slowest rank's time).
"""
from __future__ import annotations

import datetime
import os


def dist_env():
    """(rank, world size, local rank) from the torch.distributed launcher's environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def rank_seed(base: int, rank: int) -> int:
    """Seed of a rank's batch: distinct per rank, equal to `base` on rank 0."""
    return base + 7919 * rank


def init(backend: str, timeout_s: float = 300.0) -> None:
    import torch.distributed as dist
    if not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))


def _reduce(x: float, op: str, device: str) -> float:
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def max_over_ranks(x: float, device: str = "cpu") -> float:
    return _reduce(x, "max", device)


def sum_over_ranks(x: float, device: str = "cpu") -> float:
    return _reduce(x, "sum", device)


def barrier() -> None:
    import torch.distributed as dist
    if dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()


def throughput(cells_all_ranks: float, steps: int, seconds_max: float) -> float:
    """Whole-job cell-updates per second."""
    return cells_all_ranks * steps / seconds_max
