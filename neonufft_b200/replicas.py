"""Replica execution across ranks: one process per GPU, each rank running whole transforms on its
own point set. The NUFFT path has no exchange step between point sets, so no data crosses
NVLink and scaling is weak (fixed work per GPU); the only collectives are the barrier around a
timed region and the max over ranks of its duration.

Host-side helpers shared by bench.py and the multi-process tests (gloo on CPU, NCCL on GPUs).
The reference has no multi-process layer; its GPU plans run on one device and one stream
(src/neonufft/gpu/plan.cpp:22-45).
"""
from __future__ import annotations

import os
from dataclasses import dataclass


@dataclass(frozen=True)
class RankEnv:
    world: int
    rank: int
    local: int


def rank_env() -> RankEnv:
    """WORLD_SIZE / RANK / LOCAL_RANK as set by torch.distributed.run (1 / 0 / 0 without it)."""
    return RankEnv(int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
                   int(os.environ.get("LOCAL_RANK", "0")))


def rank_seed(base: int, rank: int) -> int:
    """Seed of a rank's synthetic point set: every rank transforms different points."""
    return int(base) + 97 * int(rank)


def _group_size() -> int:
    import torch.distributed as dist
    return dist.get_world_size() if dist.is_available() and dist.is_initialized() else 1


def barrier() -> None:
    if _group_size() > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(value: float, device="cpu") -> float:
    """Largest value over the ranks of the default group (the value itself on one rank)."""
    if _group_size() == 1:
        return float(value)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(world: int, units_per_rank: float, ms_per_step: float) -> float:
    """Whole-job units per second: every rank processed units_per_rank per step, and the step
    time is the max over ranks."""
    if ms_per_step <= 0:
        raise ValueError("step time must be positive")
    return world * units_per_rank / (ms_per_step * 1e-3)
