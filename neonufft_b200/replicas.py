"""Execution across ranks: one process per GPU, each rank running whole transforms. The NUFFT path
has no exchange step between transforms, so no data crosses NVLink; the only collectives are the
barrier around a timed region and the max over ranks of its duration.

Two ways to use the ranks:
  * replicas: every rank runs its own point set (weak scaling, bench.py --gpus N);
  * one batch split over the ranks (ShardedBatch): every rank sees the same list of independent
    transforms and runs a cost-balanced, disjoint subset of it, chosen by the same deterministic
    rule on every rank, so no assignment is communicated and no transform runs twice.

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


# ---- one batch of independent transforms split over the ranks ---------------------------------
def transform_cost(dim: int, num_nu: int, modes, tol: float = 1e-6, upsampfac: float = 2.0,
                   precision: str = "f32", n_spread: int = 0) -> float:
    """Estimated cost of one transform, the estimate the batch balances its streams with
    (csrc/batch.cu): spreading work M w^d plus 5 c log2 c for the FFT of the c fine-grid cells
    (fine grid max(2w, N upsampfac) per dimension). Host-only: needs no GPU."""
    import ctypes as C
    import math
    from . import _lib as L
    from .plan import check
    w = int(n_spread)
    if w <= 0:
        wc, beta, c = C.c_int(0), C.c_double(0), C.c_double(0)
        prec = L.NNB_DOUBLE if precision == "f64" else L.NNB_FLOAT
        check(L.load().nnb_es_kernel_params(tol, upsampfac, prec, C.byref(wc), C.byref(beta),
                                            C.byref(c)))
        w = wc.value
    cells = 1.0
    for m in list(modes)[:dim]:
        cells *= float(max(2 * w, int(float(m) * upsampfac)))
    return float(num_nu) * float(w) ** dim + 5.0 * cells * math.log2(max(2.0, cells))


def shard_owners(costs, world: int) -> list:
    """Owner rank of each transform: transforms in decreasing cost (ties by index), each to the
    least-loaded rank so far (ties to the lowest rank) -- the longest-processing-time rule, whose
    largest load is at most 4/3 of the optimum. Deterministic, so every rank computes the same
    owners from the same costs without communicating."""
    if world < 1:
        raise ValueError("world size must be positive")
    owners = [0] * len(costs)
    load = [0.0] * world
    for i in sorted(range(len(costs)), key=lambda j: (-float(costs[j]), j)):
        r = min(range(world), key=lambda k: (load[k], k))
        owners[i] = r
        load[r] += float(costs[i])
    return owners


def shard_loads(costs, owners, world: int) -> list:
    """Estimated cost per rank of an assignment."""
    load = [0.0] * world
    for c, r in zip(costs, owners):
        load[r] += float(c)
    return load


class ShardedBatch:
    """This rank's part of one batch of independent transforms split over `world` ranks.

    Every rank builds the same list of transforms (same order, same sizes), computes the same
    owners (shard_owners of their costs) and adds to its own Batch only the transforms it owns;
    execute() runs them. The union over the ranks is the whole batch, each transform run once.
    There is no collective on the data path: each rank reads its own transforms' inputs and
    writes their outputs."""

    def __init__(self, opt, dtype, owners, rank: int, num_streams: int = 4, stream=None,
                 device_alloc=None):
        from .plan import Batch
        self.owners = list(owners)
        self.rank = int(rank)
        self.batch = Batch(opt, dtype, num_streams=num_streams, stream=stream,
                           device_alloc=device_alloc)
        self.local = []  # indices of the whole batch held here, in the order added

    def owns(self, index: int) -> bool:
        return self.owners[index] == self.rank

    def owned(self) -> list:
        return [i for i, r in enumerate(self.owners) if r == self.rank]

    def add(self, index: int, type_: int, sign: int, loc, modes, inp, out, strides, opt=None):
        """Adds transform `index` of the whole batch; it must be owned by this rank."""
        if not self.owns(index):
            raise ValueError(f"transform {index} belongs to rank {self.owners[index]}")
        if index in self.local:
            raise ValueError(f"transform {index} added twice")
        self.batch.add(type_, sign, loc, modes, inp, out, strides, opt)
        self.local.append(index)

    def execute(self, mode=None) -> None:
        if self.local:
            self.batch.execute(self.batch.GRAPH if mode is None else mode)

    def close(self) -> None:
        self.batch.close()
