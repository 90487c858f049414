"""Replica plumbing for running the matrix-free path on several GPUs.

The weighted-quadrature operators act on independent patches: nothing on
the data path is exchanged between GPUs.  Running on N GPUs therefore means
N replicas, one process per GPU, each owning a disjoint set of patches
(weak scaling).  The only collectives are barriers and the reduction of the
per-rank device times to their maximum, which is what whole-job throughput
is quoted on.  The same functions run over NCCL (CUDA tensors) and gloo
(CPU tensors), so the host logic is testable without a GPU.
"""
from __future__ import annotations

import datetime
import os
from dataclasses import dataclass
from typing import List, Optional, Sequence

import torch


@dataclass(frozen=True)
class RankInfo:
    world: int
    rank: int
    local: int


def rank_env() -> RankInfo:
    """Rank layout from the launcher's environment (torchrun sets WORLD_SIZE,
    RANK and LOCAL_RANK; a plain launch is one rank)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", str(rank)))
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"bad rank layout: RANK={rank} WORLD_SIZE={world}")
    return RankInfo(world, rank, local)


def init_group(info: RankInfo, backend: str = "nccl", timeout_s: float = 120.0):
    """Join the process group when there is more than one rank; returns the
    `torch.distributed` module, or None for a single rank.  A short timeout
    makes a rank that never arrives end the others' next collective with an
    error instead of a hang."""
    if info.world == 1:
        return None
    import torch.distributed as dist

    if not dist.is_initialized():
        dist.init_process_group(backend, rank=info.rank, world_size=info.world,
                                timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def shard_units(n_units: int, world: int, rank: int) -> List[int]:
    """Contiguous, balanced share of `n_units` independent units (patches,
    requests) for `rank`: the first n_units % world ranks take one extra.
    Every unit lands on exactly one rank."""
    if n_units < 0 or world < 1 or not 0 <= rank < world:
        raise ValueError(f"bad shard request: units={n_units} world={world} rank={rank}")
    base, extra = divmod(n_units, world)
    lo = rank * base + min(rank, extra)
    hi = lo + base + (1 if rank < extra else 0)
    return list(range(lo, hi))


def max_over_ranks(values: Sequence[float], dist=None, device: Optional[torch.device] = None
                   ) -> List[float]:
    """Element-wise maximum of per-rank times (ms) over all ranks; identity for
    a single rank.  Every rank must call it, in the same order."""
    vals = [float(v) for v in values]
    if dist is None:
        return vals
    dev = device if device is not None else (
        torch.device("cuda", torch.cuda.current_device())
        if dist.get_backend() == "nccl" else torch.device("cpu"))
    t = torch.tensor(vals, dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]


def job_throughput(units_per_rank: float, world: int, ms_per_step: float, scale: float = 1e9
                   ) -> float:
    """Whole-job throughput: the units all ranks processed in one step over the
    slowest rank's step time (ms), in units of `scale` per second."""
    if ms_per_step <= 0:
        raise ValueError(f"step time must be positive, got {ms_per_step}")
    return world * units_per_rank / (ms_per_step * 1e-3) / scale


def finish(dist) -> None:
    """Barrier and leave the group (no-op for a single rank)."""
    if dist is None:
        return
    dist.barrier()
    dist.destroy_process_group()
