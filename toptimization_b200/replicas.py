"""Replica bookkeeping for runs on several GPUs of one node.

The SIMP loop does not shard at the sizes in scope (a PCG iteration is tens
of microseconds of HBM time, less than an all-reduce round trip), so N GPUs
run N independent replicas: one process per GPU (`torchrun`), no collective
on the data path. Independent designs (a batch, a request stream) are dealt
out across the ranks. The only collectives are the barriers around a timed
region and the max over ranks of its duration, as the measurement needs.
"""

from __future__ import annotations

import os
from dataclasses import dataclass
from datetime import timedelta

import torch
import torch.distributed as dist


@dataclass(frozen=True)
class Ranks:
    rank: int
    world: int
    local: int

    @property
    def multi(self) -> bool:
        return self.world > 1


def from_env() -> Ranks:
    return Ranks(int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
                 int(os.environ.get("LOCAL_RANK", "0")))


def init(ranks: Ranks, backend: str = "nccl", timeout_s: float = 300.0,
         device: torch.device | None = None) -> None:
    """Join the process group (N > 1 only); a short timeout makes ranks that
    wait for a failed peer end with an error instead of hanging."""
    if not ranks.multi:
        return
    kw = {"device_id": device} if (backend == "nccl" and device is not None) else {}
    dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s), **kw)


def barrier(ranks: Ranks) -> None:
    if torch.cuda.is_available():
        torch.cuda.synchronize()
    if ranks.multi:
        dist.barrier()
    if torch.cuda.is_available():
        torch.cuda.synchronize()


def max_over_ranks(x: float, ranks: Ranks, device: torch.device | None = None) -> float:
    """Largest value of x over the ranks (the job's duration is its slowest
    replica's)."""
    if not ranks.multi:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank: float, seconds_max: float, ranks: Ranks) -> float:
    """Whole-job throughput: the units all ranks processed over the slowest
    rank's time."""
    return ranks.world * units_per_rank / seconds_max


def shard(items: list, ranks: Ranks) -> list:
    """This rank's share of independent items, dealt round-robin."""
    return items[ranks.rank::ranks.world]


def finish(ranks: Ranks) -> None:
    if ranks.multi and dist.is_initialized():
        dist.destroy_process_group()


__all__ = ["Ranks", "from_env", "init", "barrier", "max_over_ranks", "job_rate", "shard",
           "finish"]
