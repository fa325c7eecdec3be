"""Replica plumbing for running independent registrations on several GPUs of one node.

Registrations do not exchange anything while they run, so the multi-GPU form is one
process per GPU, each with its own contexts, and the only collectives are the
barriers around a timed region and the maximum of the ranks' timings (the job takes
as long as its slowest rank).  Launch with torchrun; RANK / WORLD_SIZE / LOCAL_RANK /
MASTER_ADDR / MASTER_PORT come from the environment.

The backend is "nccl" for the GPU runs and "gloo" for the CPU tests of this module.
The process group gets a short timeout, so that ranks left waiting for a rank that
failed end with an error instead of hanging.
"""
from __future__ import annotations

import datetime
import os
from dataclasses import dataclass

DEFAULT_TIMEOUT_S = 120.0


@dataclass(frozen=True)
class RankEnv:
    world: int
    rank: int
    local: int

    @property
    def reports(self) -> bool:
        """Only rank 0 prints the job's result line."""
        return self.rank == 0


def rank_env() -> RankEnv:
    return RankEnv(world=int(os.environ.get("WORLD_SIZE", "1")),
                   rank=int(os.environ.get("RANK", "0")),
                   local=int(os.environ.get("LOCAL_RANK", "0")))


def init(env: RankEnv, backend: str = "nccl", timeout_s: float = DEFAULT_TIMEOUT_S):
    """Joins the process group when there is more than one rank; returns the
    torch.distributed module, or None for a single rank."""
    if env.world <= 1:
        return None
    import torch.distributed as dist

    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    dist.init_process_group(backend, rank=env.rank, world_size=env.world,
                            timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def barrier(dist) -> None:
    if dist is not None:
        dist.barrier()


def max_over_ranks(dist, value: float, device: str = "cpu") -> float:
    """The largest `value` over all ranks (every rank gets it)."""
    if dist is None:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank: float, world: int, seconds: float) -> float:
    """Whole-job throughput: the units every rank processed over the slowest rank's
    time."""
    return units_per_rank * world / seconds


def finish(dist) -> None:
    if dist is not None and dist.is_initialized():
        dist.destroy_process_group()
