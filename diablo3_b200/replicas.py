"""Independent replicas on several GPUs of one node (one process per GPU,
launched by torchrun): the substep of one channel has no data-parallel
exchange, so N GPUs run N independent channels, nothing is sharded and no
collective sits on the data path.  The only collectives are the host-side
ones of the measurement: barriers around the timed region and the MAX of the
ranks' device times.

The process group uses NCCL on GPUs and gloo on CPUs (the host logic is
tested with gloo ranks); rendezvous over MASTER_ADDR / MASTER_PORT.
"""
from __future__ import annotations

import os
from dataclasses import dataclass
from datetime import timedelta


@dataclass
class Ranks:
    world: int
    rank: int
    local: int

    @property
    def leader(self) -> bool:
        return self.rank == 0


def from_env() -> Ranks:
    """WORLD_SIZE, RANK and LOCAL_RANK as torchrun sets them (1, 0, 0 alone)."""
    return Ranks(int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
                 int(os.environ.get("LOCAL_RANK", "0")))


def init(r: Ranks, backend: str = "nccl", timeout_s: float = 300.0) -> None:
    """Join the process group when there is more than one rank; a short
    timeout makes ranks that wait for a missing peer fail instead of hang."""
    if r.world > 1:
        import torch.distributed as dist
        dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))


def barrier(r: Ranks) -> None:
    if r.world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(r: Ranks, value: float, device: str = "cuda") -> float:
    """The largest of the ranks' values (the job takes as long as its
    slowest replica)."""
    if r.world == 1:
        return float(value)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(points: int, substeps: int, r: Ranks, ms: float) -> float:
    """Whole-job grid-point substeps per second: every rank advanced `points`
    grid points by `substeps` substeps, in `ms` milliseconds (the MAX over
    ranks)."""
    return points * substeps * r.world / (ms / 1e3)


def finish(r: Ranks) -> None:
    if r.world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
