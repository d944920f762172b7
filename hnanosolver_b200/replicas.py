"""Independent replicas of the step on several GPUs of one node (one process per GPU).

The solver does not shard a grid across GPUs: under torchrun every rank steps its own copy of
the workload (seeded by its rank), and the only collectives are the timing protocol's: a
barrier on each side of the timed region and the maximum of the ranks' times. NCCL carries
them on GPUs; the same calls run over gloo on the host, which is how they are tested.
"""
from __future__ import annotations

import datetime
import os
from dataclasses import dataclass


@dataclass
class Ranks:
    rank: int
    world: int
    local: int

    @property
    def distributed(self) -> bool:
        return self.world > 1


def ranks_from_env() -> Ranks:
    """RANK / WORLD_SIZE / LOCAL_RANK as torchrun sets them (one process: 0 / 1 / 0)."""
    return Ranks(int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0)))


def start(ranks: Ranks, backend: str = "nccl", timeout_s: float = 120.0) -> None:
    """Joins the process group when there is more than one rank (a short timeout, so that ranks
    left waiting for a missing peer end with an error rather than hang)."""
    if not ranks.distributed:
        return
    import torch.distributed as td

    td.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))


def barrier(ranks: Ranks) -> None:
    if ranks.distributed:
        import torch.distributed as td

        td.barrier()


def max_over_ranks(ranks: Ranks, value: float, device=None) -> float:
    """The largest of the ranks' values (every rank gets it); the value itself on one rank."""
    if not ranks.distributed:
        return value
    import torch
    import torch.distributed as td

    t = torch.tensor([value], dtype=torch.float64, device=device)
    td.all_reduce(t, op=td.ReduceOp.MAX)
    return float(t.item())


def finish(ranks: Ranks) -> None:
    if ranks.distributed:
        import torch.distributed as td

        td.destroy_process_group()


def seed_of(ranks: Ranks) -> int:
    """Each replica's synthetic fields are seeded by its rank."""
    return ranks.rank


def aggregate_rate(ranks: Ranks, units_per_rank: int, steps: int, max_ms: float) -> float:
    """Whole-job throughput of weak-scaled replicas: all ranks' units over the slowest rank's time."""
    return ranks.world * units_per_rank * steps / (max_ms / 1e3)
