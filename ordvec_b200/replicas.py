"""Replica plumbing for multi-GPU runs of the compressed-scan path.

The path partitions by query: every rank holds a full replica of the indices
and scores its own query shard, so nothing is exchanged on the data path.  The
only collectives are the timing barrier and the max over ranks of the timed
totals (a job is as slow as its slowest rank); the whole-job rate is the units
every rank processed divided by that maximum ("weak" scaling: the per-rank
shard is fixed as ranks are added).

One process per GPU, launched by ``torch.distributed.run``; RANK, WORLD_SIZE,
LOCAL_RANK and MASTER_* come from the environment.  ``backend`` is "nccl" for
GPU ranks and "gloo" for CPU ranks (tests).
"""
from __future__ import annotations

import datetime
import os
from typing import Callable, Optional, Tuple

# Query shards are generated from the run's seed plus a per-rank offset, so
# ranks never score the same synthetic queries.
SHARD_SEED_STRIDE = 1000


def rank_env() -> Tuple[int, int, int]:
    """(rank, world_size, local_rank) from the launcher's environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard_seed(base_seed: int, rank: int) -> int:
    return base_seed + SHARD_SEED_STRIDE * rank


def whole_job_rate(units_per_rank: int, world: int, max_total_ms: float) -> float:
    """Units per second for the whole job: every rank's units over the slowest rank's time."""
    if max_total_ms <= 0.0:
        raise ValueError("timed total must be positive")
    return units_per_rank * world / (max_total_ms * 1e-3)


class ReplicaGroup:
    """Barrier and max-over-ranks for replica runs; a no-op group when world == 1."""

    def __init__(self, backend: str, device=None, timeout_s: float = 120.0,
                 sync: Optional[Callable[[], None]] = None):
        self.rank, self.world, self.local = rank_env()
        self.device = device
        self._sync = sync
        self._dist = None
        if self.world > 1:
            import torch.distributed as dist

            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self._dist = dist

    @property
    def is_root(self) -> bool:
        return self.rank == 0

    def barrier(self) -> None:
        if self._sync:
            self._sync()
        if self._dist:
            self._dist.barrier()

    def max_over_ranks(self, x: float) -> float:
        if not self._dist:
            return float(x)
        import torch

        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.MAX)
        return float(t.item())

    def close(self) -> None:
        if self._dist:
            self._dist.barrier()
            self._dist.destroy_process_group()
            self._dist = None
