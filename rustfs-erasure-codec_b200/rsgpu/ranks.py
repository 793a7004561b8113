"""One process per GPU: rank discovery from the launcher's environment, the
process group, and the reductions taken over ranks.

The erasure-coding path shards by stripe (every stripe is independent), so
ranks exchange no data: they meet only at barriers and at the max-over-ranks
reduction of step times that turns per-rank timings into a whole-job figure.
The group is created only when more than one rank runs; with one rank every
call is local and no process group exists.
"""
from __future__ import annotations

import datetime
import os
from dataclasses import dataclass
from typing import Mapping, Optional, Tuple


@dataclass(frozen=True)
class Ranks:
    rank: int
    world: int
    local: int


def from_env(env: Optional[Mapping[str, str]] = None) -> Ranks:
    """RANK / WORLD_SIZE / LOCAL_RANK as torchrun sets them (0 / 1 / 0 when unset)."""
    env = os.environ if env is None else env
    r = Ranks(int(env.get("RANK", "0")), int(env.get("WORLD_SIZE", "1")), int(env.get("LOCAL_RANK", "0")))
    if r.world < 1 or not 0 <= r.rank < r.world:
        raise ValueError(f"invalid rank {r.rank} of world {r.world}")
    return r


def stripe_share(n: int, rank: int, world: int) -> Tuple[int, int]:
    """(first, count) of rank's contiguous share of n stripes; shares differ by
    at most one stripe and cover 0..n exactly once."""
    base, extra = divmod(n, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


class Group:
    """The process group of all ranks.  `backend` is "nccl" on GPUs and
    "gloo" for host-only runs; `device` is where reduction tensors live
    ("cuda" for NCCL, "cpu" for gloo).  A short `timeout_s` makes ranks that
    wait on a rank that died or never arrived fail with an error instead of
    hanging."""

    def __init__(self, ranks: Ranks, backend: str = "nccl", timeout_s: float = 120.0, device: str = "cuda"):
        self.ranks = ranks
        self.device = device
        self._dist = None
        if ranks.world > 1:
            import torch.distributed as dist

            dist.init_process_group(backend, rank=ranks.rank, world_size=ranks.world,
                                    timeout=datetime.timedelta(seconds=timeout_s))
            self._dist = dist

    @property
    def distributed(self) -> bool:
        return self._dist is not None

    def barrier(self) -> None:
        if self._dist is not None:
            self._dist.barrier()

    def _reduce(self, x: float, op) -> float:
        import torch

        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self._dist.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x: float) -> float:
        """Largest x over all ranks (the slowest rank's time)."""
        return float(x) if self._dist is None else self._reduce(x, self._dist.ReduceOp.MAX)

    def sum(self, x: float) -> float:
        return float(x) if self._dist is None else self._reduce(x, self._dist.ReduceOp.SUM)

    def close(self) -> None:
        """Every rank takes the same last barrier, then the group is destroyed."""
        if self._dist is not None:
            self._dist.barrier()
            self._dist.destroy_process_group()
            self._dist = None
