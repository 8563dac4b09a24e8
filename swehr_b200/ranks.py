"""One process per GPU: rank coordination and placement of independent work.

SWEHR's work shards without exchange when it is many independent scenarios
(an ensemble, a serving stream): each rank holds its own scenarios and no
data crosses GPUs.  A single domain runs as one replica per rank.  The only
collectives are host-level -- a barrier around timed regions and a max (or
sum) of a few scalars for reporting -- so torch.distributed is plumbing
here: NCCL on GPUs, gloo on the CPU for tests.
"""
from __future__ import annotations

import datetime
import heapq
import os
from typing import List, Sequence


class Ranks:
    """The process group of this job, from the torchrun environment
    (RANK, WORLD_SIZE, MASTER_ADDR, MASTER_PORT).  world 1 needs no group."""

    def __init__(self, backend: str = "nccl", timeout_s: float = 600.0):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.dist = None
        if self.world > 1:
            import torch.distributed as dist
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    def _tensor(self, x: float):
        import torch
        dev = "cuda" if self.backend == "nccl" else "cpu"
        return torch.tensor([float(x)], dtype=torch.float64, device=dev)

    def barrier(self) -> None:
        if self.dist is not None:
            t = self._tensor(1.0)
            self.dist.all_reduce(t)
            if self.backend == "nccl":
                import torch
                torch.cuda.synchronize()

    def max(self, x: float) -> float:
        if self.dist is None:
            return float(x)
        t = self._tensor(x)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        if self.dist is None:
            return float(x)
        t = self._tensor(x)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return float(t.item())

    def close(self) -> None:
        if self.dist is not None:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None


def shard(weights: Sequence[float], world: int) -> List[List[int]]:
    """Split independent items over `world` ranks, balancing the summed
    weight (cells x steps): largest item first onto the least-loaded rank,
    ties to the lower rank.  Deterministic, so every rank computes the same
    placement without communicating; each rank's list keeps input order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    heap = [(0.0, r) for r in range(world)]
    out: List[List[int]] = [[] for _ in range(world)]
    for k in sorted(range(len(weights)), key=lambda k: (-weights[k], k)):
        load, r = heapq.heappop(heap)
        out[r].append(k)
        heapq.heappush(heap, (load + float(weights[k]), r))
    return [sorted(s) for s in out]
