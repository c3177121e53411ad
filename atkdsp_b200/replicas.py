"""Stream sharding across GPUs: one process per GPU, no collective on the data path.

Channelizer streams are independent (a stream's hops depend only on its own
samples and carried state, reference src/channelizer.c:214-217), so the
multi-GPU form of the path is replicas: each rank owns a disjoint set of
streams and runs the same batched kernel on its own GPU. The only cross-rank
traffic is bookkeeping -- who owns which stream, and the reductions of
timings and counts -- which this module holds:

* ``partition(weights, world)``: streams -> ranks, balancing bytes/s (a
  stream's weight is its sample rate times bytes per sample). Greedy
  longest-first onto the least-loaded rank; deterministic (ties break on the
  lower stream index, then the lower rank), so every rank computes the same
  assignment with no message exchanged.
* ``Replicas``: the process group from the launcher's environment (RANK,
  WORLD_SIZE, LOCAL_RANK, MASTER_ADDR/PORT); NCCL when CUDA is available,
  gloo otherwise; a short timeout so a rank that dies surfaces as an error
  in the others' next reduction rather than a hang. ``max`` / ``sum``
  reduce one float across ranks (a timed region is reported as the max over
  ranks, throughput as the sum of work over that max); ``gather`` collects
  small per-rank objects on every rank.
"""

from __future__ import annotations

import datetime
import os
from typing import Sequence

__all__ = ["partition", "Replicas"]


def partition(weights: Sequence[float], world: int) -> list[list[int]]:
    """Disjoint, complete assignment of len(weights) streams to `world` ranks.

    Returns one ascending index list per rank. The heaviest stream is placed
    first, each on the rank with the least total weight so far; the largest
    rank total is within one stream's weight of the mean.
    """
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(weights)), key=lambda i: (-float(weights[i]), i))
    load = [0.0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += float(weights[i])
    for lst in out:
        lst.sort()
    return out


class Replicas:
    """The rank's view of the replica group (a single process when WORLD_SIZE is 1)."""

    def __init__(self, backend: str | None = None, timeout_s: float = 120.0):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self._dist = None
        self.device = "cpu"
        if self.world > 1:
            import torch
            import torch.distributed as dist

            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            if backend is None:
                backend = "nccl" if torch.cuda.is_available() else "gloo"
            if backend == "nccl":
                torch.cuda.set_device(self.local_rank)
                self.device = f"cuda:{self.local_rank}"
            if not dist.is_initialized():
                dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self._dist = dist

    def my_streams(self, weights: Sequence[float]) -> list[int]:
        return partition(weights, self.world)[self.rank]

    def _reduce(self, x: float, op) -> float:
        if self._dist is None:
            return float(x)
        import torch

        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self._dist.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x: float) -> float:
        return self._reduce(x, self._dist.ReduceOp.MAX if self._dist else None)

    def sum(self, x: float) -> float:
        return self._reduce(x, self._dist.ReduceOp.SUM if self._dist else None)

    def barrier(self) -> None:
        if self._dist is not None:
            self._dist.barrier()

    def gather(self, obj) -> list:
        if self._dist is None:
            return [obj]
        out = [None] * self.world
        self._dist.all_gather_object(out, obj)
        return out

    def close(self) -> None:
        if self._dist is not None and self._dist.is_initialized():
            self._dist.destroy_process_group()
        self._dist = None
