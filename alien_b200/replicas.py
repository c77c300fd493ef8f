"""Replicas across the GPUs of one node.

One process per GPU (torchrun), each stepping its own worlds: either a
replica workload per rank, or one set of worlds split across the ranks by
cell count (``partition_worlds``).  The physics
stage does not partition a world, and worlds never interact, so ranks share
no data: the only cross-rank traffic is the measurement (the slowest rank's
timed region and the sum of the work done), plus barriers around the timed
region.  The reduction tensors live on the GPU under NCCL and on the CPU
under gloo, so the same code runs in multi-process CPU tests.
"""
from __future__ import annotations

import datetime
import os


class Replicas:
    def __init__(self, backend: str | None = None, timeout_s: float = 300.0):
        import torch
        import torch.distributed as dist

        self._torch, self._dist = torch, dist
        self.rank = int(os.environ.get("RANK", 0))
        self.world_size = int(os.environ.get("WORLD_SIZE", 1))
        self.local_rank = int(os.environ.get("LOCAL_RANK", 0))
        self.cuda = torch.cuda.is_available() and backend != "gloo"
        if self.cuda:
            torch.cuda.set_device(self.local_rank)
        self.backend = backend or ("nccl" if self.cuda else "gloo")
        self._own_group = False
        if self.world_size > 1 and not dist.is_initialized():
            dist.init_process_group(self.backend, timeout=datetime.timedelta(seconds=timeout_s))
            self._own_group = True

    def seed(self, base: int = 0) -> int:
        """workload seed of this rank: distinct worlds on every rank"""
        return base + 1000 * self.rank

    def share(self, sizes) -> list[int]:
        """indices of the worlds this rank steps when one set of worlds is
        split across all ranks (``partition_worlds``)"""
        return partition_worlds(sizes, self.world_size)[self.rank]

    def barrier(self) -> None:
        if self.cuda:
            self._torch.cuda.synchronize()
        if self.world_size > 1:
            self._dist.barrier()

    def _reduce(self, x: float, op) -> float:
        if self.world_size == 1:
            return float(x)
        t = self._torch.tensor([float(x)], dtype=self._torch.float64, device="cuda" if self.cuda else "cpu")
        self._dist.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x: float) -> float:
        return self._reduce(x, self._dist.ReduceOp.MAX)

    def sum(self, x: float) -> float:
        return self._reduce(x, self._dist.ReduceOp.SUM)

    def close(self) -> None:
        if self._own_group and self._dist.is_initialized():
            self._dist.destroy_process_group()
            self._own_group = False


def partition_worlds(sizes, n_ranks: int) -> list[list[int]]:
    """Split independent worlds across ranks, balancing the cells per rank.

    Greedy longest-processing-time placement: worlds in decreasing size
    (ties by index), each to the rank with the fewest cells so far (ties by
    rank).  Every rank computes the same split from the same sizes, so the
    placement needs no communication.  The largest rank load is at most
    4/3 of the optimum (Graham's bound for this rule).  Returns the world
    indices of each rank in ascending order.
    """
    if n_ranks < 1:
        raise ValueError("n_ranks must be at least 1")
    load = [0] * n_ranks
    share: list[list[int]] = [[] for _ in range(n_ranks)]
    for i in sorted(range(len(sizes)), key=lambda k: (-int(sizes[k]), k)):
        r = min(range(n_ranks), key=lambda q: (load[q], q))
        share[r].append(i)
        load[r] += int(sizes[i])
    return [sorted(s) for s in share]
