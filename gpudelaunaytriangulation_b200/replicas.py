"""Host-side plumbing for running independent replicas on several GPUs (one process per GPU).

The triangulation shards by independent point sets, so ranks never exchange point data:
the only collectives are a barrier around timed regions and a max-over-ranks reduction of
device times.  Set partitioning for ensembles keeps whole sets on one rank.
"""
from __future__ import annotations

import numpy as np


def replica_seed(base: int, rank: int) -> int:
    """Distinct, reproducible input seed per rank."""
    return int(base) + 7919 * int(rank)


def shard_sets(sizes, world: int, rank: int) -> np.ndarray:
    """Indices of the sets owned by `rank`: greedy longest-first assignment to the least
    loaded rank (points per rank balanced), whole sets only, deterministic."""
    sizes = np.asarray(sizes, dtype=np.int64)
    order = np.argsort(-sizes, kind="stable")
    load = np.zeros(world, dtype=np.int64)
    owner = np.empty(len(sizes), dtype=np.int64)
    for s in order:
        r = int(np.argmin(load))
        owner[s] = r
        load[r] += sizes[s]
    return np.nonzero(owner == rank)[0]


class ReplicaGroup:
    """Barrier and max-reduction over the ranks of an initialised torch.distributed group
    (any backend); a no-op group when world == 1."""

    def __init__(self, world: int, rank: int, device=None):
        self.world = int(world)
        self.rank = int(rank)
        self.device = device

    def barrier(self):
        if self.world > 1:
            import torch.distributed as dist

            dist.barrier()

    def max_over_ranks(self, x: float) -> float:
        if self.world == 1:
            return float(x)
        import torch
        import torch.distributed as dist

        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def sum_over_ranks(self, x: float) -> float:
        if self.world == 1:
            return float(x)
        import torch
        import torch.distributed as dist

        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return float(t.item())

    def throughput(self, points_this_rank: int, ms_this_rank: float) -> tuple[float, float]:
        """(whole-job Mpoints/s, max-over-ranks ms): all ranks' points over the slowest
        rank's device time."""
        ms = self.max_over_ranks(ms_this_rank)
        pts = self.sum_over_ranks(points_this_rank)
        return pts / (ms / 1e3) / 1e6, ms
