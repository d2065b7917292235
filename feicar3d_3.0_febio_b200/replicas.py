"""Replicas across GPUs: one process per GPU, each solving its own problems.

The pressure solves of independent problems (a batch, a serving queue, the
copies of one case in a scaling run) exchange nothing, so several GPUs run
them as replicas: every rank takes its own share of the problems and no
collective touches the data path.  The only collectives are the ones that
frame a measurement (a barrier before and after the timed region, the
maximum of the ranks' times, the sum of their counts).  They go through
``torch.distributed`` (NCCL on GPUs, gloo on the CPU) and every rank calls
them in the same order.
"""
from __future__ import annotations

from typing import Sequence


def shard_balanced(costs: Sequence[float], world: int) -> list[list[int]]:
    """Problem indices of each rank: largest-first greedy assignment to the
    rank with the least total cost so far (ties to the lower rank), so the
    slowest rank, which sets the job time, carries as little as possible.
    Deterministic: every rank computes the same split on its own."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(i)
        load[r] += float(costs[i])
    for lst in out:
        lst.sort()
    return out


class Ranks:
    """The measurement collectives of one replica job (world 1 needs no
    process group and calls none)."""

    def __init__(self, dist=None, device=None):
        self.dist = dist
        self.device = device
        if dist is not None and dist.is_initialized():
            self.rank, self.world = dist.get_rank(), dist.get_world_size()
        else:
            self.rank, self.world = 0, 1

    def barrier(self):
        if self.world > 1:
            self.dist.barrier()

    def _reduce(self, x: float, op) -> float:
        if self.world == 1:
            return float(x)
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x: float) -> float:
        """The maximum over ranks (a replica job ends with its slowest rank)."""
        return self._reduce(x, self.dist.ReduceOp.MAX if self.world > 1 else None)

    def sum(self, x: float) -> float:
        return self._reduce(x, self.dist.ReduceOp.SUM if self.world > 1 else None)
