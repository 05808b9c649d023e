"""Replicas across GPUs: one process per GPU, independent wraps per rank.

Wraps are independent problems, so multi-GPU is a host dispatcher and no
collective on the data path: each rank takes a share of the wraps, solves them
on its own GPU, and the results come back to rank 0 in submission order.  The
only collectives are host bookkeeping -- a barrier around timed regions, the
max of the ranks' times and the sum of their work, and the final gather.

The reference has no multi-GPU code (its solver uses the current device), so
there is nothing on its side to mirror; the process model is torchrun's (one
process per GPU, RANK / WORLD_SIZE / LOCAL_RANK / MASTER_ADDR from the
environment).
"""

from __future__ import annotations

import datetime
import os
from typing import Any, Callable, Sequence


def wrap_cost(case) -> float:
    """Relative cost of one wrap for load balancing: its query and assembly
    work grows with the template vertices, the hierarchy with the target
    triangles."""
    template, target = case[0], case[3]
    return float(len(template)) * 4.0 + float(len(target))


def assign(costs: Sequence[float], world: int) -> list[list[int]]:
    """Longest-processing-time-first assignment of items to `world` ranks:
    items in decreasing cost (ties by index), each to the least-loaded rank
    (ties by rank).  Deterministic, so every rank computes the same split
    without talking to the others.  Each rank's list is in submission order."""
    loads = [0.0] * world
    shares: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda i: (-costs[i], i)):
        r = min(range(world), key=lambda r: (loads[r], r))
        loads[r] += costs[i]
        shares[r].append(i)
    return [sorted(s) for s in shares]


class ReplicaGroup:
    """The process group of a replica run.  With WORLD_SIZE unset or 1 it is a
    single process and every collective is the identity."""

    def __init__(self, backend: str = "nccl", timeout_s: float = 600.0):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self._dist = None
        if self.world > 1:
            import torch
            import torch.distributed as dist

            if backend == "nccl":
                torch.cuda.set_device(self.local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self._dist = dist
            self._torch = torch

    @property
    def distributed(self) -> bool:
        return self._dist is not None

    def _tensor(self, value: float):
        device = "cuda" if self.backend == "nccl" else "cpu"
        return self._torch.tensor([float(value)], dtype=self._torch.float64, device=device)

    def barrier(self) -> None:
        if self._dist:
            self._dist.barrier()

    def max(self, value: float) -> float:
        if not self._dist:
            return float(value)
        t = self._tensor(value)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, value: float) -> float:
        if not self._dist:
            return float(value)
        t = self._tensor(value)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.SUM)
        return float(t.item())

    def share(self, cases: Sequence[Any], cost: Callable[[Any], float] = wrap_cost) -> list[int]:
        """Indices of the cases this rank solves."""
        return assign([cost(c) for c in cases], self.world)[self.rank]

    def gather(self, mine: dict[int, Any]) -> list[Any] | None:
        """Rank 0 receives every rank's {index: result} and returns the results
        in index order; the other ranks return None."""
        if not self._dist:
            return [mine[i] for i in sorted(mine)]
        parts = [None] * self.world if self.rank == 0 else None
        self._dist.gather_object(mine, parts, dst=0)
        if self.rank != 0:
            return None
        merged: dict[int, Any] = {}
        for part in parts:
            merged.update(part)
        return [merged[i] for i in sorted(merged)]

    def close(self) -> None:
        if self._dist:
            self._dist.destroy_process_group()
            self._dist = None


def solve_replicated(group: ReplicaGroup, cases: Sequence[Any],
                     solve: Callable[[list[Any]], list[Any]],
                     cost: Callable[[Any], float] = wrap_cost) -> list[Any] | None:
    """Solves `cases` across the group: `solve` gets this rank's share (a list
    of cases, e.g. one batched launch) and returns one result per case.  Rank 0
    returns all results in submission order, the others None."""
    idx = group.share(cases, cost)
    results = solve([cases[i] for i in idx]) if idx else []
    if len(results) != len(idx):
        raise RuntimeError(f"solve returned {len(results)} results for {len(idx)} cases")
    return group.gather(dict(zip(idx, results)))
