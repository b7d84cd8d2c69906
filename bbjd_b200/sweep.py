"""sigma-sweep across GPUs: independent JDQZ solves, one process per GPU.

The reference's deployment runs one shift sigma per MPI rank with no
communication (reference README.md:59-83, include/bbjd.h:14-48); it ships
no driver.  This module partitions a list of solve items (pencil, sigma,
parameters) over ranks by estimated cost, runs each rank's share, and
gathers the results on every rank with one host-side all_gather at the end
(the only exchange: nothing flows between ranks while they solve).

    python -m torch.distributed.run --nproc-per-node N my_sweep.py

where my_sweep.py builds the items and calls :func:`run_sweep`.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Any, Callable, Sequence


@dataclass
class SweepItem:
    key: Any                 # caller's label (e.g. the sigma)
    n: int                   # problem size, for the cost estimate
    k: int                   # eigenpairs wanted
    payload: Any = None      # whatever the solve function needs
    cost: float = field(default=0.0)

    def estimate(self) -> float:
        # per outer iteration the device work is ~ n * maxsub; k sets how
        # many iterations are needed: cost ~ n * k
        return self.cost if self.cost > 0 else float(self.n) * max(1, self.k)


def partition(items: Sequence[SweepItem], world: int) -> list[list[int]]:
    """Longest-processing-time-first assignment of item indices to ranks.

    Deterministic: ties are broken by item index and by rank index, so every
    rank computes the same partition without communicating."""
    order = sorted(range(len(items)), key=lambda i: (-items[i].estimate(), i))
    loads = [0.0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda q: (loads[q], q))
        parts[r].append(i)
        loads[r] += items[i].estimate()
    for p in parts:
        p.sort()
    return parts


def run_sweep(items: Sequence[SweepItem], solve: Callable[[SweepItem], Any], rank: int = 0,
              world: int = 1, group=None) -> list[Any]:
    """Solve this rank's share of `items`; return every item's result, in
    item order, on every rank (one all_gather_object at the end when
    world > 1)."""
    parts = partition(items, world)
    mine = {i: solve(items[i]) for i in parts[rank]}
    if world == 1:
        return [mine[i] for i in range(len(items))]
    import torch.distributed as dist
    gathered: list[dict] = [None] * world  # type: ignore[list-item]
    dist.all_gather_object(gathered, mine, group=group)
    out: dict = {}
    for g in gathered:
        out.update(g)
    return [out[i] for i in range(len(items))]
