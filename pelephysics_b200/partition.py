"""Cells over GPUs: one process per GPU, contiguous cell ranges balanced by
cost, no data-path collective.

Cells are independent in react(), so a batch shards without any exchange
inside the integration.  The reference balances its boxes over MPI ranks
with the per-cell cost it writes to FC (the number of right-hand-side
evaluations, box_unflatten at Source/Reactions/ReactorUtils.H:289) through
AMReX's cost-weighted distribution mapping
(Testing/Exec/ReactEval/main.cpp:202-203); here the unit is a contiguous
range of the flat batch:

* ``balanced_ranges(cost, nranks)`` splits cells 0..n-1 into nranks
  contiguous ranges whose summed costs are as equal as the cell granularity
  allows (prefix sums cut at k * total / nranks); with no cost history the
  ranges are equal in cell count.
* ``ShardedReactor`` reacts the calling rank's range of a batch every rank
  holds (the caller's host or device arrays), then makes one int64 sum
  all-reduce of the counters (RHS evaluations, steps, failed cells; the
  reference reduces its timings the same way, main.cpp:682,720) and one sum
  all-reduce of the per-cell costs of the range, zero elsewhere, so that
  every rank plans the next call's ranges from the same costs.  The state
  itself never crosses ranks.

The collectives go through ``torch.distributed`` (NCCL between GPUs, gloo on
CPU); every rank makes the same collective calls in the same order.
"""

from __future__ import annotations

import numpy as np


def balanced_ranges(cost, nranks):
    """Contiguous [start, end) cell ranges, one per rank, whose summed costs
    are as equal as the cells allow.  cost: per-cell cost (>= 0) of the
    previous call; all zeros (no history) gives an equal split by cell
    count."""
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    cost = np.asarray(cost, dtype=np.float64).reshape(-1)
    n = cost.size
    if np.any(cost < 0) or not np.all(np.isfinite(cost)):
        raise ValueError("costs must be finite and >= 0")
    if not np.any(cost > 0):
        cuts = [(n * k) // nranks for k in range(nranks + 1)]
        return [(cuts[k], cuts[k + 1]) for k in range(nranks)]
    csum = np.concatenate([[0.0], np.cumsum(cost)])
    total = csum[-1]
    cuts = [0]
    for k in range(1, nranks):
        target = total * k / nranks
        # the first cell boundary whose prefix reaches the target, or the one
        # before it when that one is closer
        j = int(np.searchsorted(csum, target, side="left"))
        j = min(j, n)
        if j > 0 and abs(csum[j - 1] - target) <= abs(csum[j] - target):
            j -= 1
        cuts.append(max(j, cuts[-1]))
    cuts.append(n)
    return [(cuts[k], cuts[k + 1]) for k in range(nranks)]


class ShardedReactor:
    """One rank's share of a batch that every rank holds.

    reactor: this rank's reactor (pelephysics_b200.reactor.Reactor, or any
    object with the same react / cell_stats / cell_status methods); dist:
    torch.distributed (initialised) or None for one rank."""

    def __init__(self, reactor, ncells, dist=None, device="cpu"):
        self.r = reactor
        self.ncells = int(ncells)
        self.dist = dist
        self.device = device
        self.rank = dist.get_rank() if dist else 0
        self.world = dist.get_world_size() if dist else 1
        self.cost = np.zeros(self.ncells)
        self.ranges = balanced_ranges(self.cost, self.world)

    def react(self, rY, rYsrc, rX, rX_src, dt_react):
        """React this rank's range of the YCOrder batch in place; returns the
        batch totals summed over all ranks: (RHS evaluations, steps, failed
        cells), and the ranges used."""
        import torch

        a, b = self.ranges[self.rank]
        m = b - a
        nfe = steps = failed = 0
        local_cost = np.zeros(self.ncells, dtype=np.int64)
        if m > 0:
            self.r.react(rY[a:b], rYsrc[a:b], rX[a:b], rX_src[a:b], dt_react, raise_on_fail=False)
            st = self.r.cell_stats(m)
            status, cost = self.r.cell_status(m)
            nfe = int(np.asarray(st)[:, 1].sum())
            steps = int(np.asarray(st)[:, 0].sum())
            failed = int(np.sum(np.asarray(status) < 0))
            local_cost[a:b] = np.asarray(cost, dtype=np.int64)
        counters = torch.tensor([nfe, steps, failed], dtype=torch.int64, device=self.device)
        costs = torch.as_tensor(local_cost, device=self.device)
        if self.dist:
            self.dist.all_reduce(counters)  # sum
            self.dist.all_reduce(costs)
        used = list(self.ranges)
        self.cost = costs.cpu().numpy().astype(np.float64)
        self.ranges = balanced_ranges(self.cost, self.world)
        return tuple(int(v) for v in counters.cpu().tolist()), used
