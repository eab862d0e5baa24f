"""Batches of independent grids spread over the ranks of a job, one GPU per rank.

Grids of a batch share nothing, so the batch shards with no data exchange: every rank holds the same
list of grid specifications, computes the same cost-based partition of it, and projects only its own
grids (one ``BatchProjector`` per rank, i.e. one CUDA-graph launch per GPU).  The only collective is
the final gather of the per-grid scalars (max|div|, relative residual, steps) so that every rank can
report the whole batch.

Cost of a grid: cells x (expected refinement steps + 2).  The two extra units stand for the passes
every grid pays once per projection whatever its step count (the divergence, the gradient update and
the wavelet recovery: about two V-cycles of memory traffic).  The partition is the longest-processing-
time rule: grids in decreasing cost, each to the least loaded rank (ties to the lower rank, then the
lower grid index), which keeps the heaviest rank within one grid's cost of the mean load.

The reference runs one grid per process on device 0 and has no multi-GPU code; this module has no
reference counterpart.
"""
from __future__ import annotations

import math


def grid_cells(dim) -> int:
    return int(math.prod(int(v) for v in dim))


def expected_steps(rel_tol: float, rate: float = 0.1) -> int:
    """Refinement steps a grid is expected to need: the tolerance over a per-step residual reduction
    of `rate` (0.1 is what a V(2,2) step with trilinear prolongation gives on these problems)."""
    if not (0.0 < rel_tol < 1.0) or not (0.0 < rate < 1.0):
        raise ValueError("expected_steps: rel_tol and rate must lie in (0, 1)")
    return max(1, math.ceil(round(math.log(rel_tol) / math.log(rate), 9)))


def grid_cost(dim, steps: int) -> float:
    return float(grid_cells(dim)) * (int(steps) + 2)


def partition(costs, world: int) -> list[int]:
    """Rank of each grid: longest-processing-time assignment, deterministic (the same on every rank)."""
    if world < 1:
        raise ValueError("partition: world must be >= 1")
    costs = [float(c) for c in costs]
    if any(not (c >= 0.0) for c in costs):
        raise ValueError("partition: costs must be non-negative numbers")
    load = [0.0] * world
    owner = [0] * len(costs)
    for i in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        r = min(range(world), key=lambda j: (load[j], j))
        owner[i] = r
        load[r] += costs[i]
    return owner


def rank_loads(costs, owner, world: int) -> list[float]:
    load = [0.0] * world
    for c, r in zip(costs, owner):
        load[r] += float(c)
    return load


def gather_results(local: dict, count: int, world: int) -> list:
    """Every rank's {grid index: result} merged into one list in grid order, on every rank (a host
    gather of a few scalars per grid through torch.distributed; with world 1 no collective)."""
    parts = [local]
    if world > 1:
        import torch.distributed as dist
        parts = [None] * world
        dist.all_gather_object(parts, local)
    out = [None] * count
    for part in parts:
        for i, v in part.items():
            if out[i] is not None:
                raise RuntimeError(f"gather_results: grid {i} reported by two ranks")
            out[i] = v
    missing = [i for i, v in enumerate(out) if v is None]
    if missing:
        raise RuntimeError(f"gather_results: grids {missing} reported by no rank")
    return out


class ShardedBatch:
    """The grids of one batch spread over the ranks: ``grids`` (the same list on every rank, in the
    format of ``BatchProjector``) is partitioned by cost; this rank builds a ``BatchProjector`` over
    its share.  ``fields`` / ``outs`` passed to ``plan`` and ``run`` are this rank's, in the order of
    ``self.mine``.  ``results()`` returns the whole batch's per-grid scalars on every rank."""

    def __init__(self, grids, rank: int = 0, world: int = 1, rel_tol: float = 1e-6, steps=None, **kw):
        if not (0 <= rank < world):
            raise ValueError("ShardedBatch: need 0 <= rank < world")
        self.count = len(grids)
        self.rank, self.world = rank, world
        est = expected_steps(rel_tol) if steps is None else None
        self.costs = [grid_cost(g["dim"], est if steps is None else steps[i]) for i, g in enumerate(grids)]
        self.owner = partition(self.costs, world)
        self.mine = [i for i in range(self.count) if self.owner[i] == rank]
        self.bp = None
        if self.mine:
            from .api import BatchProjector
            self.bp = BatchProjector([grids[i] for i in self.mine], rel_tol=rel_tol, **kw)

    def plan(self, fields, stream=None):
        return self.bp.plan(fields, stream) if self.bp else []

    def run(self, fields, outs, stream=None):
        if self.bp:
            self.bp.run(fields, outs, stream)

    def local_results(self, stream=None) -> dict:
        """{grid index: per-grid scalars} for this rank's grids."""
        local = {}
        if self.bp:
            r = self.bp.results(stream)
            for k, i in enumerate(self.mine):
                local[i] = {"max_abs_div": r["max_abs_div"][k], "rel_residual": r["rel_residual"][k],
                            "cycles": r["cycles"][k], "over_tol": r["over_tol"][k], "rank": self.rank}
        return local

    def results(self, stream=None) -> list:
        return gather_results(self.local_results(stream), self.count, self.world)

    def close(self):
        if self.bp:
            self.bp.close()
            self.bp = None
