"""Many independent problems spread over processes, one GPU each.

The batched form (``Batch``, fvm2d_batch_* in include/fvm2d.h) advances
problems of mixed sizes, presets and end times in the same launches on one
GPU.  Across GPUs the problems share nothing, so they are dealt out whole:
no halo, no collective on the data path, weak scaling.  Each rank solves its
share as one batch; the results stay on the rank that computed them
(``results``) or are gathered to one rank (``gather``).

The deal depends on the problem list alone, so every rank computes the same
plan without communicating: problems are ordered by an estimate of their
cost, largest first, and each goes to the rank with the least estimated work
so far (longest processing time first; ties to the lower rank and the lower
problem index).  The estimate is cell-updates to the end time with a guessed
largest wave speed (the true one is known only while solving).
"""
from __future__ import annotations

import heapq

PARAMS = ("width", "height", "t_end", "cfl", "alpha", "gamma", "strategy")
DEFAULTS = dict(width=1.0, height=1.0, t_end=0.0, cfl=0.5, alpha=1.9, gamma=1.4, strategy=0)


def estimated_cost(nx: int, ny: int, width: float = 1.0, height: float = 1.0, t_end: float = 0.0,
                   cfl: float = 0.5, speed: float = 1.0) -> float:
    """Cell-updates to reach t_end: nx * ny cells times the steps of the
    reference's dt rule (dt = cfl * h / speed, h the smaller cell spacing)
    for a wave speed `speed`, at least one step."""
    h = min(width / nx, height / ny)
    return float(nx) * float(ny) * max(1.0, t_end * speed / (cfl * h))


def plan_shards(costs, world: int) -> list[list[int]]:
    """Problem indices of each of `world` ranks, each list in problem order."""
    if world < 1:
        raise ValueError("world size must be at least 1")
    heap = [(0.0, r) for r in range(world)]
    shards: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i)):
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(s) for s in shards]


def batch_solve(problems, precision: int):
    """Solves [(U, params)] as one batch on this process's current GPU and
    returns [(state (ny, nx, 4), t, steps)] in the same order."""
    from ._lib import Batch

    b = Batch([(U.shape[1], U.shape[0]) for U, _ in problems])
    try:
        b.set_precision(precision)
        for p, (U, kw) in enumerate(problems):
            b.set_problem(p, **{k: kw.get(k, DEFAULTS[k]) for k in PARAMS})
            b.set_state(p, U)
        b.solve()
        out = []
        for p in range(len(problems)):
            t, steps = b.time(p)
            out.append((b.get_state(p), t, steps))
        return out
    finally:
        b.close()


class EnsembleSolver:
    """This rank's share of a list of independent problems.

    ``problems`` is the whole list, the same on every rank: pairs (U, params)
    with U of shape (ny, nx, 4|5) and params a dict of the keys in PARAMS
    (missing keys take the solver defaults).  With ``torch.distributed``
    initialised the ranks of ``group`` (default: the world) split the list;
    without it one process solves everything.  ``solve`` is the function
    that solves one rank's share (default: one batch on the current GPU).
    """

    def __init__(self, problems, precision: int = 0, group=None, solve=batch_solve, speed: float = 1.0):
        import torch.distributed as dist

        self._dist = dist if (dist.is_available() and dist.is_initialized()) else None
        self.group = group
        self.rank = self._dist.get_rank(group) if self._dist else 0
        self.world = self._dist.get_world_size(group) if self._dist else 1
        self.problems = list(problems)
        self.precision = precision
        self._solve = solve
        costs = []
        for U, kw in self.problems:
            p = {k: kw.get(k, DEFAULTS[k]) for k in PARAMS}
            costs.append(estimated_cost(U.shape[1], U.shape[0], p["width"], p["height"], p["t_end"], p["cfl"],
                                        speed))
        self.plan = plan_shards(costs, self.world)
        self.mine = self.plan[self.rank]
        self.results: dict = {}

    def solve(self) -> int:
        """Solves this rank's problems; returns how many."""
        if self.mine:
            out = self._solve([self.problems[i] for i in self.mine], self.precision)
            self.results = dict(zip(self.mine, out))
        return len(self.mine)

    def gather(self, dst: int = 0):
        """Every problem's result, in problem order, on rank `dst` (None on
        the others).  The results travel pickled through the process group
        (with NCCL, the current CUDA device must be this rank's); for large
        ensembles, use ``results`` where they were computed instead."""
        if self._dist is None:
            return [self.results[i] for i in range(len(self.problems))]
        got = [None] * self.world if self.rank == dst else None
        self._dist.gather_object(self.results, got, dst=dst, group=self.group)
        if self.rank != dst:
            return None
        merged: dict = {}
        for part in got:
            merged.update(part)
        return [merged[i] for i in range(len(self.problems))]
