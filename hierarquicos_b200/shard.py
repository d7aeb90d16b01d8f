"""One system's force evaluation sharded over GPUs (one process per GPU).

Every rank builds the whole tree from the same bodies (the build is cheap next
to the walk), walks a contiguous range of the Morton-ordered target groups into
a zeroed output, and one sum all-reduce over NCCL combines the ranks' outputs:
every body's force is written by exactly one rank and added to zeros elsewhere,
so the result is bit for bit the single-GPU walk's.  The first split is even
by group count (groups hold at most 64 bodies, so the split of bodies is even
to within a group per rank).  Groups do not cost the same: in a centrally
concentrated system a group near the centre opens far more of the tree than
one in the halo, so an even count leaves the central ranks with most of the
walk.  ``Balancer`` therefore moves the boundaries after every evaluation:
each rank times its own walk, the times are all-gathered, and the new cut
points split the measured cost evenly, taking the cost to be spread uniformly
over each rank's previous range (``rebalance``).  The boundaries only change
which rank computes a body, never the body's result.
"""
from __future__ import annotations

import numpy as np
import torch

from ._lib import BHParams, default_params
from .system import BHSystem


def group_range(n_groups: int, rank: int, world: int) -> tuple[int, int]:
    """Groups [g0, g1) of `rank` among `world` ranks: contiguous, disjoint,
    covering [0, n_groups), sizes differing by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    base, extra = divmod(n_groups, world)
    g0 = rank * base + min(rank, extra)
    return g0, g0 + base + (1 if rank < extra else 0)


def rebalance(bounds, times) -> list[int]:
    """New cut points [0, b_1, ..., n_groups] from the previous ones and the
    measured cost (walk time) of every rank's range: the cumulative cost is
    interpolated linearly inside each range and cut into equal parts.  The
    result is contiguous, ordered and covers [0, n_groups); every rank that
    calls it with the same arguments gets the same cut points."""
    b = np.asarray(bounds, dtype=np.float64)
    t = np.maximum(np.asarray(times, dtype=np.float64), 0.0)
    world = t.size
    if b.size != world + 1 or b[0] != 0 or np.any(np.diff(b) < 0):
        raise ValueError("bounds must be world + 1 ordered cut points starting at 0")
    n_groups = int(b[-1])
    # a range with groups always has some cost, so the cumulative cost
    # increases strictly across non-empty ranges
    width = np.diff(b)
    t = np.where(width > 0, np.maximum(t, 1e-9 * max(float(t.max()), 1e-30) + 1e-300), 0.0)
    cum = np.concatenate([[0.0], np.cumsum(t)])
    keep = np.concatenate([[True], width > 0])
    xs, ys = cum[keep], b[keep]
    if xs[-1] <= 0.0:
        return [int(v) for v in bounds]
    cuts = np.rint(np.interp(xs[-1] * np.arange(1, world) / world, xs, ys)).astype(np.int64)
    cuts = np.clip(np.maximum.accumulate(cuts), 0, n_groups)
    return [0, *(int(c) for c in cuts), n_groups]


class Balancer:
    """Cut points of the target groups over the ranks, moved after every
    evaluation by the ranks' measured walk times (``rebalance``)."""

    def __init__(self, world: int):
        self.world = world
        self.bounds: list[int] | None = None

    def range(self, n_groups: int, rank: int) -> tuple[int, int]:
        if self.bounds is None or self.bounds[-1] != n_groups:
            self.bounds = [group_range(n_groups, r, self.world)[0] for r in range(self.world)]
            self.bounds.append(n_groups)
        return self.bounds[rank], self.bounds[rank + 1]

    def update(self, walk_ms: float, group=None) -> list[float]:
        """All-gathers every rank's walk time (all ranks call this with their
        own) and moves the cut points; returns the gathered times."""
        import torch.distributed as dist

        times = [float(walk_ms)]
        if dist.is_available() and dist.is_initialized() and self.world > 1:
            dev = torch.device("cuda", torch.cuda.current_device()) \
                if dist.get_backend(group) == "nccl" else torch.device("cpu")
            mine = torch.tensor([float(walk_ms)], dtype=torch.float64, device=dev)
            allt = [torch.zeros_like(mine) for _ in range(self.world)]
            dist.all_gather(allt, mine, group=group)
            times = [float(x.item()) for x in allt]
        if self.bounds is not None and len(times) == self.world:
            self.bounds = rebalance(self.bounds, times)
        return times


def combine(out: torch.Tensor, group=None) -> torch.Tensor:
    """Sum of the ranks' partial outputs, in place (a no-op on one rank)."""
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(out, op=dist.ReduceOp.SUM, group=group)
    return out


def sharded_forces(system: BHSystem, m, x, y, z, params: BHParams | None = None, out=None,
                   rank: int = 0, world: int = 1, group=None, balancer: Balancer | None = None,
                   **kw) -> torch.Tensor:
    """Build the whole system, walk this rank's share of the target groups and
    combine the shares: the (3N,) SoA forces in the original order on every
    rank.  With a ``balancer`` the share is its current range, and the walk is
    timed and the cut points moved for the next call."""
    p = params if params is not None else default_params(**kw)
    system.build(m, x, y, z, p)
    system.sync()  # the strict-key check may rebuild: settle the groups first
    n = system.n
    if out is None:
        out = torch.empty(3 * n, dtype=torch.float64, device=f"cuda:{system.device}")
    out.zero_()
    n_groups = system.info()["n_groups"]
    if balancer is None:
        g0, g1 = group_range(n_groups, rank, world)
        system.walk(p, out, groups=(g0, g1))
        system.sync()
        return combine(out, group)
    g0, g1 = balancer.range(n_groups, rank)
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record()
    system.walk(p, out, groups=(g0, g1))
    b.record()
    system.sync()
    b.synchronize()
    balancer.update(a.elapsed_time(b), group)
    return combine(out, group)
