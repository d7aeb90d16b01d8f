"""One system's force evaluation sharded over GPUs (one process per GPU).

Every rank builds the whole tree from the same bodies (the build is cheap next
to the walk), walks a contiguous range of the Morton-ordered target groups into
a zeroed output, and one sum all-reduce over NCCL combines the ranks' outputs:
every body's force is written by exactly one rank and added to zeros elsewhere,
so the result is bit for bit the single-GPU walk's.  The ranges split the
groups evenly by count (groups hold at most 64 bodies, so the split of bodies
is even to within a group per rank).
"""
from __future__ import annotations

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


def combine(out: torch.Tensor, group=None) -> torch.Tensor:
    """Sum of the ranks' partial outputs, in place (a no-op on one rank)."""
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(out, op=dist.ReduceOp.SUM, group=group)
    return out


def sharded_forces(system: BHSystem, m, x, y, z, params: BHParams | None = None, out=None,
                   rank: int = 0, world: int = 1, group=None, **kw) -> torch.Tensor:
    """Build the whole system, walk this rank's share of the target groups and
    combine the shares: the (3N,) SoA forces in the original order on every
    rank."""
    p = params if params is not None else default_params(**kw)
    system.build(m, x, y, z, p)
    system.sync()  # the strict-key check may rebuild: settle the groups first
    n = system.n
    if out is None:
        out = torch.empty(3 * n, dtype=torch.float64, device=f"cuda:{system.device}")
    out.zero_()
    n_groups = system.info()["n_groups"]
    g0, g1 = group_range(n_groups, rank, world)
    system.walk(p, out, groups=(g0, g1))
    system.sync()
    return combine(out, group)
