"""Multi-GPU transitive closure by x-range partitioning.

In ``path(x, z) :- path(x, y), edge(y, z)`` the join output keeps the left x,
so the rows of path that start in a range of x values are derived only from
rows that start in the same range: each rank can close its own x range
against a replicated EDB with no exchange of relation rows. Every operator
(join, distinct, anti-join, union) stays partition-local; the global round
count is the largest per-rank count (ranks run the same rounds in lock step
in the reference, and a rank whose DELTA empties early would only run empty
rounds), and the new rows add up. One all-reduce at the end combines them.
"""

from __future__ import annotations

import numpy as np


def x_range(nodes: int, rank: int, world: int) -> tuple[int, int]:
    """The contiguous node range [lo, hi) owned by `rank`."""
    return nodes * rank // world, nodes * (rank + 1) // world


def balanced_bounds(src: np.ndarray, nodes: int, world: int) -> list[int]:
    """x boundaries [b_0 = 0, ..., b_world = nodes] that give every rank about
    the same number of seed rows (src sorted): for skewed graphs, where equal
    node ranges would give some ranks most of the work. Boundaries fall on x
    values, so no x is split between ranks."""
    n = len(src)
    bounds = [0]
    for r in range(1, world):
        k = n * r // world
        x = int(src[k]) if k < n else nodes
        bounds.append(max(bounds[-1], min(x, nodes)))
    bounds.append(nodes)
    return bounds


def partition_seed(src: np.ndarray, dst: np.ndarray, nodes: int, rank: int, world: int, balanced: bool = False):
    """Seed rows whose x lies in this rank's range (src must be sorted):
    equal node ranges, or with ``balanced`` the ranges of balanced_bounds."""
    if balanced:
        bounds = balanced_bounds(src, nodes, world)
        lo, hi = bounds[rank], bounds[rank + 1]
    else:
        lo, hi = x_range(nodes, rank, world)
    a = np.searchsorted(src, lo, side="left")
    b = np.searchsorted(src, hi, side="left")
    return src[a:b], dst[a:b]


def combine_summaries(iterations: int, new_rows: int, group=None, device=None) -> tuple[int, int]:
    """Global (iterations, new_rows): max and sum over ranks (one all-reduce each)."""
    import torch
    import torch.distributed as dist

    if group is None and not (dist.is_available() and dist.is_initialized()):
        return iterations, new_rows
    t = torch.tensor([iterations], dtype=torch.int64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    n = torch.tensor([new_rows], dtype=torch.int64, device=device)
    dist.all_reduce(n, op=dist.ReduceOp.SUM, group=group)
    return int(t.item()), int(n.item())
