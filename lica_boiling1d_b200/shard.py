"""Sharding of independent work over ranks (one process per GPU).

The columns of a batch never exchange data, so the ranks take contiguous blocks of the
column list balanced by cells (a column step's work grows with its cells), step their
block with no collective, and gather the per-column histories once at the end.  The bubble
statistics of several level sets shard the same way: each rank tracks a contiguous block of
the level sets (equal work: every level set reads one field) and the records are gathered.
"""
import numpy as np


def partition(cells, world):
    """Contiguous blocks [lo, hi) of the column list, one per rank, whose cell totals are
    as close to total / world as the column boundaries allow."""
    cells = np.asarray(cells, dtype=np.int64)
    if world < 1:
        raise ValueError("world must be >= 1")
    cum = np.concatenate([[0], np.cumsum(cells)])
    total = int(cum[-1])
    bounds = [0]
    for r in range(1, world):
        target = total * r / world
        k = int(np.searchsorted(cum, target))
        if 0 < k <= len(cells) and abs(cum[k - 1] - target) <= abs(cum[k] - target):
            k -= 1
        bounds.append(min(max(bounds[-1], k), len(cells)))
    bounds.append(len(cells))
    return [(bounds[r], bounds[r + 1]) for r in range(world)]


def gather_histories(local, world, group=None):
    """The ranks' per-column records concatenated in rank order, on every rank (one
    all_gather at the end of a run; nothing is exchanged per step)."""
    if world == 1:
        return list(local)
    import torch.distributed as dist
    parts = [None] * world
    dist.all_gather_object(parts, list(local), group=group)
    return [rec for part in parts for rec in part]


def gather_records(local, world, group=None):
    """The ranks' structured-array records (e.g. bubbles.RECORD) concatenated in rank order,
    on every rank (one all_gather)."""
    if world == 1:
        return np.asarray(local)
    import torch.distributed as dist
    parts = [None] * world
    dist.all_gather_object(parts, np.asarray(local), group=group)
    return np.concatenate(parts)
