"""Host-side plumbing for batched replicas on several GPUs (one process per
GPU): the replicas of one ensemble are independent, so they are dealt to the
ranks by balanced site count and stepped with no exchange at all; the only
collective is an all-gather of per-replica scalars at the end of a run.

DASH runs one State per process and has no counterpart; this follows the
batched form's own design (every replica a full TIP4P/2005 box of its own).
"""
from __future__ import annotations

from typing import List, Sequence


def shard_by_sites(sites: Sequence[int], world: int) -> List[List[int]]:
    """Deal replica indices to `world` ranks so that the site totals are
    balanced: longest-processing-time greedy (largest replica first, to the
    rank with the smallest total so far; ties go to the lower rank, equal
    sizes in index order), deterministic on every rank.  Each rank's list is
    returned in increasing replica index."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(sites)), key=lambda r: (-int(sites[r]), r))
    load = [0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for r in order:
        k = min(range(world), key=lambda w: (load[w], w))
        out[k].append(r)
        load[k] += int(sites[r])
    return [sorted(x) for x in out]


def gather_replica_scalars(dist, mine: Sequence[int], values: Sequence[float], total: int, device=None):
    """All-gather one float per replica: rank k holds `values` for its replica
    indices `mine`; every rank gets the list of all `total` values in replica
    order.  dist may be None (one process)."""
    import torch

    full = torch.zeros(total, dtype=torch.float64, device=device)
    for r, v in zip(mine, values):
        full[r] = float(v)
    if dist is not None:
        # each replica is owned by exactly one rank: a sum is the gather
        dist.all_reduce(full)
    return [float(v) for v in full.cpu().tolist()]
