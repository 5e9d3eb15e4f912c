"""Host logic of a query run by several ranks, one process per GPU: which
fact rows a rank owns and how the ranks' partial results combine.

The star query shards by fact rows. Dimensions are replicated (every rank
builds the same tables and filters), each rank probes its own rows, and the
partial grouped sums merge once at the end: a gather of a few groups per
rank, no exchange on the data path."""
from __future__ import annotations

import math
from typing import Dict, List, Tuple

Groups = Dict[int, Tuple[float, int]]  # group -> (SUM, COUNT)


def weak_shard(rows_per_rank: int, rank: int) -> Tuple[int, int]:
    """Rows [row0, row0 + rows) of a rank when every rank keeps the same
    number of rows (weak scaling: the job grows with the ranks)."""
    return rank * rows_per_rank, rows_per_rank


def strong_shard(total: int, rank: int, world: int) -> Tuple[int, int]:
    """Rows [row0, row0 + rows) of a rank when `total` rows split as evenly
    as they can (the first total % world ranks take one row more)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank out of range")
    base, extra = divmod(total, world)
    row0 = rank * base + min(rank, extra)
    return row0, base + (1 if rank < extra else 0)


def merge_groups(partials: List[Groups]) -> Groups:
    """Combines per-rank grouped (SUM, COUNT) results: counts add, sums are
    summed with one correctly rounded addition (math.fsum) per group."""
    keys = sorted({g for p in partials for g in p})
    out: Groups = {}
    for g in keys:
        parts = [p[g] for p in partials if g in p]
        out[g] = (math.fsum(s for s, _ in parts), sum(c for _, c in parts))
    return out


def all_merge_groups(dist, partial: Groups) -> Groups:
    """Gathers every rank's partial groups (torch.distributed) and merges
    them; every rank returns the same merged result."""
    world = dist.get_world_size()
    got: List[Groups] = [None] * world
    dist.all_gather_object(got, partial)
    return merge_groups(got)


def max_over_ranks(dist, value: float, device="cpu") -> float:
    """The largest `value` over the ranks (timings: the job ends with its
    slowest rank). `dist` None means one rank."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
