"""Host logic of a query run by several ranks, one process per GPU: which
fact rows a rank owns and how the ranks' partial results combine.

The star query shards by fact rows. Dimensions are replicated (every rank
builds the same tables and filters), each rank probes its own rows, and the
partial grouped sums merge once at the end: a gather of a few groups per
rank, no exchange on the data path.

A grouped aggregate with many groups has a real exchange step: each rank
aggregates its own rows into partial states (krv_agg with
KRV_AGG_OUTPUT_PARTIAL), `exchange` sends every state row to the rank that
owns its key (`key_owner`) with one all-to-all per column (NCCL over NVLink
for device tensors, gloo for host tensors), and each rank merges the states
of the keys it owns (KRV_AGG_INPUT_STATE): every group ends on exactly one
rank.

A hash join whose both sides are sharded exchanges both sides by key
(`join_owner`, `exchange_join_sides`): the top bits of the join's own row
hash h (the bits the reference's level-0 partition takes,
crates/krishiv-exec/src/join/keys.rs:118-128; `krv_hash_rows_device` gives
them on the device) choose the owning rank, one all-to-all per column moves
each side's rows there, and every rank then builds and probes its own rows:
equal keys meet on one rank, so every output row (padded outer rows
included) is made exactly once. Rows whose key is NULL match nothing and
stay where they are. The ranks' runtime key filters combine by a bitwise OR
of their Bloom words (`union_bloom`, RuntimeBloom::union_with,
crates/krishiv-io/src/runtime_filter/bloom.rs:153)."""
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


_MASK32 = (1 << 32) - 1


def _shr(z, s: int):
    """Logical right shift of an int64 tensor (its bits as unsigned)."""
    return (z >> s) & ((1 << (64 - s)) - 1)


def key_owner(keys, world: int):
    """The rank owning each int64 key's group: the top 32 bits of a
    SplitMix64 finalisation of the key, scaled to `world` (any mixing
    function would do: owners only decide where a group is merged, never its
    result). `keys` is an int64 torch tensor on any device."""
    import torch
    z = keys.to(torch.int64)
    z = (z ^ _shr(z, 30)) * -4658895280553007687   # 0xbf58476d1ce4e5b9
    z = (z ^ _shr(z, 27)) * -7723592293110705685   # 0x94d049bb133111eb
    z = z ^ _shr(z, 31)
    return (_shr(z, 32) * world) >> 32


def exchange(dist, columns, owner):
    """Sends row i of every column (equal-length torch tensors, one device)
    to rank owner[i]; returns this rank's received rows of every column,
    grouped by sending rank in rank order. One all_to_all_single for the
    counts, one per column."""
    import torch
    world = dist.get_world_size()
    owner = owner.to(torch.int64)
    order = torch.argsort(owner, stable=True)
    send = torch.bincount(owner, minlength=world).to(torch.int64)
    recv = torch.empty_like(send)
    dist.all_to_all_single(recv, send)
    send_l, recv_l = send.tolist(), recv.tolist()
    out = []
    for c in columns:
        src = c[order].contiguous()
        dst = torch.empty((sum(recv_l),) + tuple(c.shape[1:]), dtype=c.dtype, device=c.device)
        dist.all_to_all_single(dst, src, recv_l, send_l)
        out.append(dst)
    return out


def join_owner(h, key_valid, world: int, rank: int):
    """The rank that joins each row: the top 32 bits of its key hash `h`
    (int64 tensor holding the uint64 h) scaled to `world`; a row whose key is
    NULL (`key_valid` False; None: no NULLs) stays on `rank`."""
    import torch
    owner = (_shr(h.to(torch.int64), 32) * world) >> 32
    if key_valid is not None:
        owner = torch.where(key_valid.to(torch.bool), owner, torch.full_like(owner, rank))
    return owner


def exchange_join_sides(dist, build_columns, build_h, build_valid, probe_columns, probe_h, probe_valid):
    """Both sides of a sharded hash join moved to the ranks that own their
    keys (one `exchange` per side): returns (build columns, build key
    validity, probe columns, probe key validity) of this rank. Validity
    tensors (bool, or None for no NULLs) travel with their rows."""
    import torch
    world, rank = dist.get_world_size(), dist.get_rank()
    out = []
    for cols, h, valid in ((build_columns, build_h, build_valid), (probe_columns, probe_h, probe_valid)):
        owner = join_owner(h, valid, world, rank)
        extra = [valid.to(torch.uint8)] if valid is not None else []
        moved = exchange(dist, list(cols) + extra, owner)
        if valid is not None:
            out += [moved[:-1], moved[-1].to(torch.bool)]
        else:
            out += [moved, None]
    return tuple(out)


def union_bloom(dist, words):
    """The bitwise OR of every rank's Bloom words (equal-length integer
    tensors): the filter of all ranks' keys. An all-gather and a local OR,
    so that it runs on NCCL (which has no bitwise reduction) as on gloo."""
    import torch
    world = dist.get_world_size()
    got = [torch.empty_like(words) for _ in range(world)]
    dist.all_gather(got, words)
    acc = got[0].clone()
    for g in got[1:]:
        acc |= g
    return acc
