"""The multi-rank host logic on the CPU: two `gloo` ranks each run the star
query (CPU oracle) over their own fact rows against replicated dimensions,
merge their partial group sums, and agree with the one-rank answer within
1e-12 relative; the max-over-ranks timing and the shard arithmetic."""
import datetime
import importlib
import os
import socket

import pytest

from helpers import rel_err

SEED = 0x4B52560003
SCALE = 0.002  # fact 600,000 rows, dimensions 40,000 / 2,000


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, total, queue):
    import torch.distributed as dist
    import oracle as O
    shard = importlib.import_module("krishiv-engine_b200.shard")
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        row0, rows = shard.strong_shard(total, rank, world)
        fact, dims = O.star_inputs(SCALE, SEED, fact_row0=row0, fact_rows=rows)
        partial, passed, joined, _, _ = O.star_query(fact, dims)
        merged = shard.all_merge_groups(dist, partial)
        slowest = shard.max_over_ranks(dist, float(10 + rank))
        counts = [None] * world
        dist.all_gather_object(counts, (passed, joined, rows))
        dist.barrier()
        queue.put((rank, merged, slowest, counts))
    finally:
        dist.destroy_process_group()


def test_strong_and_weak_shards_cover_the_rows():
    shard = importlib.import_module("krishiv-engine_b200.shard")
    for total, world in ((10, 3), (600_001, 2), (5, 8), (0, 4)):
        spans = [shard.strong_shard(total, r, world) for r in range(world)]
        assert sum(n for _, n in spans) == total
        pos = 0
        for row0, n in spans:
            assert row0 == pos
            pos += n
        assert max(n for _, n in spans) - min(n for _, n in spans) <= 1
    assert [shard.weak_shard(100, r) for r in range(3)] == [(0, 100), (100, 100), (200, 100)]
    with pytest.raises(ValueError):
        shard.strong_shard(10, 2, 2)


def test_merge_groups_is_exactly_rounded():
    shard = importlib.import_module("krishiv-engine_b200.shard")
    a = {1: (1e16, 1), 2: (0.5, 2)}
    b = {1: (1.0, 1), 3: (-2.0, 1)}
    c = {1: (-1e16, 1)}
    m = shard.merge_groups([a, b, c])
    assert m == {1: (1.0, 3), 2: (0.5, 2), 3: (-2.0, 1)}


def test_two_gloo_ranks_match_one(oracle):
    import torch.multiprocessing as mp
    total = int(300_000_000 * SCALE)
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, total, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted([q.get() for _ in procs], key=lambda x: x[0])
    fact, dims = oracle.star_inputs(SCALE, SEED)
    want, passed, joined, _, _ = oracle.star_query(fact, dims)
    for rank, merged, slowest, counts in got:
        assert slowest == 11.0
        assert sum(c[2] for c in counts) == total
        assert sum(c[0] for c in counts) == passed and sum(c[1] for c in counts) == joined
        assert sorted(merged) == sorted(want)
        for g, (s, n) in want.items():
            assert merged[g][1] == n
            assert rel_err(merged[g][0], s) <= 1e-12
