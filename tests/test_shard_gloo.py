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


def _agg_rank(rank, world, port, queue):
    """One rank of a two-phase grouped aggregate: partial states of its own
    rows (the oracle stands in for the device's partial aggregate), the
    exchange by key owner, the merge of the states of the keys it owns."""
    import numpy as np
    import torch
    import torch.distributed as dist
    import oracle as O
    shard = importlib.import_module("krishiv-engine_b200.shard")
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        keys, x, y, yv = _agg_rows(rank)
        cols = [{"values": x, "type": O.T_I64}, {"values": y, "valid": yv.astype(np.uint8), "type": O.T_F64}]
        wk, _, wr = O.hash_aggregate(keys, None, cols, [(O.COUNT_STAR, 0), (O.SUM, 0), (O.MIN, 0), (O.MAX, 0),
                                                        (O.SUM, 1), (O.COUNT, 1)])
        state = [torch.tensor(wk), torch.tensor(wr[0]["i64"]), torch.tensor(wr[1]["i64"]), torch.tensor(wr[2]["i64"]),
                 torch.tensor(wr[3]["i64"]), torch.tensor(wr[4]["f64"]),
                 torch.tensor(wr[4]["valid"].astype(np.uint8)), torch.tensor(wr[5]["i64"])]
        owner = shard.key_owner(state[0], world)
        got = [t.numpy() for t in shard.exchange(dist, state, owner)]
        mine = bool((shard.key_owner(torch.tensor(got[0]), world) == rank).all())
        mcols = [{"values": got[1], "type": O.T_I64}, {"values": got[2], "type": O.T_I64},
                 {"values": got[3], "type": O.T_I64}, {"values": got[4], "type": O.T_I64},
                 {"values": got[5], "valid": got[6], "type": O.T_F64}, {"values": got[7], "type": O.T_I64}]
        mk, _, mr = O.hash_aggregate(got[0], None, mcols, [(O.SUM, 0), (O.SUM, 1), (O.MIN, 2), (O.MAX, 3),
                                                            (O.SUM, 4), (O.SUM, 5)])
        merged = {}
        for j, k in enumerate(mk.tolist()):
            sy = float(mr[4]["f64"][j]) if mr[4]["valid"][j] else None
            merged[k] = (int(mr[0]["i64"][j]), int(mr[1]["i64"][j]), int(mr[2]["i64"][j]), int(mr[3]["i64"][j]), sy,
                         int(mr[5]["i64"][j]))
        dist.barrier()
        queue.put((rank, merged, mine))
    finally:
        dist.destroy_process_group()


def _agg_rows(rank):
    import numpy as np
    rng = np.random.default_rng(100 + rank)
    n = 40_000
    keys = rng.integers(-3000, 3000, n).astype(np.int64)
    x = rng.integers(-10**12, 10**12, n).astype(np.int64)
    y = rng.random(n) * 200 - 100
    yv = rng.random(n) > 0.05
    return keys, x, y, yv


def test_two_phase_aggregate_exchange_on_two_gloo_ranks(oracle):
    """Partial states exchanged by key owner (shard.key_owner / exchange):
    every group is merged on exactly one rank, the rank that owns it, and the
    merged groups equal the one-phase aggregate of both ranks' rows."""
    import numpy as np
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_agg_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    # the results are read before the joins: a rank blocks on its put until
    # its (large) result is taken from the pipe
    got = sorted([q.get(timeout=240) for _ in procs], key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    assert all(mine for _, _, mine in got)
    assert not set(got[0][1]) & set(got[1][1])
    merged = {**got[0][1], **got[1][1]}
    rows = [_agg_rows(r) for r in range(2)]
    keys = np.concatenate([r[0] for r in rows])
    cols = [{"values": np.concatenate([r[1] for r in rows]), "type": oracle.T_I64},
            {"values": np.concatenate([r[2] for r in rows]), "valid": np.concatenate([r[3] for r in rows]).astype(np.uint8),
             "type": oracle.T_F64}]
    wk, _, wr = oracle.hash_aggregate(keys, None, cols, [(oracle.COUNT_STAR, 0), (oracle.SUM, 0), (oracle.MIN, 0),
                                                        (oracle.MAX, 0), (oracle.SUM, 1), (oracle.COUNT, 1)])
    assert len(merged) == len(wk)
    for j, k in enumerate(wk.tolist()):
        m = merged[k]
        assert m[:4] == (int(wr[0]["i64"][j]), int(wr[1]["i64"][j]), int(wr[2]["i64"][j]), int(wr[3]["i64"][j]))
        assert m[5] == int(wr[5]["i64"][j])
        if wr[4]["valid"][j]:
            assert rel_err(m[4], float(wr[4]["f64"][j])) <= 1e-12
        else:
            assert m[4] is None


def test_key_owner_is_balanced_and_stable():
    import torch
    shard = importlib.import_module("krishiv-engine_b200.shard")
    k = torch.arange(-50_000, 50_000, dtype=torch.int64)
    for world in (2, 3, 8):
        o = shard.key_owner(k, world)
        assert int(o.min()) == 0 and int(o.max()) == world - 1
        counts = torch.bincount(o, minlength=world).tolist()
        assert max(counts) - min(counts) < 0.05 * len(k) / world * world
        assert torch.equal(o, shard.key_owner(k.clone(), world))


def _join_rows(rank, n_build=20_000, n_probe=60_000):
    """One rank's own build rows (k, b) and probe rows (k, p): keys with
    duplicates and 2% NULLs, payloads that name the row uniquely."""
    import numpy as np
    rng = np.random.default_rng(300 + rank)
    bk = rng.integers(0, 30_000, n_build).astype(np.int64)
    bv = rng.random(n_build) > 0.02
    pk = rng.integers(0, 60_000, n_probe).astype(np.int64)
    pv = rng.random(n_probe) > 0.02
    b = np.arange(n_build, dtype=np.int64) + rank * 10**9
    p = np.arange(n_probe, dtype=np.int64) + rank * 10**9
    return bk, bv, b, pk, pv, p


def _join_output(oracle, jt, bk, bv, b, pk, pv, p):
    """The join's output rows (probe key or None, p, b or None) as a multiset
    (the oracle joins; the device's HashJoin gives the same rows)."""
    import collections
    pi, bi = oracle.hash_join(jt, [(bk, bv.astype("uint8"), False)],
                              [(pk, pv.astype("uint8"), False)])
    out = collections.Counter()
    for i, j in zip(pi.tolist(), bi.tolist()):
        out[(int(pk[i]) if pv[i] else None, int(p[i]), int(b[j]) if j >= 0 else None)] += 1
    return out


def _join_rank(rank, world, port, jt, queue):
    """One rank of a sharded hash join: its own rows of both sides, hashed by
    the join's row hash h (the oracle's restatement; krv_hash_rows_device on
    the device), exchanged by key owner, joined locally; and the union of the
    ranks' Bloom filters."""
    import numpy as np
    import torch
    import torch.distributed as dist
    import oracle as O
    shard = importlib.import_module("krishiv-engine_b200.shard")
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bk, bv, b, pk, pv, p = _join_rows(rank)
        hb = O.row_hash([(bk, bv.astype(np.uint8), False)]).view(np.int64)
        hp = O.row_hash([(pk, pv.astype(np.uint8), False)]).view(np.int64)
        rb, rbv, rp, rpv = shard.exchange_join_sides(
            dist, [torch.tensor(bk), torch.tensor(b)], torch.tensor(hb), torch.tensor(bv),
            [torch.tensor(pk), torch.tensor(p)], torch.tensor(hp), torch.tensor(pv))
        lbk, lb = rb[0].numpy(), rb[1].numpy()
        lpk, lp = rp[0].numpy(), rp[1].numpy()
        lbv, lpv = rbv.numpy(), rpv.numpy()
        # every non-NULL key landed on its owner
        own_b = shard.join_owner(torch.tensor(O.row_hash([(lbk, lbv.astype(np.uint8), False)]).view(np.int64)),
                                 torch.tensor(lbv), world, rank)
        own_p = shard.join_owner(torch.tensor(O.row_hash([(lpk, lpv.astype(np.uint8), False)]).view(np.int64)),
                                 torch.tensor(lpv), world, rank)
        mine = bool((own_b == rank).all()) and bool((own_p == rank).all())
        out = _join_output(O, jt, lbk, lbv, lb, lpk, lpv, lp)
        nbytes = O.bloom_bytes_for(40_000, 0.01)
        words = torch.tensor(O.bloom_build(O.xxh64_int(bk[bv]), nbytes).view(np.int32))
        union = shard.union_bloom(dist, words).numpy().view(np.uint32)
        dist.barrier()
        queue.put((rank, out, mine, union, len(lbk), len(lpk)))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
@pytest.mark.parametrize("jt", [0, 1])  # inner, left outer
def test_sharded_join_exchange_on_two_gloo_ranks(oracle, jt):
    """Both sides exchanged by the owner of their key hash, then joined on
    each rank: the union of the ranks' outputs is the one-rank join of all
    rows (NULL keys never match; left outer pads every unmatched probe row
    once), every key sits on its owner, and the OR of the ranks' Bloom words
    is the filter of all build keys."""
    import numpy as np
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    port = _free_port()
    procs = [ctx.Process(target=_join_rank, args=(r, 2, port, jt, q)) for r in range(2)]
    for p in procs:
        p.start()
    # read the results before joining: a result larger than the pipe's buffer
    # holds its rank in put() until it is read
    got = [q.get() for _ in range(2)]
    for p in procs:
        p.join(timeout=240)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    rows = [_join_rows(r) for r in range(2)]
    cat = [np.concatenate([rows[0][i], rows[1][i]]) for i in range(6)]
    want = _join_output(oracle, jt, *cat)
    total = got[0][1] + got[1][1]
    assert total == want
    assert all(g[2] for g in got)
    assert sum(g[4] for g in got) == len(cat[0]) and sum(g[5] for g in got) == len(cat[3])
    nbytes = oracle.bloom_bytes_for(40_000, 0.01)
    all_words = oracle.bloom_build(oracle.xxh64_int(cat[0][cat[1]]), nbytes)
    assert np.array_equal(got[0][3], all_words) and np.array_equal(got[1][3], all_words)


def test_join_owner_is_balanced_and_keeps_null_keys_local(oracle):
    """The owner of a row is the top bits of its key hash h scaled to the
    world size: every rank gets a near-equal share of distinct keys, equal
    keys one owner, and a NULL key stays on the rank that holds it."""
    import numpy as np
    import torch
    shard = importlib.import_module("krishiv-engine_b200.shard")
    rng = np.random.default_rng(3)
    keys = rng.integers(0, 1 << 40, 200_000).astype(np.int64)
    valid = rng.random(keys.size) > 0.01
    h = torch.tensor(oracle.row_hash([(keys, valid.astype(np.uint8), False)]).view(np.int64))
    for world in (2, 3, 8):
        o = shard.join_owner(h, torch.tensor(valid), world, rank=1)
        assert int(o.min()) >= 0 and int(o.max()) < world
        assert bool((o[~torch.tensor(valid)] == 1).all())
        counts = torch.bincount(o[torch.tensor(valid)], minlength=world).double()
        assert float(counts.max() / counts.min()) < 1.05
        dup = shard.join_owner(h[:1000].clone(), torch.tensor(valid[:1000]), world, rank=1)
        assert torch.equal(dup, o[:1000])
