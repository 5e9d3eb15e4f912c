"""The partitioned (grace) hash join against the CPU oracle and the
unpartitioned join: the output multiset is exact for left outer and inner
joins with NULL keys, heavy probe keys and duplicate build keys, whether the
partitions stay in HBM, spill to host memory, or spill and split again; a
partition of one key that cannot fit joins by the fallback (the build side in
groups that fit, probe rows padded once no group matched them) and gives the
oracle's rows, where the reference falls back to a sort-merge join
(crates/krishiv-exec/src/join/fallback.rs, started at join/grace.rs:1006-1013)."""
import collections

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def make(seed=7, nb=60_000, np_=240_000, dom=120_000, heavy=20):
    rng = np.random.default_rng(seed)
    bk = rng.integers(0, dom, nb).astype(np.int64)
    bval = rng.random(nb) > 0.01
    b1 = rng.integers(-(2**62), 2**62, nb).astype(np.int64)
    b2 = rng.integers(-(2**62), 2**62, nb).astype(np.int64)
    hk = rng.integers(0, dom, heavy)
    pk = np.where(rng.random(np_) < 0.1, hk[rng.integers(0, heavy, np_)], rng.integers(0, dom, np_)).astype(np.int64)
    pval = rng.random(np_) > 0.01
    pp = rng.integers(-(2**62), 2**62, np_).astype(np.int64)
    return (bk, bval, b1, b2), (pk, pval, pp)


def dev(kb, cols):
    import torch
    out = []
    for name, a, valid in cols:
        v = None
        if valid is not None:
            bits = np.concatenate([np.packbits(valid.astype(np.uint8), bitorder="little"), np.zeros(8, np.uint8)])
            v = torch.tensor(bits, device="cuda")
        out.append((name, torch.tensor(a, device="cuda"), v))
    return kb.DeviceBatch(out)


def rows_of(res):
    """(k or None, p, b1 or None, b2 or None) per output row."""
    if res.rows == 0:
        return []
    cols = [c.cpu().numpy() for c in res.columns]
    valid = []
    for i, v in enumerate(res.valid):
        if v is None:
            valid.append(np.ones(res.rows, bool))
        else:
            bits = np.unpackbits(v.cpu().numpy(), bitorder="little")[: res.rows]
            valid.append(bits.astype(bool))
    return [tuple(int(cols[c][i]) if valid[c][i] else None for c in range(len(cols))) for i in range(res.rows)]


def run(kb, rt, build, probe, jt, partitioned, budget=0, radix=3, batches=3, max_out=50_000, filter_bits=None):
    bk, bval, b1, b2 = build
    pk, pval, pp = probe
    spec = kb.join_spec(jt, probe_keys=(0,), build_keys=(0,), probe_out=[0, 1], build_out=[1, 2], radix_bits=radix,
                        max_output_rows=max_out)
    j = kb.HashJoin(rt, spec, partitioned=partitioned, device_budget=budget,
                    probe_filter_bits=filter_bits if partitioned else None)
    keep = []
    for s in np.array_split(np.arange(bk.size), batches):
        db = dev(kb, [("k", bk[s], bval[s]), ("p1", b1[s], None), ("p2", b2[s], None)])
        keep.append(db)
        j.build_push_device(db)
    j.build_finish()
    got = []
    for s in np.array_split(np.arange(pk.size), batches):
        db = dev(kb, [("k", pk[s], pval[s]), ("p", pp[s], None)])
        keep.append(db)
        for r in j.probe_device_all(db):
            got += rows_of(r)
    for r in j.finish_device():
        got += rows_of(r)
    return collections.Counter(got), j


def oracle_rows(oracle, build, probe, jt):
    bk, bval, b1, b2 = build
    pk, pval, pp = probe
    pi, bi = oracle.hash_join({"inner": 0, "left_outer": 1}[jt], [(bk, bval.astype(np.uint8))],
                              [(pk, pval.astype(np.uint8))])
    out = []
    for i, b in zip(pi.tolist(), bi.tolist()):
        k = int(pk[i]) if pval[i] else None
        out.append((k, int(pp[i]), int(b1[b]) if b >= 0 else None, int(b2[b]) if b >= 0 else None))
    return collections.Counter(out)


@pytest.mark.parametrize("filter_bits", [None, 0])
@pytest.mark.parametrize("jt", ["left_outer", "inner"])
@pytest.mark.parametrize("budget", [0, 2 << 20, 256 << 10])
def test_partitioned_join_matches_the_oracle(kb, rt, oracle, jt, budget, filter_bits):
    """budget 0: every partition resident; 2 MiB: some spill (and rows of
    resident partitions are deferred once a call's output reaches its cap);
    256 KiB: all spill and split again at finish. With the Bloom filter of
    the partition pass (the default) and without it (0 bits)."""
    build, probe = make()
    got, j = run(kb, rt, build, probe, jt, True, budget=budget, filter_bits=filter_bits)
    want = oracle_rows(oracle, build, probe, jt)
    assert got == want
    c = j.counters()
    assert c["output_rows"] == sum(want.values())
    # about 60% of the probe rows have a key no build row holds
    filtered = j.filtered_probe_rows()
    if filter_bits == 0:
        assert filtered == 0
    elif budget == 0:
        bk, bval = build[0], build[1]
        pk, pval = probe[0], probe[1]
        absent = int((pval & ~np.isin(pk, bk[bval])).sum())
        assert 0.5 * absent < filtered <= absent  # no false negatives: only absent keys are ruled out
    if budget == 256 << 10:
        assert j.spilled_partitions() == 8 and c["partitions"] > 8  # spilled, then split
    if budget == 0:
        assert j.spilled_partitions() == 0
    if budget == 2 << 20:
        assert 0 < j.spilled_partitions() < 8


def test_partitioned_equals_unpartitioned(kb, rt):
    build, probe = make(seed=3, nb=100_000, np_=300_000, dom=150_000)
    a, _ = run(kb, rt, build, probe, "left_outer", True, budget=4 << 20, radix=5)
    b, _ = run(kb, rt, build, probe, "left_outer", False)
    assert a == b


@pytest.mark.parametrize("jt", ["left_outer", "inner"])
def test_one_heavy_build_key_that_cannot_fit(kb, rt, oracle, jt):
    """50,000 build rows of one key under a 256 KiB budget: no split can shrink
    that partition, so it joins by the fallback; the output is the oracle's
    (every probe row of the key pairs with all 50,000 rows, the others are
    padded or dropped)."""
    n = 50_000
    rng = np.random.default_rng(3)
    build = (np.full(n, 42, np.int64), np.ones(n, bool), np.arange(n, dtype=np.int64),
             rng.integers(-(2**62), 2**62, n).astype(np.int64))
    pk = np.array([42, 7, 42, 9, 42] * 3, np.int64)
    probe = (pk, np.ones(pk.size, bool), np.arange(pk.size, dtype=np.int64))
    got, j = run(kb, rt, build, probe, jt, True, budget=256 << 10, batches=1)
    want = oracle_rows(oracle, build, probe, jt)
    assert got == want
    assert sum(got.values()) == 9 * n + (6 if jt == "left_outer" else 0)
