"""GPU hash join parity against the CPU oracle (the reference's join semantics
restated in oracle/krv_oracle.c), through the C ABI. Results are compared as
multisets of (probe row, build row) pairs, which is bit-exact for this
integer work."""
import collections

import numpy as np
import pyarrow as pa
import pytest

from helpers import batch, concat, pairs_from_output

pytestmark = pytest.mark.gpu

TYPES = ["inner", "left_outer", "left_semi", "left_anti", "null_aware_anti", "existence", "right_semi",
         "right_anti", "right_outer", "full_outer"]
TYPE_ID = {n: i for i, n in enumerate(TYPES)}

EDGE_PROBE = [(1, 10), (1, 10), (2, None), (None, 10), (None, None), (7, 70)]
EDGE_BUILD = [(1, 10), (1, 10), (1, 11), (2, None), (None, None), (None, 10)]
ALL_NULL = [(None, None), (None, None)]


def rows_batch(rows, idname):
    k1 = pa.array([r[0] for r in rows], type=pa.int64())
    k2 = pa.array([r[1] for r in rows], type=pa.int32())
    return batch(k1=k1, k2=k2, **{idname: pa.array(np.arange(len(rows), dtype=np.int64))})


def oracle_pairs(oracle, jt, probe, build, nkeys, null_safe):
    def cols(rows):
        out = []
        for k in range(nkeys):
            dt = np.int64 if k == 0 else np.int32
            v = np.array([r[k] if r[k] is not None else 0 for r in rows], dtype=dt)
            m = np.array([r[k] is not None for r in rows], dtype=np.uint8)
            out.append((v, m, False))
        return out
    p, b = oracle.hash_join(TYPE_ID[jt], cols(build), cols(probe), null_safe=[int(null_safe)] * nkeys)
    return collections.Counter(zip(p.tolist(), b.tolist()))


def gpu_pairs(kb, rt, jt, probe, build, nkeys, null_safe, build_batches=1, max_out=0):
    spec = kb.join_spec(jt, probe_keys=tuple(range(nkeys)), build_keys=tuple(range(nkeys)),
                        null_safe=[null_safe] * nkeys, max_output_rows=max_out)
    j = kb.HashJoin(rt, spec)
    b = rows_batch(build, "bid")
    step = max(1, -(-len(build) // build_batches))
    if len(build) == 0:
        j.build_push(b)
    for s in range(0, len(build), step):
        j.build_push(b.slice(s, step))
    j.build_finish()
    outs = j.probe(rows_batch(probe, "pid"))
    outs += j.finish()
    t = concat(outs)
    if jt == "existence":
        return collections.Counter(zip(t.column("pid").to_pylist(), [int(x) for x in t.column("exists").to_pylist()]))
    return pairs_from_output(t)


@pytest.mark.parametrize("jt", TYPES)
def test_join_types_edge_cases(kb, rt, oracle, jt):
    # tests/hash_join/main.rs:243-299: NULLs, duplicates, empty and all-NULL
    # inputs, `=` and `<=>` keys, one and two key columns.
    inputs = [(EDGE_PROBE, EDGE_BUILD), (EDGE_PROBE, []), ([], EDGE_BUILD), (EDGE_PROBE, ALL_NULL),
              (ALL_NULL, EDGE_BUILD)]
    for nkeys in (1, 2):
        for safe in (False, True):
            if jt == "null_aware_anti" and (nkeys > 1 or safe):
                continue
            for probe, build in inputs:
                want = oracle_pairs(oracle, jt, probe, build, nkeys, safe)
                got = gpu_pairs(kb, rt, jt, probe, build, nkeys, safe)
                assert got == want, (jt, nkeys, safe, len(probe), len(build))


@pytest.mark.parametrize("jt", TYPES)
def test_join_types_random_duplicates(kb, rt, oracle, jt):
    rng = np.random.default_rng(11)
    probe = [(int(x) if x >= 0 else None, int(y)) for x, y in zip(rng.integers(-20, 3000, 20000),
                                                                   rng.integers(0, 3, 20000))]
    build = [(int(x) if x >= 0 else None, int(y)) for x, y in zip(rng.integers(-20, 3000, 9000),
                                                                   rng.integers(0, 3, 9000))]
    for nkeys in ((1,) if jt == "null_aware_anti" else (1, 2)):
        want = oracle_pairs(oracle, jt, probe, build, nkeys, False)
        got = gpu_pairs(kb, rt, jt, probe, build, nkeys, False, build_batches=3)
        assert got == want, (jt, nkeys)


def test_output_bound_and_multi_batch_build(kb, rt, oracle):
    rng = np.random.default_rng(12)
    probe = [(int(x), 0) for x in rng.integers(0, 50, 5000)]
    build = [(int(x), 0) for x in rng.integers(0, 50, 400)]
    want = oracle_pairs(oracle, "inner", probe, build, 1, False)
    got = gpu_pairs(kb, rt, "inner", probe, build, 1, False, build_batches=7, max_out=1000)
    assert got == want


def test_single_match_error(kb, rt):
    spec = kb.join_spec("left_outer", single_match=True)
    j = kb.HashJoin(rt, spec)
    j.build_push(rows_batch([(1, 0), (1, 0), (2, 0)], "bid"))
    j.build_finish()
    assert len(j.probe(rows_batch([(2, 0), (3, 0)], "pid"))[0]) == 2
    with pytest.raises(kb.KrvError) as e:
        j.probe(rows_batch([(1, 0)], "pid"))
    assert e.value.status == kb.TOO_MANY_ROWS


def test_residual_filter_flag_needs_a_filter(kb, rt):
    """has_residual_filter without krv_join_set_filter is an error at the first
    probe; a null-aware anti join takes no residual condition (the reference
    rejects that combination, join/mod.rs:746-752)."""
    spec = kb.join_spec("inner")
    spec.has_residual_filter = 1
    j = kb.HashJoin(rt, spec)
    j.build_push(rows_batch([(1, 0)], "bid"))
    j.build_finish()
    with pytest.raises(kb.KrvError) as e:
        j.probe(rows_batch([(1, 0)], "pid"))
    assert e.value.status == kb.INVALID_ARGUMENT
    spec = kb.join_spec("null_aware_anti")
    spec.has_residual_filter = 1
    with pytest.raises(kb.KrvError) as e:
        kb.HashJoin(rt, spec)
    assert e.value.status == kb.UNSUPPORTED
    with pytest.raises(kb.KrvError) as e:
        kb.HashJoin(rt, kb.join_spec("null_aware_anti"), filter=[(("probe", 1), "<", ("build", 1))])
    assert e.value.status == kb.UNSUPPORTED


def test_float_and_decimal_keys(kb, rt, oracle):
    # float keys normalize -0.0/NaN (rows/layout.rs:1147-1149); decimal128 keys hash both words
    f_build = np.array([0.0, -0.0, np.nan, 1.5, 2.5], dtype=np.float64)
    f_probe = np.array([-0.0, np.nan, 1.5, 3.0], dtype=np.float64)
    j = kb.HashJoin(rt, kb.join_spec("inner"))
    j.build_push(batch(k=pa.array(f_build), bid=pa.array(np.arange(5, dtype=np.int64))))
    j.build_finish()
    got = pairs_from_output(concat(j.probe(batch(k=pa.array(f_probe), pid=pa.array(np.arange(4, dtype=np.int64))))))
    p, b = oracle.hash_join(0, [(f_build, None, True)], [(f_probe, None, True)])
    assert got == collections.Counter(zip(p.tolist(), b.tolist()))
    dec = pa.array([1, -1, 10**20, 5], type=pa.decimal128(30, 2))
    j = kb.HashJoin(rt, kb.join_spec("inner"))
    j.build_push(batch(k=dec, bid=pa.array(np.arange(4, dtype=np.int64))))
    j.build_finish()
    got = pairs_from_output(concat(j.probe(batch(k=pa.array([10**20, 1, 7], type=pa.decimal128(30, 2)),
                                                 pid=pa.array(np.arange(3, dtype=np.int64))))))
    assert got == collections.Counter({(0, 2): 1, (1, 0): 1})


def test_plain_inner_join_shape(kb, rt, oracle):
    """The plain inner join of the reference's CPU-operator workload at a
    tenth of its size: build k = a permutation of 0..n-1 with an int64
    payload, probe keys uniform over twice the range (about half match) with
    an int32 payload; output (k, v, w) compared as a sorted multiset."""
    nb, np_ = 100_000, 1_000_000
    rng = np.random.default_rng(13)
    bk = rng.permutation(nb).astype(np.int64)
    bv = rng.integers(-2**62, 2**62, nb, dtype=np.int64)
    pk = rng.integers(0, 2 * nb, np_, dtype=np.int64)
    pw = rng.integers(-2**31, 2**31 - 1, np_, dtype=np.int64).astype(np.int32)
    spec = kb.join_spec("inner", probe_out=[0, 1], build_out=[1])
    j = kb.HashJoin(rt, spec)
    for s in range(0, nb, 8192):
        j.build_push(batch(k=pa.array(bk[s:s + 8192]), v=pa.array(bv[s:s + 8192])))
    j.build_finish()
    out = concat(j.probe(batch(k=pa.array(pk), w=pa.array(pw))))
    got = np.stack([out.column("k").to_numpy(), out.column("v").to_numpy(), out.column("w").to_numpy().astype(np.int64)], 1)
    p, b = oracle.hash_join(0, [(bk, None, False)], [(pk, None, False)])
    want = np.stack([pk[p], bv[b], pw[p].astype(np.int64)], 1)
    got = got[np.lexsort(got.T[::-1])]
    want = want[np.lexsort(want.T[::-1])]
    assert np.array_equal(got, want)
    c = j.counters()
    assert c["build_rows"] == nb and c["build_keys"] == nb and c["output_rows"] == len(want)


def test_device_path_matches_host_path(kb, rt, oracle):
    import torch
    nb, np_ = 50_000, 400_000
    rng = np.random.default_rng(14)
    bk = torch.tensor(rng.integers(0, 60_000, nb), dtype=torch.int64, device="cuda")
    bv = torch.arange(nb, dtype=torch.int64, device="cuda")
    pk = torch.tensor(rng.integers(0, 60_000, np_), dtype=torch.int64, device="cuda")
    pid = torch.arange(np_, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    j = kb.HashJoin(rt, kb.join_spec("inner"))
    j.build_push_device(kb.DeviceBatch([("k", bk, None), ("bid", bv, None)]))
    j.build_finish()
    res = j.probe_device(kb.DeviceBatch([("k", pk, None), ("pid", pid, None)]))
    rt.synchronize()
    got = collections.Counter(zip(res.columns[1].cpu().tolist(), res.columns[3].cpu().tolist()))
    p, b = oracle.hash_join(0, [(bk.cpu().numpy(), None, False)], [(pk.cpu().numpy(), None, False)])
    assert got == collections.Counter(zip(p.tolist(), b.tolist()))


def test_budget_need_memory(kb):
    import torch
    small = kb.Runtime(0, 1 << 20, torch.cuda.current_stream().cuda_stream or None)
    j = kb.HashJoin(small, kb.join_spec("inner"))
    with pytest.raises(kb.KrvError) as e:
        j.build_push(batch(k=pa.array(np.arange(1 << 20, dtype=np.int64))))
    assert e.value.status == kb.NEED_MEMORY
    assert kb.lib().krv_last_need_bytes() > 0


@pytest.mark.parametrize("jt", ["inner", "left_outer"])
def test_dense_unique_build_keys(kb, rt, oracle, jt):
    """Unique build keys over a dense range starting below zero, with holes
    and NULL keys, probed by keys inside, just outside and far outside the
    range (the int64 extremes) and NULLs: the oracle's pairs."""
    rng = np.random.default_rng(15)
    lo, span = -500_000, 140_000
    keys = lo + rng.permutation(span)[:100_000]
    build = [(int(k), 0) for k in keys] + [(None, 0)] * 50
    rng.shuffle(build)
    pk = rng.integers(lo - 1000, lo + span + 1000, 300_000)
    probe = [(int(k), 0) for k in pk] + [(None, 0)] * 20 + [(-2**63, 0), (2**63 - 1, 0), (lo, 0), (lo - 1, 0)]
    want = oracle_pairs(oracle, jt, probe, build, 1, False)
    got = gpu_pairs(kb, rt, jt, probe, build, 1, False, build_batches=2)
    assert got == want


def str_of(v):
    """A string key per int key (one to one, some over 8 bytes), None kept."""
    return None if v is None else ("key-%d-" % v) * (1 + abs(v) % 3)


def rows_batch_str(rows, idname):
    k1 = pa.array([str_of(r[0]) for r in rows], type=pa.string())
    k2 = pa.array([r[1] for r in rows], type=pa.int32())
    return batch(k1=k1, k2=k2, **{idname: pa.array(np.arange(len(rows), dtype=np.int64))})


def gpu_pairs_str(kb, rt, jt, probe, build, nkeys, null_safe, build_batches=1):
    """gpu_pairs with a string first key: the id columns are projected, the
    string key is not (`test_string_keys_in_the_output` projects it)."""
    spec = kb.join_spec(jt, probe_keys=tuple(range(nkeys)), build_keys=tuple(range(nkeys)),
                        null_safe=[null_safe] * nkeys, probe_out=[2], build_out=[2])
    j = kb.HashJoin(rt, spec)
    b = rows_batch_str(build, "bid")
    step = max(1, -(-len(build) // build_batches))
    if len(build) == 0:
        j.build_push(b)
    for s in range(0, len(build), step):
        j.build_push(b.slice(s, step))
    j.build_finish()
    outs = j.probe(rows_batch_str(probe, "pid"))
    outs += j.finish()
    t = concat(outs)
    if jt == "existence":
        return collections.Counter(zip(t.column("pid").to_pylist(), [int(x) for x in t.column("exists").to_pylist()]))
    return pairs_from_output(t)


@pytest.mark.parametrize("jt", TYPES)
def test_string_keys_match_the_oracle(kb, rt, oracle, jt):
    """String join keys (one string key, or a string and an int32 key, `=`
    and `<=>`), coded by the key dictionary: every join type gives the
    oracle's pairs on the edge cases and on random keys with duplicates and
    NULLs (the oracle joins the int keys the strings stand for)."""
    rng = np.random.default_rng(16)
    probe_r = [(int(x) if x >= 0 else None, int(y)) for x, y in zip(rng.integers(-20, 3000, 20000),
                                                                     rng.integers(0, 3, 20000))]
    build_r = [(int(x) if x >= 0 else None, int(y)) for x, y in zip(rng.integers(-20, 3000, 9000),
                                                                     rng.integers(0, 3, 9000))]
    inputs = [(EDGE_PROBE, EDGE_BUILD), (EDGE_PROBE, []), ([], EDGE_BUILD), (EDGE_PROBE, ALL_NULL),
              (ALL_NULL, EDGE_BUILD), (probe_r, build_r)]
    for nkeys in (1, 2):
        for safe in (False, True):
            if jt == "null_aware_anti" and (nkeys > 1 or safe):
                continue
            for probe, build in inputs:
                want = oracle_pairs(oracle, jt, probe, build, nkeys, safe)
                got = gpu_pairs_str(kb, rt, jt, probe, build, nkeys, safe, build_batches=3 if len(build) > 100 else 1)
                assert got == want, (jt, nkeys, safe, len(probe), len(build))


def test_string_key_types_must_agree(kb, rt):
    spec = kb.join_spec("inner", probe_out=[1], build_out=[1])
    j = kb.HashJoin(rt, spec)
    j.build_push(batch(k=pa.array(["a", "b"]), bid=pa.array([0, 1])))
    j.build_finish()
    with pytest.raises(kb.KrvError) as e:
        j.probe(batch(k=pa.array([1, 2]), pid=pa.array([0, 1])))
    assert e.value.status in (kb.INVALID_ARGUMENT, kb.UNSUPPORTED)


@pytest.mark.parametrize("jt", ["inner", "left_outer", "right_outer", "full_outer", "left_semi", "existence"])
def test_string_keys_in_the_output(kb, rt, oracle, jt):
    """A join on a string key (plus an int32 key) that projects the string
    keys of both sides: the pairs are the oracle's, and every output row's
    strings are those of the rows it came from (NULL on a padded side)."""
    rng = np.random.default_rng(21)
    probe = [(int(x) if x >= 0 else None, int(y)) for x, y in zip(rng.integers(-20, 400, 3000), rng.integers(0, 2, 3000))]
    build = [(int(x) if x >= 0 else None, int(y)) for x, y in zip(rng.integers(-20, 400, 1500), rng.integers(0, 2, 1500))]
    spec = kb.join_spec(jt, probe_keys=(0, 1), build_keys=(0, 1), probe_out=[2, 0], build_out=[2, 0])
    j = kb.HashJoin(rt, spec)
    j.build_push(rows_batch_str(build, "bid"))
    j.build_finish()
    t = concat(j.probe(rows_batch_str(probe, "pid")) + j.finish())
    pk, pid = t.column(1).to_pylist(), t.column("pid").to_pylist()
    for i, p in enumerate(pid):
        assert pk[i] == (str_of(probe[p][0]) if p is not None else None)
    want = oracle_pairs(oracle, jt, probe, build, 2, False)
    if jt == "existence":
        assert collections.Counter(zip(pid, [int(x) for x in t.column("exists").to_pylist()])) == want
        return
    if jt != "left_semi":
        bk, bid = t.column(3).to_pylist(), t.column("bid").to_pylist()
        for i, b in enumerate(bid):
            assert bk[i] == (str_of(build[b][0]) if b is not None else None)
    assert pairs_from_output(t) == want
