"""Grouped aggregates over composite and string group keys (the key
dictionary, csrc/keydict.cu), through the C ABI with host Arrow batches:
Spark 4.2.0's answers for TPC-H Q1 (two string keys, decimal sums and
averages) and Q18's outer aggregate (five keys: string, int64, int64,
date32, decimal), and random composite keys against the CPU oracle, whose
single-key aggregate is fed one code per distinct key tuple (group identity
does not depend on how groups are numbered). Integer and decimal results
are exact; float64 sums within 1e-12 relative."""
import math
import os
from decimal import Decimal

import numpy as np
import pyarrow as pa
import pytest

from helpers import concat, rel_err

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def table_of(d):
    """The Arrow batch of a fixture written by tests/golden/make_golden.py."""
    arrays, names = [], []
    for name in d["__order"].tolist():
        valid = d[name + "__valid"].astype(bool)
        n = valid.size
        vbuf = None if valid.all() else pa.py_buffer(np.packbits(valid, bitorder="little").tobytes())
        if name + "__str" in d:
            arr = pa.array([s if v else None for s, v in zip(d[name + "__str"].tolist(), valid)], pa.string())
        elif name + "__dec_lo" in d:
            p, s = (int(x) for x in d[name + "__dec_ps"])
            words = np.stack([d[name + "__dec_lo"], d[name + "__dec_hi"]], 1).reshape(-1)
            arr = pa.Array.from_buffers(pa.decimal128(p, s), n, [vbuf, pa.py_buffer(words.tobytes())])
        elif name + "__date32" in d:
            arr = pa.Array.from_buffers(pa.date32(), n, [vbuf, pa.py_buffer(d[name + "__date32"].astype(np.int32).tobytes())])
        else:
            arr = pa.Array.from_buffers(pa.int64(), n, [vbuf, pa.py_buffer(d[name + "__int64"].astype(np.int64).tobytes())])
        arrays.append(arr)
        names.append(name)
    return pa.RecordBatch.from_arrays(arrays, names=names)


def run(kb, rt, b, group_by, aggs, mode=2, batches=1, expected_groups=0):
    a = kb.HashAggregate(rt, kb.agg_spec(group_by, aggs, mode=mode, expected_groups=expected_groups))
    step = max(1, -(-b.num_rows // batches))
    for s in range(0, b.num_rows, step):
        a.push(b.slice(s, step))
    a.finish()
    return concat(a.result())


def text(v):
    if isinstance(v, Decimal):
        return str(v)
    if hasattr(v, "isoformat"):
        return v.isoformat()
    return str(v)


@pytest.mark.parametrize("mode", [1, 2])
@pytest.mark.parametrize("batches", [1, 5])
def test_tpch_q1_spark_answer(kb, rt, mode, batches):
    d = np.load(os.path.join(GOLDEN, "tpch_q1.npz"))
    b = table_of(d)
    aggs = [("sum", 2), ("sum", 3), ("sum", 4), ("sum", 5), ("avg", 2), ("avg", 3), ("avg", 6), ("count_star", 0)]
    out = run(kb, rt, b, [0, 1], aggs, mode=mode, batches=batches)
    assert out.schema.field(0).type == pa.string() and out.schema.field(1).type == pa.string()
    # sum_decimal / AVG decimal result types (aggregate/mod.rs:929-931, 588-740)
    assert [out.schema.field(i).type for i in range(2, 9)] == [
        pa.decimal128(25, 2), pa.decimal128(25, 2), pa.decimal128(38, 4), pa.decimal128(38, 6),
        pa.decimal128(19, 6), pa.decimal128(19, 6), pa.decimal128(19, 6)]
    rows = sorted(",".join(text(v) for v in r) for r in zip(*[c.to_pylist() for c in out.columns]))
    assert rows == d["expected"].tolist()


@pytest.mark.parametrize("mode", [1, 2])
def test_tpch_q18_five_keys_spark_answer(kb, rt, mode):
    d = np.load(os.path.join(GOLDEN, "tpch_q18_keys.npz"))
    b = table_of(d)
    out = run(kb, rt, b, [0, 1, 2, 3, 4], [("sum", 5)], mode=mode, batches=3)
    assert [f.type for f in out.schema] == [pa.string(), pa.int64(), pa.int64(), pa.date32(), pa.decimal128(15, 2),
                                           pa.decimal128(25, 2)]
    rows = sorted(",".join(text(v) for v in r) for r in zip(*[c.to_pylist() for c in out.columns]))
    assert rows == d["expected"].tolist()


def random_keys(rng, n):
    """Composite keys with collisions across columns, NULLs, signed zeros, a
    NaN, empty and long strings (several 8-byte hash words)."""
    words = ["", "a", "b", "ab", "ba", "alpha", "beta", "x" * 9, "x" * 17, "long string of text " * 3, "ünïcode"]
    s = [None if rng.random() < 0.03 else words[int(rng.integers(0, len(words)))] for _ in range(n)]
    i32 = rng.integers(-3, 4, n).astype(np.int32)
    i32_valid = rng.random(n) > 0.02
    f = rng.choice(np.array([0.0, -0.0, 1.5, -2.25, np.nan, 1e300]), n)
    dec = rng.integers(-5, 5, n).astype(np.int64)
    return s, i32, i32_valid, f, dec


def key_tuple(s, i, iv, f, dv):
    # GROUP BY semantics: NULL is a value; -0.0 is 0.0; every NaN is one NaN
    ff = "nan" if math.isnan(f) else (0.0 if f == 0.0 else f)
    return (s, int(i) if iv else None, ff, dv)


def test_random_composite_keys_match_the_oracle(kb, rt, oracle):
    rng = np.random.default_rng(21)
    n = 200_000
    s, i32, i32v, f, dec = random_keys(rng, n)
    dec_valid = rng.random(n) > 0.02
    x = rng.integers(-10**12, 10**12, n, dtype=np.int64)
    y = rng.random(n) * 100 - 50
    yv = rng.random(n) > 0.02
    b = pa.RecordBatch.from_arrays(
        [pa.array(s, pa.string()), pa.array(i32, mask=~i32v), pa.array(f), pa.array(x),
         pa.array([Decimal(int(v)).scaleb(-2) if ok else None for v, ok in zip(dec, dec_valid)], pa.decimal128(20, 2)),
         pa.array(y, mask=~yv)],
        names=["s", "i", "f", "x", "d", "y"])
    aggs = [("sum", 3), ("min", 3), ("max", 3), ("count", 5), ("sum", 5), ("avg", 5), ("count_star", 0)]
    out = run(kb, rt, b, [0, 1, 2, 4], aggs, batches=4)
    # the oracle, fed one dense code per key tuple
    tuples = [key_tuple(s[r], i32[r], i32v[r], float(f[r]), int(dec[r]) if dec_valid[r] else None) for r in range(n)]
    code_of = {}
    codes = np.array([code_of.setdefault(t, len(code_of)) for t in tuples], dtype=np.int64)
    cols = [{"values": x, "type": oracle.T_I64}, {"values": y, "valid": yv.astype(np.uint8), "type": oracle.T_F64}]
    F = {"sum": oracle.SUM, "count": oracle.COUNT, "min": oracle.MIN, "max": oracle.MAX, "avg": oracle.AVG,
         "count_star": oracle.COUNT_STAR}
    wk, _, wr = oracle.hash_aggregate(codes, None, cols, [(F[fn], {3: 0, 5: 1, 0: 0}[c]) for fn, c in aggs])
    tuple_of = {c: t for t, c in code_of.items()}
    want = {}
    for j, c in enumerate(wk.tolist()):
        vals = []
        for e, (fn, _) in enumerate(aggs):
            w = wr[e]
            if "valid" in w and not w["valid"][j]:
                vals.append(None)
            elif fn in ("sum", "avg") and aggs[e][1] == 5:
                vals.append(float(w["f64"][j]))
            else:
                vals.append(int(w["i64"][j]))
        want[tuple_of[c]] = vals
    assert out.num_rows == len(want)
    cols_out = [c.to_pylist() for c in out.columns]
    for r in range(out.num_rows):
        fv = cols_out[2][r]
        key = key_tuple(cols_out[0][r], cols_out[1][r] if cols_out[1][r] is not None else 0,
                        cols_out[1][r] is not None, fv, None)
        dv = cols_out[3][r]
        key = key[:3] + (int(dv.scaleb(2)) if dv is not None else None,)
        w = want[key]
        got = [cols_out[4 + e][r] for e in range(len(aggs))]
        for e, (fn, c) in enumerate(aggs):
            if w[e] is None or got[e] is None:
                assert w[e] is None and got[e] is None, (key, fn)
            elif isinstance(w[e], float):
                assert rel_err(got[e], w[e]) <= 1e-12, (key, fn)
            else:
                assert got[e] == w[e], (key, fn)


def test_string_keys_across_batches(kb, rt):
    """One string key over many batches: codes and key bytes kept across
    pushes (the dictionary and its byte heap grow), NULL and empty strings
    their own groups, every distinct string one output row."""
    rng = np.random.default_rng(22)
    n = 300_000
    vocab = ["k%d" % i * (1 + i % 5) for i in range(5000)] + [""]
    s = [None if rng.random() < 0.01 else vocab[int(rng.integers(0, len(vocab)))] for _ in range(n)]
    v = rng.integers(0, 1000, n, dtype=np.int64)
    b = pa.RecordBatch.from_arrays([pa.array(s, pa.string()), pa.array(v)], names=["s", "v"])
    out = run(kb, rt, b, [0], [("sum", 1), ("count_star", 0)], batches=7, expected_groups=16)
    want = {}
    for k, x in zip(s, v.tolist()):
        a, c = want.get(k, (0, 0))
        want[k] = (a + x, c + 1)
    got = {k: (a, c) for k, a, c in zip(*[c.to_pylist() for c in out.columns])}
    assert got == want


def test_binary_and_float_single_keys(kb, rt):
    """A binary key and a float64 key each take the dictionary (one key of
    a type the single-key tables do not take)."""
    rng = np.random.default_rng(23)
    n = 50_000
    raw = [bytes(rng.integers(0, 256, int(rng.integers(0, 12)), dtype=np.uint8)) for _ in range(300)]
    keys = [raw[int(i)] for i in rng.integers(0, len(raw), n)]
    v = rng.integers(-100, 100, n, dtype=np.int64)
    b = pa.RecordBatch.from_arrays([pa.array(keys, pa.binary()), pa.array(v)], names=["k", "v"])
    out = run(kb, rt, b, [0], [("sum", 1)], batches=2)
    want = {}
    for k, x in zip(keys, v.tolist()):
        want[k] = want.get(k, 0) + x
    assert dict(zip(*[c.to_pylist() for c in out.columns])) == want
    f = rng.choice(np.array([0.0, -0.0, np.nan, -np.nan, 3.5]), n)
    b2 = pa.RecordBatch.from_arrays([pa.array(f), pa.array(v)], names=["f", "v"])
    out2 = run(kb, rt, b2, [0], [("count_star", 0)])
    got = {("nan" if math.isnan(k) else k): c for k, c in zip(*[c.to_pylist() for c in out2.columns])}
    want2 = {}
    for k in f.tolist():
        kk = "nan" if math.isnan(k) else (0.0 if k == 0.0 else k)
        want2[kk] = want2.get(kk, 0) + 1
    assert got == want2 and out2.num_rows == len(want2)


def test_strings_elsewhere_are_unsupported(kb, rt):
    """A string argument of SUM fails with UNSUPPORTED; string payloads of
    a join on fixed-width keys are taken, and so are the string keys of a
    join on string keys (every column projected)."""
    b = pa.RecordBatch.from_arrays([pa.array(["a", "b"]), pa.array([1, 2])], names=["s", "v"])
    j = kb.HashJoin(rt, kb.join_spec("inner", probe_keys=(1,), build_keys=(1,)))
    j.build_push(b)
    j.build_finish()
    from helpers import concat
    out = concat(j.probe(b))
    assert sorted(zip(out.column(1).to_pylist(), out.column(2).to_pylist())) == [(1, "a"), (2, "b")]
    j2 = kb.HashJoin(rt, kb.join_spec("inner"))  # key 0 is a string, every column projected
    j2.build_push(b)
    j2.build_finish()
    out2 = concat(j2.probe(b))
    assert sorted(zip(*[c.to_pylist() for c in out2.columns])) == [("a", 1, "a", 1), ("b", 2, "b", 2)]
    a = kb.HashAggregate(rt, kb.agg_spec(1, [("sum", 0)]))
    with pytest.raises(kb.KrvError) as e:
        a.push(b)
    assert e.value.status == kb.UNSUPPORTED


@pytest.mark.parametrize("mode", [1, 2])
def test_count_of_string_columns(kb, rt, oracle, mode):
    """COUNT(s) and COUNT(b) of UTF-8 and binary columns with NULLs count
    their non-NULL values per group (the one-pass kernels and, at 300,000
    rows in the shared-memory mode, the partitioned path), beside SUM of an
    int column; equal to the oracle's COUNT over the same validity."""
    rng = np.random.default_rng(44)
    n = 300_000
    key = rng.integers(0, 5000, n).astype(np.int64)
    sv = rng.random(n) > 0.1
    bv = rng.random(n) > 0.3
    s = pa.array([("v%d" % (i % 97)) if sv[i] else None for i in range(n)], pa.string())
    bb = pa.array([bytes([i % 251]) * (i % 5) if bv[i] else None for i in range(n)], pa.binary())
    x = rng.integers(-1000, 1000, n).astype(np.int64)
    b = pa.RecordBatch.from_arrays([pa.array(key), s, bb, pa.array(x)], names=["k", "s", "b", "x"])
    a = kb.HashAggregate(rt, kb.agg_spec(0, [("count", 1), ("count", 2), ("sum", 3)], mode=mode))
    a.push(b)
    a.finish()
    out = pa.Table.from_batches(a.result())
    assert out.schema.field(1).type == pa.int64() and out.schema.field(2).type == pa.int64()
    cols = [{"values": np.zeros(n, np.int64), "valid": sv.astype(np.uint8), "type": oracle.T_I64},
            {"values": np.zeros(n, np.int64), "valid": bv.astype(np.uint8), "type": oracle.T_I64},
            {"values": x, "type": oracle.T_I64}]
    keys, _, res = oracle.hash_aggregate(key, None, cols, [(oracle.COUNT, 0), (oracle.COUNT, 1), (oracle.SUM, 2)])
    want = {int(k): (int(res[0]["i64"][i]), int(res[1]["i64"][i]), int(res[2]["i64"][i])) for i, k in enumerate(keys)}
    got = {k: (c1, c2, sm) for k, c1, c2, sm in zip(*[c.to_pylist() for c in out.columns])}
    assert got == want
    with pytest.raises(kb.KrvError) as e:  # SUM of a string column stays unsupported
        kb.HashAggregate(rt, kb.agg_spec(0, [("sum", 1)])).push(b)
    assert e.value.status == kb.UNSUPPORTED


@pytest.mark.parametrize("mode", [1, 2])
def test_min_max_of_string_columns(kb, rt, mode):
    """MIN and MAX of UTF-8 and binary columns (NULLs, empty values, prefixes
    of one another, multi-byte characters, groups with no value) over three
    batches: per group, the least and greatest values in byte order, as
    the reference's MinMax over Values::Bytes (aggregate/accumulator.rs:
    238-248) and Spark order them; NULL for a group with no value. The same
    aggregates in two phases (partial states, then their merge) agree."""
    rng = np.random.default_rng(45)
    n = 120_000
    key = rng.integers(0, 3000, n).astype(np.int64)
    words = ["", "a", "ab", "abc", "b", "zz", "é", "éa", "日本", "Z", "a" * 300]
    sv = rng.random(n) > 0.05
    sv[key == 7] = False  # a group with no string value
    svals = [words[int(w)] for w in rng.integers(0, len(words), n)]
    bvals = [bytes(rng.integers(0, 256, int(l), dtype=np.uint8)) for l in rng.integers(0, 6, n)]
    bv = rng.random(n) > 0.2
    s = pa.array([svals[i] if sv[i] else None for i in range(n)], pa.string())
    bb = pa.array([bvals[i] if bv[i] else None for i in range(n)], pa.binary())
    b = pa.RecordBatch.from_arrays([pa.array(key), s, bb], names=["k", "s", "b"])
    aggs = [("min", 1), ("max", 1), ("min", 2), ("max", 2), ("count", 1)]
    want = {}
    for i in range(n):
        w = want.setdefault(int(key[i]), [None, None, None, None, 0])
        if sv[i]:
            v = svals[i].encode()
            w[0] = v if w[0] is None or v < w[0] else w[0]
            w[1] = v if w[1] is None or v > w[1] else w[1]
            w[4] += 1
        if bv[i]:
            v = bvals[i]
            w[2] = v if w[2] is None or v < w[2] else w[2]
            w[3] = v if w[3] is None or v > w[3] else w[3]

    def norm(row):
        return [x.encode() if isinstance(x, str) else x for x in row]

    def check(table):
        got = {r[0]: norm(list(r[1:])) for r in zip(*[c.to_pylist() for c in table.columns])}
        assert got == {k: list(v) for k, v in want.items()}
        assert got[7][0] is None and got[7][1] is None

    a = kb.HashAggregate(rt, kb.agg_spec(0, aggs, mode=mode))
    for s0 in range(0, n, 40_000):
        a.push(b.slice(s0, 40_000))
    a.finish()
    out = pa.Table.from_batches(a.result())
    assert [out.schema.field(i).type for i in range(1, 5)] == [pa.string(), pa.string(), pa.binary(), pa.binary()]
    check(out)
    parts = []
    for s0 in range(0, n, 40_000):
        p = kb.HashAggregate(rt, kb.agg_spec(0, aggs, mode=mode, partial=True))
        p.push(b.slice(s0, 40_000))
        p.finish()
        parts += p.result()
    states = pa.Table.from_batches(parts).combine_chunks().to_batches()[0]
    m = kb.HashAggregate(rt, kb.agg_spec(0, kb.merging(aggs, 1, [pa.string(), pa.string(), pa.binary(),
                                                                 pa.binary(), pa.string()]), mode=mode))
    m.push(states)
    m.finish()
    check(pa.Table.from_batches(m.result()))
