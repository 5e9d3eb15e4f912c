"""GPU grouped aggregate parity against the CPU oracle and Spark 4.2's TPC-H
answers, through the C ABI. Integer and decimal results are bit-exact;
float64 SUM/AVG are within 1e-12 relative of the oracle's compensated sum;
MIN/MAX and COUNT are exact."""
import os
from decimal import Decimal

import decimal

import numpy as np
import pyarrow as pa
import pytest

from helpers import batch, concat, rel_err

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FLOAT_TOL = 1e-12  # relative, against the FP64 compensated-sum oracle


def run(kb, rt, b, group_by, aggs, mode, expected_groups=0, ansi=True, batches=1):
    a = kb.HashAggregate(rt, kb.agg_spec(group_by, aggs, ansi=ansi, mode=mode, expected_groups=expected_groups))
    step = max(1, -(-b.num_rows // batches))
    for s in range(0, b.num_rows, step):
        a.push(b.slice(s, step))
    a.finish()
    return concat(a.result())


@pytest.mark.parametrize("mode", [1, 2])
def test_tpch_q13_spark_answer(kb, rt, mode):
    d = np.load(os.path.join(GOLDEN, "tpch_q13.npz"))
    b = batch(c_custkey=pa.array(d["c_custkey"]),
              o_orderkey=pa.array(d["o_orderkey"], mask=d["o_orderkey_valid"] == 0))
    inner = run(kb, rt, b, 0, [("count", 1)], mode, batches=3)
    mid = batch(c_custkey=inner.column(0).combine_chunks(), c_count=inner.column(1).combine_chunks())
    outer = run(kb, rt, mid, 1, [("count_star", 0)], mode)
    got = sorted(zip(outer.column(0).to_pylist(), outer.column(1).to_pylist()))
    assert got == [tuple(r) for r in d["expected"].tolist()]


@pytest.mark.parametrize("mode", [1, 2])
def test_tpch_q18_spark_answer(kb, rt, mode):
    d = np.load(os.path.join(GOLDEN, "tpch_q18.npz"))
    from decimal import Decimal
    qty = pa.array([Decimal(int(v)).scaleb(-int(d["scale"])) for v in d["l_quantity_unscaled"]],
                   type=pa.decimal128(int(d["precision"]), int(d["scale"])))
    b = batch(o_orderkey=pa.array(d["o_orderkey"]), l_quantity=qty)
    out = run(kb, rt, b, 0, [("sum", 1)], mode)
    assert out.schema.field(1).type == pa.decimal128(25, 2)  # sum_decimal (aggregate/mod.rs:929-931)
    got = sorted((k, int(v.scaleb(2))) for k, v in zip(out.column(0).to_pylist(), out.column(1).to_pylist()))
    assert got == [tuple(r) for r in d["expected"].tolist()]


def value_batch(n, key, rng, nulls=0.02):
    def mask():
        return rng.random(n) < nulls
    dec = rng.integers(100, 10_000_000, n, dtype=np.int64)
    f = rng.random(n)
    q = rng.integers(1, 51, n).astype(np.int32)
    i64 = rng.integers(-2**40, 2**40, n, dtype=np.int64)
    m = [mask() for _ in range(4)]
    cols = {
        "k": pa.array(key),
        "dec": pa.Array.from_buffers(pa.decimal64(15, 2), n, [pa.array(~m[0]).buffers()[1], pa.py_buffer(dec.tobytes())]),
        "f": pa.array(f, mask=m[1]),
        "q": pa.array(q, mask=m[2]),
        "i": pa.array(i64, mask=m[3]),
    }
    raw = {"dec": (dec, ~m[0]), "f": (f, ~m[1]), "q": (q, ~m[2]), "i": (i64, ~m[3])}
    return batch(**cols), raw


FUNCS = ["sum", "count", "min", "max", "avg"]


def check_against_oracle(oracle, out, key, raw, aggs, names):
    T = {"dec": oracle.T_DEC64, "f": oracle.T_F64, "q": oracle.T_I32, "i": oracle.T_I64}
    cols = [{"values": raw[n][0], "valid": raw[n][1].astype(np.uint8), "type": T[n], "precision": 15, "scale": 2}
            for n in names]
    F = {"sum": oracle.SUM, "count": oracle.COUNT, "min": oracle.MIN, "max": oracle.MAX, "avg": oracle.AVG,
         "count_star": oracle.COUNT_STAR}
    keys, kv, res = oracle.hash_aggregate(key, None, cols, [(F[f], c - 1) for f, c in aggs])
    order = {int(k): i for i, k in enumerate(keys)}
    got_keys = out.column(0).to_pylist()
    assert sorted(got_keys) == sorted(order)
    for e, (f, c) in enumerate(aggs):
        col = out.column(1 + e).to_pylist()
        name = names[c - 1] if c > 0 else None
        for k, v in zip(got_keys, col):
            gi = order[k]
            r = res[e]
            if not r["valid"][gi]:
                assert v is None, (f, name, k)
                continue
            assert v is not None, (f, name, k)
            if f in ("count", "count_star"):
                assert v == r["i64"][gi]
            elif name == "f" and f in ("sum", "avg"):
                assert rel_err(v, r["f64"][gi]) <= FLOAT_TOL, (f, k, v, r["f64"][gi])
            elif name == "f" or (name in ("q", "i") and f == "avg"):
                assert v == r["f64"][gi], (f, name, k)
            elif name == "dec":
                unscaled = int(v.scaleb(out.schema.field(1 + e).type.scale))
                want = int(r["lo"][gi]) + (int(r["hi"][gi]) << 64) if f in ("sum", "avg") else int(r["i64"][gi])
                assert unscaled == want, (f, k)
            else:
                assert v == r["i64"][gi], (f, name, k)


@pytest.mark.parametrize("mode", [1, 2])
def test_all_functions_with_nulls(kb, rt, oracle, mode):
    rng = np.random.default_rng(21)
    n = 300_000
    key = rng.integers(0, 5000, n, dtype=np.int64)
    b, raw = value_batch(n, key, rng)
    names = ["dec", "f", "q", "i"]
    aggs = [("count_star", 0)] + [(f, c) for c in (1, 2, 3, 4) for f in FUNCS]
    out = run(kb, rt, b, 0, aggs, mode, expected_groups=5000, batches=2)
    types = [out.schema.field(i).type for i in range(out.num_columns)]
    assert types[1] == pa.int64()
    assert types[2] == pa.decimal128(25, 2) and types[6] == pa.decimal128(19, 6)  # mod.rs:929, 1018
    assert types[7] == pa.float64() and types[13] == pa.int64() and types[14] == pa.int32()
    assert types[16] == pa.float64() and types[17] == pa.int64() and types[4] == pa.decimal64(15, 2)
    check_against_oracle(oracle, out, key, {k: raw[k] for k in names}, aggs, names)


@pytest.mark.parametrize("mode", [1, 2])
def test_zipf_keys_and_table_growth(kb, rt, oracle, mode):
    """Zipf(1.1) keys over 200,000 values (the grouped-aggregate workload's
    distribution at a smaller size) with no group estimate: the table grows."""
    rng = np.random.default_rng(22)
    n, domain = 2_000_000, 200_000
    cdf = oracle.zipf_cdf(1.1, domain)
    rank = np.searchsorted(cdf, rng.random(n), side="right")
    perm = rng.permutation(domain)
    key = perm[np.minimum(rank, domain - 1)].astype(np.int64)
    b, raw = value_batch(n, key, rng)
    names = ["dec", "f", "q", "i"]
    aggs = [(f, c) for c in (1, 2, 3) for f in FUNCS] + [("count_star", 0)]
    out = run(kb, rt, b, 0, aggs, mode, expected_groups=0)
    check_against_oracle(oracle, out, key, {k: raw[k] for k in names}, aggs, names)


def test_null_keys_and_int32_keys(kb, rt, oracle):
    key = np.array([1, 2, 0, 1, 0, 3], dtype=np.int32)
    kvalid = np.array([1, 1, 0, 1, 0, 1], dtype=bool)
    v = np.array([10, 20, 30, 40, 50, 60], dtype=np.int64)
    b = batch(k=pa.array(key, mask=~kvalid), v=pa.array(v))
    for mode in (1, 2):
        out = run(kb, rt, b, 0, [("sum", 1), ("count_star", 0)], mode)
        got = sorted(zip(out.column(0).to_pylist(), out.column(1).to_pylist(), out.column(2).to_pylist()),
                     key=lambda t: (t[0] is not None, t[0]))
        assert got == [(None, 80, 2), (1, 50, 2), (2, 20, 1), (3, 60, 1)]


def test_marker_key_value(kb, rt):
    # the table's empty marker is a legal key value too
    marker = int(np.array([0x8080808080808080], dtype=np.uint64).view(np.int64)[0])
    b = batch(k=pa.array(np.array([marker, 5, marker], dtype=np.int64)), v=pa.array(np.array([1, 2, 3], dtype=np.int64)))
    for mode in (1, 2):
        out = run(kb, rt, b, 0, [("sum", 1)], mode)
        assert sorted(zip(out.column(0).to_pylist(), out.column(1).to_pylist())) == [(marker, 4), (5, 2)]


def test_ansi_overflow(kb, rt):
    b = batch(k=pa.array(np.zeros(3, dtype=np.int64)), v=pa.array(np.array([2**62, 2**62, 2**62], dtype=np.int64)))
    with pytest.raises(kb.KrvError) as e:
        run(kb, rt, b, 0, [("sum", 1)], 1, ansi=True)
    assert e.value.status == kb.ARITHMETIC_OVERFLOW
    out = run(kb, rt, b, 0, [("sum", 1)], 1, ansi=False)
    assert out.column(1).to_pylist() == [int(np.int64(3 * 2**62 - 2**64))]  # wraps


def test_device_path(kb, rt, oracle):
    import torch
    rng = np.random.default_rng(23)
    n = 1_000_000
    key = rng.integers(0, 1000, n, dtype=np.int64)
    v = rng.integers(-1000, 1000, n, dtype=np.int64)
    kt = torch.tensor(key, device="cuda")
    vt = torch.tensor(v, device="cuda")
    torch.cuda.synchronize()
    a = kb.HashAggregate(rt, kb.agg_spec(0, [("sum", 1), ("min", 1), ("count_star", 0)], expected_groups=1000))
    a.push_device(kb.DeviceBatch([("k", kt, None), ("v", vt, None)]))
    a.finish()
    res = a.result_device()
    rt.synchronize()
    got_k = res.columns[0].cpu().numpy()
    got_s = res.columns[1].cpu().numpy()
    keys, _, r = oracle.hash_aggregate(key, None, [{"values": v, "type": oracle.T_I64}],
                                       [(oracle.SUM, 0), (oracle.MIN, 0), (oracle.COUNT_STAR, 0)])
    want = dict(zip(keys.tolist(), r[0]["i64"].tolist()))
    assert dict(zip(got_k.tolist(), got_s.tolist())) == want


@pytest.mark.parametrize("mode", [1, 2])
def test_decimal128_columns(kb, rt, oracle, mode):
    """decimal128(15,2) values (the carrier Spark-written Arrow files use for
    decimal(15,2)), negative and NULL: SUM, COUNT, MIN, MAX and AVG exact
    against the oracle; MIN/MAX keep the input type."""
    rng = np.random.default_rng(41)
    n = 200_000
    key = rng.integers(0, 3000, n, dtype=np.int64)
    v = rng.integers(-10**13, 10**13, n, dtype=np.int64)
    valid = rng.random(n) > 0.03
    words = np.stack([v, np.where(v < 0, -1, 0)], 1).astype(np.int64).reshape(-1)
    dec = pa.Array.from_buffers(pa.decimal128(15, 2), n, [pa.py_buffer(np.packbits(valid, bitorder="little").tobytes()),
                                                         pa.py_buffer(words.tobytes())])
    b = batch(k=pa.array(key), d=dec)
    aggs = [(f, 1) for f in FUNCS]
    out = run(kb, rt, b, 0, aggs, mode, batches=3)
    assert [out.schema.field(i).type for i in range(1, 6)] == [pa.decimal128(25, 2), pa.int64(), pa.decimal128(15, 2),
                                                              pa.decimal128(15, 2), pa.decimal128(19, 6)]
    cols = [{"values": words, "valid": valid.astype(np.uint8), "type": oracle.T_DEC128, "precision": 15, "scale": 2}]
    F = {"sum": oracle.SUM, "count": oracle.COUNT, "min": oracle.MIN, "max": oracle.MAX, "avg": oracle.AVG}
    keys, _, res = oracle.hash_aggregate(key, None, cols, [(F[f], 0) for f, _ in aggs])
    order = {int(k): i for i, k in enumerate(keys)}
    got = {k: r for k, *r in zip(*[c.to_pylist() for c in out.columns])}
    assert sorted(got) == sorted(order)
    for k, vals in got.items():
        gi = order[k]
        for e, (f, _) in enumerate(aggs):
            r = res[e]
            if not r["valid"][gi]:
                assert vals[e] is None
                continue
            if f == "count":
                assert vals[e] == r["i64"][gi]
            elif f in ("sum", "avg"):
                scale = out.schema.field(1 + e).type.scale
                assert int(vals[e].scaleb(scale)) == int(r["lo"][gi]) + (int(r["hi"][gi]) << 64), (f, k)
            else:
                assert int(vals[e].scaleb(2)) == int(r["i64"][gi]), (f, k)


def dec38(rng, n):
    """decimal(38,4) words (lo, hi per value) across the 128-bit range: large
    values of both signs, values inside and at the edges of int64, ties."""
    hi = rng.integers(-2**40, 2**40, n, dtype=np.int64)
    lo = rng.integers(-2**63, 2**63 - 1, n, dtype=np.int64)
    small = rng.random(n) < 0.4  # int64 values: hi is lo's sign
    lo[small] = rng.choice(np.array([-2**63, -1, 0, 1, 2**63 - 1], np.int64), int(small.sum()))
    hi[small] = np.where(lo[small] < 0, -1, 0)
    return np.stack([lo, hi], 1).reshape(-1)


@pytest.mark.parametrize("mode", [1, 2])
def test_decimal38_min_max(kb, rt, oracle, mode):
    """MIN/MAX of decimal(38,4) values beyond int64 (both signs, NULLs, three
    batches) equal the oracle's 128-bit MinMax (Values::Int(i128),
    aggregate/accumulator.rs:238-248); SUM and COUNT beside them exact. The
    same aggregates run in two phases (partial states, then their merge)
    give the same answer."""
    rng = np.random.default_rng(77)
    n = 150_000
    key = rng.integers(0, 700, n, dtype=np.int64)
    words = dec38(rng, n)
    valid = rng.random(n) > 0.03
    t = pa.decimal128(38, 4)
    dec = pa.Array.from_buffers(t, n, [pa.py_buffer(np.packbits(valid, bitorder="little").tobytes()),
                                       pa.py_buffer(words.tobytes())])
    b = batch(k=pa.array(key), d=dec)
    aggs = [("min", 1), ("max", 1), ("sum", 1), ("count", 1)]
    out = run(kb, rt, b, 0, aggs, mode, batches=3)
    assert [out.schema.field(i).type for i in range(1, 5)] == [t, t, pa.decimal128(38, 4), pa.int64()]
    cols = [{"values": words, "valid": valid.astype(np.uint8), "type": oracle.T_DEC128, "precision": 38, "scale": 4}]
    F = {"sum": oracle.SUM, "count": oracle.COUNT, "min": oracle.MIN, "max": oracle.MAX}
    keys, _, res = oracle.hash_aggregate(key, None, cols, [(F[f], 0) for f, _ in aggs])
    order = {int(k): i for i, k in enumerate(keys)}

    def check(got):
        assert sorted(got) == sorted(order)
        beyond = 0
        for k, vals in got.items():
            gi = order[k]
            for e, (f, _) in enumerate(aggs):
                r = res[e]
                if not r["valid"][gi]:
                    assert vals[e] is None
                    continue
                if f == "count":
                    assert vals[e] == r["i64"][gi]
                    continue
                want = int(r["lo"][gi]) + (int(r["hi"][gi]) << 64)
                # exact: 38 digits need more than the default 28-digit context
                assert int(vals[e].scaleb(4, decimal.Context(prec=80))) == want, (f, k)
                beyond += f in ("min", "max") and not -2**63 <= want < 2**63
        assert beyond > 100  # the extremes are beyond int64

    check({k: r for k, *r in zip(*[c.to_pylist() for c in out.columns])})
    # two phases: each batch's partial states, then one merge of them all
    parts = []
    for s_ in np.array_split(np.arange(n), 3):
        pa_ = kb.HashAggregate(rt, kb.agg_spec(0, aggs, mode=mode, partial=True))
        pa_.push(b.slice(int(s_[0]), len(s_)))
        pa_.finish()
        parts += pa_.result()
    states = pa.Table.from_batches(parts).combine_chunks().to_batches()[0]
    m = kb.HashAggregate(rt, kb.agg_spec(0, kb.merging(aggs, 1, [t] * 4), mode=mode))
    m.push(states)
    m.finish()
    merged = pa.Table.from_batches(m.result())
    check({k: r for k, *r in zip(*[c.to_pylist() for c in merged.columns])})
