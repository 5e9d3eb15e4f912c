"""Two-phase aggregation: partial aggregates (KRV_AGG_OUTPUT_PARTIAL) over
slices of the input emit each aggregate's state columns (COUNT: count; SUM:
sum, plus nonempty for decimals; AVG: sum, count; MIN/MAX: value), and a
final aggregate over the concatenated states (KRV_AGG_INPUT_STATE, the
reference's AggregateExpr::merging) gives the single-phase answer: Spark's
TPC-H Q1 answer, as the reference's own two-phase Q1 test checks, and the
single-phase GPU result on random data with NULLs, empty groups and a
decimal sum that overflows in one partial."""
import os
from decimal import Decimal

import numpy as np
import pyarrow as pa
import pytest

from helpers import concat, rel_err
from test_agg_keys_gpu import table_of, text

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def as_batch(t):
    return pa.RecordBatch.from_arrays([c.combine_chunks() for c in t.columns], schema=t.schema)


def aggregate(kb, rt, b, group_by, aggs, partial=False, ansi=True, mode=2):
    a = kb.HashAggregate(rt, kb.agg_spec(group_by, aggs, partial=partial, ansi=ansi, mode=mode))
    a.push(b)
    a.finish()
    return as_batch(concat(a.result()))


def two_phase(kb, rt, b, group_by, raw, merge, parts=3, ansi=True, mode=2):
    step = -(-b.num_rows // parts)
    states = [aggregate(kb, rt, b.slice(s, step), group_by, raw, partial=True, ansi=ansi, mode=mode)
              for s in range(0, b.num_rows, step)]
    mid = as_batch(pa.Table.from_batches(states))
    return mid, aggregate(kb, rt, mid, list(range(len(group_by))), merge, ansi=ansi, mode=mode)


@pytest.mark.parametrize("mode", [1, 2])
def test_tpch_q1_two_phase_spark_answer(kb, rt, mode):
    d = np.load(os.path.join(GOLDEN, "tpch_q1.npz"))
    b = table_of(d)
    raw = [("sum", 2), ("sum", 3), ("sum", 4), ("sum", 5), ("avg", 2), ("avg", 3), ("avg", 6), ("count_star", 0)]
    dec = (15, 2, 128)
    merge = [("sum", "state", 2, 3), ("sum", "state", 4, 5), ("sum", "state", 6, 7), ("sum", "state", 8, 9),
             ("avg", "state", 10, 11, dec), ("avg", "state", 12, 13, dec), ("avg", "state", 14, 15, dec),
             ("count_star", "state", 16)]
    mid, out = two_phase(kb, rt, b, [0, 1], raw, merge, parts=4, mode=mode)
    # the state columns (AggregateExpr::state_fields, aggregate/mod.rs:747-800)
    assert [f.type for f in mid.schema][2:] == [
        pa.decimal128(25, 2), pa.bool_(), pa.decimal128(25, 2), pa.bool_(), pa.decimal128(38, 4), pa.bool_(),
        pa.decimal128(38, 6), pa.bool_(), pa.decimal128(25, 2), pa.int64(), pa.decimal128(25, 2), pa.int64(),
        pa.decimal128(25, 2), pa.int64(), pa.int64()]
    assert [f.name for f in mid.schema][2:4] == ["sum(l_quantity)#sum", "sum(l_quantity)#nonempty"]
    rows = sorted(",".join(text(v) for v in r) for r in zip(*[c.to_pylist() for c in out.columns]))
    assert rows == d["expected"].tolist()


# (raw aggregates, their merges over the state columns): integer columns,
# then float64 and decimal ones; each set within 16 aggregated columns
# (state columns plus one overflow flag per decimal SUM)
INT_SET = ([("sum", 1), ("min", 1), ("max", 1), ("avg", 1), ("count", 1), ("sum", 2), ("avg", 2), ("min", 2),
            ("count_star", 0)],
           [("sum", "state", 1), ("min", "state", 2), ("max", "state", 3), ("avg", "state", 4, 5),
            ("count", "state", 6), ("sum", "state", 7), ("avg", "state", 8, 9), ("min", "state", 10),
            ("count_star", "state", 11)])
FLOAT_DEC_SET = ([("sum", 3), ("avg", 3), ("max", 3), ("sum", 4), ("avg", 4), ("count", 4), ("count_star", 0)],
                 [("sum", "state", 1), ("avg", "state", 2, 3), ("max", "state", 4), ("sum", "state", 5, 6),
                  ("avg", "state", 7, 8, (16, 3, 128)), ("count", "state", 9), ("count_star", "state", 10)])


@pytest.mark.parametrize("which", ["int", "float_dec"])
def test_two_phase_equals_one_phase(kb, rt, which):
    raw, merge = INT_SET if which == "int" else FLOAT_DEC_SET
    rng = np.random.default_rng(31)
    n = 120_000
    k = rng.integers(0, 3000, n)
    k[:500] = 77777  # a group whose values are all NULL below
    i64 = rng.integers(-2**40, 2**40, n)
    i32 = rng.integers(-1000, 1000, n).astype(np.int32)
    f = rng.random(n) * 1e6 - 5e5
    dec = rng.integers(-10**12, 10**12, n)
    masks = [rng.random(n) < 0.03 for _ in range(4)]
    for m in masks:
        m[:500] = True
    b = pa.RecordBatch.from_arrays(
        [pa.array(k), pa.array(i64, mask=masks[0]), pa.array(i32, mask=masks[1]), pa.array(f, mask=masks[2]),
         pa.Array.from_buffers(pa.decimal128(16, 3), n, [
             pa.py_buffer(np.packbits(~masks[3], bitorder="little").tobytes()),
             pa.py_buffer(np.stack([dec, np.where(dec < 0, -1, 0)], 1).astype(np.int64).reshape(-1).tobytes())])],
        names=["k", "a", "b", "c", "d"])
    one = aggregate(kb, rt, b, [0], raw)
    counts = [e for e, a in enumerate(raw) if a[0] in ("count", "count_star")]
    for mode in (1, 2):
        _, two = two_phase(kb, rt, b, [0], raw, merge, parts=5, mode=mode)
        assert two.schema.types == one.schema.types
        got = {r[0]: r[1:] for r in zip(*[c.to_pylist() for c in two.columns])}
        want = {r[0]: r[1:] for r in zip(*[c.to_pylist() for c in one.columns])}
        assert got.keys() == want.keys()
        # every value NULL: NULL results, zero counts (500 rows)
        for e, a in enumerate(raw):
            if e in counts:
                assert got[77777][e] == (500 if a[0] == "count_star" else 0)
            else:
                assert got[77777][e] is None
        for key, w in want.items():
            g = got[key]
            for e, (x, y) in enumerate(zip(g, w)):
                if isinstance(y, float):
                    assert rel_err(x, y) <= 1e-12, (key, e)
                else:
                    assert x == y, (key, e)


def test_overflowed_partial_sum(kb, rt):
    """A decimal(37,0) SUM (result decimal(38,0)) that overflows in one
    partial: NULL sum with nonempty set; the merge gives NULL for that group
    (ANSI off) and fails with ARITHMETIC_OVERFLOW (ANSI on)."""
    big = 9 * 10**36
    k = np.array([1] * 12 + [2, 2], dtype=np.int64)
    v = [big] * 12 + [5, 6]
    b = pa.RecordBatch.from_arrays([pa.array(k), pa.array([Decimal(x) for x in v], pa.decimal128(37, 0))],
                                   names=["k", "v"])
    mid = aggregate(kb, rt, b, [0], [("sum", 1)], partial=True, ansi=False)
    rows = {r[0]: r[1:] for r in zip(*[c.to_pylist() for c in mid.columns])}
    assert rows[1] == (None, True) and rows[2] == (Decimal(11), True)
    out = aggregate(kb, rt, mid, [0], [("sum", "state", 1, 2)], ansi=False)
    assert dict(zip(*[c.to_pylist() for c in out.columns])) == {1: None, 2: Decimal(11)}
    with pytest.raises(kb.KrvError) as e:
        aggregate(kb, rt, mid, [0], [("sum", "state", 1, 2)], ansi=True)
    assert e.value.status == kb.ARITHMETIC_OVERFLOW
