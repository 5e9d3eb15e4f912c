"""The grouped aggregate's partitioned path (batches of 256K rows and more in
the shared-memory mode): hot keys combined within warps into shared-memory
records, the other rows written to hash partitions and folded per partition
in shared memory, each group merged once into the global table. Checked
against the CPU oracle group by group (integers and decimals exact, float64
SUM/AVG within 1e-12 relative of the compensated oracle) over the cases that
reach each of its branches: Zipf keys (hot and cold rows), all-hot and
all-cold key sets, NULL keys and the table's marker key, a table that must
grow while partitions run (windows retried), partitions that overflow their
capacity (rows deferred to the global table), int32 keys and decimal128
values, and several batches mixing the partitioned and one-pass kernels."""
import numpy as np
import pyarrow as pa
import pytest

from helpers import batch
from test_agg_gpu import FUNCS, check_against_oracle, run, value_batch

pytestmark = pytest.mark.gpu
SHARED, GLOBAL = 2, 1
MARKER = -0x7F7F7F7F7F7F7F80  # 0x8080808080808080 as int64: the table's empty-slot key


def zipf_keys(rng, n, domain, s=1.1):
    ranks = rng.zipf(s, n * 2)
    ranks = ranks[ranks <= domain][:n]
    while len(ranks) < n:
        more = rng.zipf(s, n)
        ranks = np.concatenate([ranks, more[more <= domain]])[:n]
    perm = rng.permutation(domain).astype(np.int64) * 7919 - 3_000_000
    return perm[ranks - 1]


ALL = [("count_star", 0)] + [(f, c) for c in (1, 2, 3, 4) for f in FUNCS]
NAMES = ["dec", "f", "q", "i"]


@pytest.mark.parametrize("mode", [SHARED, GLOBAL])
def test_zipf_keys_hot_and_cold(kb, rt, oracle, mode):
    rng = np.random.default_rng(5)
    n = 2_000_000
    key = zipf_keys(rng, n, 200_000)
    b, raw = value_batch(n, key, rng)
    out = run(kb, rt, b, 0, ALL, mode, expected_groups=200_000)
    check_against_oracle(oracle, out, key, raw, ALL, NAMES)


def test_few_keys_all_hot_with_null_and_marker_keys(kb, rt, oracle):
    rng = np.random.default_rng(6)
    n = 1_000_000
    key = rng.integers(0, 12, n, dtype=np.int64)
    key[::1000] = MARKER
    kvalid = rng.random(n) > 0.01
    b, raw = value_batch(n, key, rng)
    b = pa.RecordBatch.from_arrays([pa.array(key, mask=~kvalid)] + b.columns[1:], names=b.schema.names)
    out = run(kb, rt, b, 0, ALL, SHARED)
    # the oracle groups by the valid keys; the NULL group is checked on its own
    sel = kvalid
    sub = {k: (v[0][sel], v[1][sel]) for k, v in raw.items()}
    nonnull = out.filter(pa.compute.is_valid(out.column(0)))
    check_against_oracle(oracle, nonnull, key[sel], sub, ALL, NAMES)
    null_row = out.filter(pa.compute.is_null(out.column(0)))
    assert null_row.num_rows == 1 and null_row.column(1)[0].as_py() == int((~kvalid).sum())


def test_uniform_keys_all_cold_table_grows(kb, rt, oracle):
    """1.5M distinct keys, no hot ones, a table sized for 1,000 groups: the
    partitions' merges run out of table room, stop, and run again after the
    table grows; every group still appears once with all its rows."""
    rng = np.random.default_rng(7)
    n = 3_000_000
    key = rng.integers(-(2**50), 2**50, 1_500_000, dtype=np.int64)[rng.integers(0, 1_500_000, n)]
    b, raw = value_batch(n, key, rng)
    aggs = [("count_star", 0), ("sum", 1), ("min", 2), ("max", 3), ("avg", 4), ("count", 2), ("sum", 2)]
    out = run(kb, rt, b, 0, aggs, SHARED, expected_groups=1000)
    check_against_oracle(oracle, out, key, raw, aggs, NAMES)


def test_later_batch_overflows_partitions(kb, rt, oracle):
    """The first batch is nearly all one key (few cold rows expected, small
    partitions); the second has only distinct cold keys, so partitions fill
    and their extra rows go to the global table."""
    rng = np.random.default_rng(8)
    n = 600_000
    k1 = np.where(rng.random(n) < 0.995, 42, rng.integers(0, 10**9, n)).astype(np.int64)
    k2 = rng.integers(0, 10**9, n, dtype=np.int64)
    key = np.concatenate([k1, k2])
    b, raw = value_batch(2 * n, key, rng)
    out = run(kb, rt, b, 0, ALL, SHARED, batches=2)
    check_against_oracle(oracle, out, key, raw, ALL, NAMES)


def test_int32_keys_and_decimal128_values(kb, rt, oracle):
    rng = np.random.default_rng(9)
    n = 700_000
    key = zipf_keys(rng, n, 50_000).astype(np.int32)
    big = rng.integers(-10**17, 10**17, n, dtype=np.int64)
    valid = rng.random(n) > 0.03
    words = np.stack([big, np.where(big < 0, -1, 0)], 1).astype(np.int64).reshape(-1)
    dec = pa.Array.from_buffers(pa.decimal128(38, 3), n, [pa.py_buffer(np.packbits(valid, bitorder="little").tobytes()),
                                                         pa.py_buffer(words.tobytes())])
    b = batch(k=pa.array(key), d=dec)
    aggs = [("sum", 1), ("count", 1), ("avg", 1), ("count_star", 0)]
    out = run(kb, rt, b, 0, aggs, SHARED)
    keys, _, res = oracle.hash_aggregate(key, None, [{"values": words,
                                                      "valid": valid.astype(np.uint8), "type": oracle.T_DEC128,
                                                      "precision": 38, "scale": 3}],
                                         [(oracle.SUM, 0), (oracle.COUNT, 0), (oracle.AVG, 0), (oracle.COUNT_STAR, 0)])
    order = {int(k): i for i, k in enumerate(keys)}
    got = out.to_pydict()
    names = out.schema.names
    assert sorted(got[names[0]]) == sorted(order)
    for j, k in enumerate(got[names[0]]):
        i = order[k]
        s = got[names[1]][j]
        want = int(res[0]["lo"][i]) + (int(res[0]["hi"][i]) << 64)
        assert (s is None) == (not res[0]["valid"][i])
        if s is not None:
            assert int(s.scaleb(3)) == want
        assert got[names[2]][j] == res[1]["i64"][i]
        a = got[names[3]][j]
        if a is not None:
            wa = int(res[2]["lo"][i]) + (int(res[2]["hi"][i]) << 64)
            assert int(a.scaleb(out.schema.field(3).type.scale)) == wa
        assert got[names[4]][j] == res[3]["i64"][i]


def test_batches_mix_partitioned_and_one_pass(kb, rt, oracle):
    rng = np.random.default_rng(10)
    sizes = [100_000, 900_000, 50_000, 400_000]
    key = zipf_keys(rng, sum(sizes), 80_000)
    b, raw = value_batch(len(key), key, rng)
    a = kb.HashAggregate(rt, kb.agg_spec(0, ALL, mode=SHARED))
    at = 0
    for s in sizes:
        a.push(b.slice(at, s))
        at += s
    a.finish()
    from helpers import concat
    out = concat(a.result())
    check_against_oracle(oracle, out, key, raw, ALL, NAMES)


def test_partitioned_equals_one_pass(kb, rt):
    """The same batch through the partitioned path and the global-table path:
    identical groups, integer results equal, float sums within 1e-12."""
    rng = np.random.default_rng(11)
    n = 1_500_000
    key = zipf_keys(rng, n, 300_000)
    b, _ = value_batch(n, key, rng)
    p = run(kb, rt, b, 0, ALL, SHARED).sort_by("k")
    g = run(kb, rt, b, 0, ALL, GLOBAL).sort_by("k")
    assert p.column(0).to_pylist() == g.column(0).to_pylist()
    for c in range(1, p.num_columns):
        x, y = p.column(c).to_pylist(), g.column(c).to_pylist()
        if pa.types.is_floating(p.schema.field(c).type):
            for u, v in zip(x, y):
                assert (u is None) == (v is None)
                if u is not None:
                    assert u == v or abs(u - v) <= 1e-12 * abs(v)
        else:
            assert x == y, p.schema.field(c).name
