"""The CPU oracle pinned against the reference's known answers and golden
vectors (tests/golden/, made by tests/golden/make_golden.py), and against
independent implementations (python-xxhash, a transcription of the Parquet
SBBF specification, a nested-loop join, Spark 4.2's TPC-H answers)."""
import collections
import itertools
import json
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def known():
    with open(os.path.join(GOLDEN, "known_answers.json")) as f:
        return json.load(f)


def test_row_hash_known_answer(oracle):
    # crates/krishiv-exec/src/join/keys.rs:348
    h = oracle.row_hash([(np.array([0.0]), None, True),
                         (np.array([0], dtype=np.int32), np.array([0], dtype=np.uint8), False)], [0, 1])
    assert int(h[0]) == known()["row_hash_f64_0_i32_null_nullsafe"]


def test_float_keys_normalize(oracle):
    # keys.rs:290-310: -0.0 and 0.0 hash alike, every NaN alike
    v = np.array([-0.0, 0.0, np.nan, -np.nan], dtype=np.float64)
    h = oracle.row_hash([(v, None, True)])
    assert h[0] == h[1] and h[2] == h[3] and h[0] != h[2]


def test_partition_known_answers(oracle):
    L = oracle.lib()
    for c in known()["partition_cases"]:
        assert L.orc_partition(c["h"], c["depth"], c["radix"], 1) == c["partition"]
    # deeper levels depend on the seed through g (keys.rs:368-369)
    assert any(L.orc_partition(x << 20, 1, 3, 1) != L.orc_partition(x << 20, 1, 3, 2) for x in range(64))
    for d in range(1, 8):
        assert 0 <= L.orc_partition((1 << 64) - 1, d, 3, 1) < 8


def test_xxh64_matches_python_xxhash(oracle):
    for case in known()["xxh64"]:
        got = oracle.xxh64_int(np.array([case["value"]], dtype=np.int64), case["width"])[0]
        assert int(got) == case["hash"], case


SALT = [0x47b6137b, 0x44974d91, 0x8824ad5b, 0xa2b7289d, 0x705495c7, 0x2df1424b, 0x9efc4947, 0x5c6bfb31]


def sbbf_spec_insert(words, nblocks, h):
    """The Parquet split-block Bloom filter insert, transcribed from the
    Parquet format specification (BloomFilter.md), in pure Python."""
    block = ((h >> 32) * nblocks) >> 32
    x = h & 0xFFFFFFFF
    for i in range(8):
        y = (x * SALT[i]) & 0xFFFFFFFF
        words[block * 8 + i] |= 1 << (y >> 27)


def test_sbbf_matches_parquet_spec(oracle):
    rng = np.random.default_rng(1)
    keys = rng.integers(-2**62, 2**62, 3000, dtype=np.int64)
    hashes = oracle.xxh64_int(keys)
    nbytes = oracle.bloom_bytes_for(len(keys), 0.01)
    words = oracle.bloom_build(hashes, nbytes)
    spec = [0] * (nbytes // 4)
    for h in hashes:
        sbbf_spec_insert(spec, nbytes // 32, int(h))
    assert words.tolist() == spec
    # zero false negatives (runtime_filter/tests.rs:54, :787)
    assert oracle.bloom_check(words, hashes).all()
    other = oracle.xxh64_int(rng.integers(-2**62, 2**62, 20000, dtype=np.int64))
    fpp = oracle.bloom_check(words, other).mean()
    assert fpp < 0.03


def test_bloom_sizing(oracle):
    # bloom.rs:96-110: Parquet's -8n/ln(1 - fpp^(1/8)) bits, whole 32-byte blocks
    for n, fpp in [(1, 0.01), (1000, 0.01), (50000, 0.01), (1000000, 0.01), (4000000, 0.05)]:
        bits = -8.0 * n / np.log(1.0 - fpp ** (1.0 / 8.0))
        want = max(1, -(-int(np.ceil(bits / 8.0)) // 32)) * 32
        assert oracle.bloom_bytes_for(n, fpp) == want
    assert oracle.bloom_bytes_for(1000000, 0.01) == 1210208


def test_key_filter_forms(oracle):
    # finish_with (filter.rs:533-593): dense range, exact set, Bloom, empty
    f = oracle.KeyFilter(np.arange(100, 200, dtype=np.int64))
    assert f.form == oracle.FORM_RANGE
    f = oracle.KeyFilter(np.array([5, 1000, 77, 5], dtype=np.int64))
    assert f.form == oracle.FORM_EXACT
    assert f.evaluate(np.array([5, 6, 77, 1000, 1001], dtype=np.int64)).tolist() == [1, 0, 1, 1, 0]
    keys = np.random.default_rng(2).permutation(1 << 20)[:100000].astype(np.int64)
    f = oracle.KeyFilter(keys)
    assert f.form == oracle.FORM_BLOOM
    assert f.evaluate(keys).all()
    f = oracle.KeyFilter(np.zeros(3, dtype=np.int64), np.zeros(3, dtype=np.uint8))
    assert f.form == oracle.FORM_EMPTY
    assert not f.evaluate(np.array([0, 1], dtype=np.int64)).any()


# ---- the join oracle against a nested loop (tests/hash_join/main.rs:128-181) ----
TYPES = ["inner", "left_outer", "left_semi", "left_anti", "null_aware_anti", "existence", "right_semi",
         "right_anti", "right_outer", "full_outer"]
TYPE_ID = {n: i for i, n in enumerate(TYPES)}


def nested_loop(jt, probe, build, null_safe):
    """probe/build: lists of key tuples (None = NULL). Returns the multiset of
    (probe_row, build_row) pairs with -1 for the padded side (existence: the
    flag)."""
    def eq(p, b):
        return all((x == y) if s else (x is not None and x == y) for x, y, s in zip(p, b, null_safe))
    out = []
    bmatched = [False] * len(build)
    for i, p in enumerate(probe):
        m = [j for j, b in enumerate(build) if eq(p, b)]
        for j in m:
            bmatched[j] = True
        if jt in ("inner", "left_outer", "right_outer", "full_outer"):
            out += [(i, j) for j in m]
        if jt in ("left_outer", "full_outer") and not m:
            out.append((i, -1))
        if jt == "left_semi" and m:
            out.append((i, -1))
        if jt == "left_anti" and not m:
            out.append((i, -1))
        if jt == "null_aware_anti":
            keep = len(build) == 0 or (not any(b[0] is None for b in build) and p[0] is not None and not m)
            if keep:
                out.append((i, -1))
        if jt == "existence":
            out.append((i, 1 if m else 0))
    for j, b in enumerate(build):
        if jt == "right_semi" and bmatched[j]:
            out.append((-1, j))
        if jt in ("right_anti", "right_outer", "full_outer") and not bmatched[j]:
            out.append((-1, j))
    return collections.Counter(out)


def to_cols(rows, nkeys):
    cols = []
    for k in range(nkeys):
        vals = np.array([r[k] if r[k] is not None else 0 for r in rows], dtype=np.int64 if k == 0 else np.int32)
        valid = np.array([r[k] is not None for r in rows], dtype=np.uint8)
        cols.append((vals, valid, False))
    return cols


EDGE_PROBE = [(1, 10), (1, 10), (2, None), (None, 10), (None, None), (7, 70)]
EDGE_BUILD = [(1, 10), (1, 10), (1, 11), (2, None), (None, None), (None, 10)]
ALL_NULL = [(None, None), (None, None)]


@pytest.mark.parametrize("jt", TYPES)
def test_join_oracle_matches_nested_loop_on_edge_cases(oracle, jt):
    inputs = [(EDGE_PROBE, EDGE_BUILD), (EDGE_PROBE, []), ([], EDGE_BUILD), (EDGE_PROBE, ALL_NULL),
              (ALL_NULL, EDGE_BUILD)]
    for nkeys in (1, 2):
        for safe in (False, True):
            if jt == "null_aware_anti" and (nkeys > 1 or safe):
                continue
            ns = [safe] * nkeys
            for probe, build in inputs:
                if not probe and not build:
                    continue
                want = nested_loop(jt, [p[:nkeys] for p in probe], [b[:nkeys] for b in build], ns)
                pc = to_cols(probe or [(0, 0)], nkeys)
                bc = to_cols(build or [(0, 0)], nkeys)
                pc = [(c[0][:len(probe)], c[1][:len(probe)], c[2]) for c in pc]
                bc = [(c[0][:len(build)], c[1][:len(build)], c[2]) for c in bc]
                p, b = oracle.hash_join(TYPE_ID[jt], bc, pc, null_safe=[int(x) for x in ns])
                got = collections.Counter(zip(p.tolist(), b.tolist()))
                assert got == want, (jt, nkeys, safe, len(probe), len(build))


def test_join_oracle_random_duplicates(oracle):
    rng = np.random.default_rng(3)
    for jt in TYPES:
        probe = [(int(x) if x >= 0 else None,) for x in rng.integers(-3, 40, 300)]
        build = [(int(x) if x >= 0 else None,) for x in rng.integers(-3, 40, 200)]
        want = nested_loop(jt, probe, build, [False])
        p, b = oracle.hash_join(TYPE_ID[jt], to_cols(build, 1), to_cols(probe, 1))
        assert collections.Counter(zip(p.tolist(), b.tolist())) == want, jt


def test_single_match_raises(oracle):
    with pytest.raises(RuntimeError, match="TOO_MANY_ROWS"):
        oracle.hash_join(TYPE_ID["left_outer"], [(np.array([1, 1], dtype=np.int64), None, False)],
                         [(np.array([1], dtype=np.int64), None, False)], single_match=True)


# ---- the aggregate oracle against Spark's answers ------------------------------------
def test_aggregate_oracle_tpch_q13(oracle):
    d = np.load(os.path.join(GOLDEN, "tpch_q13.npz"))
    keys, kv, res = oracle.hash_aggregate(
        d["c_custkey"], None,
        [{"values": d["o_orderkey"], "valid": d["o_orderkey_valid"], "type": oracle.T_I64}],
        [(oracle.COUNT, 0)])
    counts = res[0]["i64"]
    k2, _, r2 = oracle.hash_aggregate(counts.astype(np.int64), None, [], [(oracle.COUNT_STAR, 0)])
    got = sorted(zip(k2.tolist(), r2[0]["i64"].tolist()))
    assert got == [tuple(r) for r in d["expected"].tolist()]


def test_aggregate_oracle_tpch_q18(oracle):
    d = np.load(os.path.join(GOLDEN, "tpch_q18.npz"))
    q = d["l_quantity_unscaled"]
    dec128 = np.zeros((len(q), 2), dtype=np.int64)
    dec128[:, 0] = q
    dec128[:, 1] = np.where(q < 0, -1, 0)
    keys, kv, res = oracle.hash_aggregate(
        d["o_orderkey"], None,
        [{"values": dec128, "type": oracle.T_DEC128, "precision": int(d["precision"]), "scale": int(d["scale"])}],
        [(oracle.SUM, 0)])
    got = sorted(zip(keys.tolist(), res[0]["lo"].astype(np.int64).tolist()))
    assert got == [tuple(r) for r in d["expected"].tolist()]


def test_aggregate_oracle_against_numpy(oracle):
    rng = np.random.default_rng(4)
    n = 20000
    key = rng.integers(0, 300, n).astype(np.int64)
    q = rng.integers(1, 51, n).astype(np.int32)
    qv = (rng.random(n) > 0.02).astype(np.uint8)
    f = rng.random(n)
    keys, kv, res = oracle.hash_aggregate(
        key, None, [{"values": q, "valid": qv, "type": oracle.T_I32}, {"values": f, "type": oracle.T_F64}],
        [(oracle.SUM, 0), (oracle.COUNT, 0), (oracle.MIN, 0), (oracle.MAX, 0), (oracle.AVG, 0), (oracle.SUM, 1)])
    for gi, k in enumerate(keys):
        m = key == k
        mv = m & (qv == 1)
        assert res[0]["i64"][gi] == q[mv].sum()
        assert res[1]["i64"][gi] == mv.sum()
        assert res[2]["i64"][gi] == q[mv].min() and res[3]["i64"][gi] == q[mv].max()
        assert res[4]["f64"][gi] == q[mv].astype(np.float64).sum() / mv.sum()
        exact = float(np.sum(f[m].astype(np.longdouble)))
        assert abs(res[5]["f64"][gi] - exact) <= 1e-12 * abs(exact)


def test_avg_decimal_half_up(oracle):
    L = oracle.lib()
    import ctypes as C
    lo, hi = C.c_uint64(), C.c_int64()
    cases = [  # (sum, sum scale, count, p, s) -> HALF_UP(sum * 10^(s-ss) / count)
        (5, 2, 2, 19, 6, 25000), (1, 2, 3, 19, 6, 3333), (2, 2, 3, 19, 6, 6667), (-2, 2, 3, 19, 6, -6667),
        (10, 0, 4, 14, 4, 25000), (1, 0, 8, 14, 4, 1250), (-1, 0, 16, 14, 4, -625),
    ]
    for s, ss, c, p, rs, want in cases:
        assert L.orc_avg_decimal(s, -1 if s < 0 else 0, ss, c, p, rs, C.byref(lo), C.byref(hi)) == 1
        assert (hi.value << 64) + lo.value == want, (s, ss, c, p, rs)
    # the digit loop (scale above 19) agrees with exact rational rounding
    from fractions import Fraction
    for s, c in [(7, 3), (123456789, 7), (-5, 9)]:
        assert L.orc_avg_decimal(s, -1 if s < 0 else 0, 2, c, 38, 25, C.byref(lo), C.byref(hi)) == 1
        q = Fraction(abs(s) * 10 ** 23, c)
        r = int(q) + (1 if q - int(q) >= Fraction(1, 2) else 0)
        assert (hi.value << 64) + lo.value == (r if s >= 0 else -r)


def test_generators_are_deterministic_and_permute(oracle):
    L = oracle.lib()
    assert L.orc_rand(7, 1, 5) == L.orc_rand(7, 1, 5)
    assert L.orc_rand(7, 1, 5) != L.orc_rand(7, 2, 5)
    for n in (1, 2, 3, 10, 1000, 4097):
        vals = sorted(L.orc_permute(99, n, i) for i in range(n))
        assert vals == list(range(n))
    cdf = oracle.zipf_cdf(1.1, 1000)
    assert np.all(np.diff(cdf) > 0) and cdf[-1] == 1.0
    assert abs(cdf[0] - 1.0 / sum(k ** -1.1 for k in range(1, 1001))) < 1e-12
