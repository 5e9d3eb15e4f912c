"""Residual join filters (JoinSpec::filter, crates/krishiv-exec/src/join/
probe.rs:393-489, the filter at :425-436) against the CPU oracle: a candidate
pair of equal keys counts only where every comparison of the filter is TRUE;
a NULL operand is not TRUE; outer padding, semi/anti/existence results and
the build-side marks of right and full joins follow the filtered matches.
Results are compared as multisets of (probe row, build row) pairs, exactly."""
import collections

import numpy as np
import pyarrow as pa
import pytest

from helpers import batch, concat, pairs_from_output

pytestmark = pytest.mark.gpu

TYPES = ["inner", "left_outer", "left_semi", "left_anti", "existence", "right_semi", "right_anti", "right_outer",
         "full_outer"]
TYPE_ID = {"inner": 0, "left_outer": 1, "left_semi": 2, "left_anti": 3, "existence": 5, "right_semi": 6,
           "right_anti": 7, "right_outer": 8, "full_outer": 9}


def side(rng, n, key_hi, null_key=0.03):
    """One side's columns: k (int64, some NULL), a (int64), i (int32), f
    (float64 with -0.0, NaN and NULLs), d (decimal(12,2) unscaled), id."""
    k = rng.integers(0, key_hi, n).astype(np.int64)
    kv = rng.random(n) > null_key
    a = rng.integers(-50, 50, n).astype(np.int64)
    av = rng.random(n) > 0.05
    i = rng.integers(-1000, 1000, n).astype(np.int32)
    f = rng.standard_normal(n)
    f[rng.random(n) < 0.02] = -0.0
    f[rng.random(n) < 0.02] = 0.0
    f[rng.random(n) < 0.02] = np.nan
    fv = rng.random(n) > 0.05
    d = rng.integers(-100000, 100000, n).astype(np.int64)
    return {"k": (k, kv), "a": (a, av), "i": (i, None), "f": (f, fv), "d": (d, None)}


def arrow(cols, idname):
    def col(name):
        v, m = cols[name]
        if name == "d":
            return pa.Array.from_buffers(pa.decimal64(12, 2), len(v), [None, pa.py_buffer(v.tobytes())])
        return pa.array(v, mask=None if m is None else ~m)
    names = ["k", "a", "i", "f", "d"]
    arrays = [col(n) for n in names] + [pa.array(np.arange(len(cols["k"][0]), dtype=np.int64))]
    return pa.RecordBatch.from_arrays(arrays, names=names + [idname])


IDX = {"k": 0, "a": 1, "i": 2, "f": 3, "d": 4}
FILTERS = [
    # probe.a < build.a
    [(("probe", "a"), "<", ("build", "a"))],
    # probe.i >= 0 and build.f != probe.f (floats, Spark order) and build.a <= 30
    [(("probe", "i"), ">=", 0), (("build", "f"), "!=", ("probe", "f")), (("build", "a"), "<=", 30)],
    # probe.f > 0.25 (int vs float promotion: build.i > probe.f)
    [(("probe", "f"), ">", 0.25), (("build", "i"), ">", ("probe", "f"))],
    # decimals of one scale, and a constant at that scale
    [(("probe", "d"), "=", ("build", "d"))],
    [(("build", "d"), ">", 1234), (("probe", "d"), "<=", ("build", "d"))],
    # always false, always true
    [(("probe", "a"), "<", -1000)],
    [(("probe", "i"), ">=", -1000)],
]


def gpu_terms(filt):
    out = []
    for l, op, r in filt:
        def o(x):
            return (x[0], IDX[x[1]]) if isinstance(x, tuple) else x
        out.append((o(l), op, o(r)))
    return out


def oracle_pairs(oracle, jt, probe, build, filt):
    names = ["k", "a", "i", "f", "d"]
    pcols = [probe[n] for n in names]
    bcols = [build[n] for n in names]
    f = oracle.make_filter(gpu_terms(filt), pcols, bcols)
    p, b = oracle.hash_join(TYPE_ID[jt], [(build["k"][0], build["k"][1].astype(np.uint8), False)],
                            [(probe["k"][0], probe["k"][1].astype(np.uint8), False)], filter=f)
    return collections.Counter(zip(p.tolist(), b.tolist()))


def gpu_pairs(kb, rt, jt, probe, build, filt, build_batches=1):
    j = kb.HashJoin(rt, kb.join_spec(jt), filter=gpu_terms(filt))
    b = arrow(build, "bid")
    step = max(1, -(-b.num_rows // build_batches))
    for s in range(0, b.num_rows, step):
        j.build_push(b.slice(s, step))
    j.build_finish()
    outs = j.probe(arrow(probe, "pid"))
    outs += j.finish()
    t = concat(outs)
    if jt == "existence":
        return collections.Counter(zip(t.column("pid").to_pylist(), [int(x) for x in t.column("exists").to_pylist()]))
    return pairs_from_output(t)


@pytest.mark.parametrize("jt", TYPES)
def test_filtered_join_types(kb, rt, oracle, jt):
    rng = np.random.default_rng(TYPE_ID[jt] + 100)
    probe = side(rng, 6000, 800)
    build = side(rng, 2500, 800)
    for fi, filt in enumerate(FILTERS):
        want = oracle_pairs(oracle, jt, probe, build, filt)
        got = gpu_pairs(kb, rt, jt, probe, build, filt, build_batches=2)
        assert got == want, (jt, fi)


def test_filter_on_unique_keys_and_single_match(kb, rt, oracle):
    """Unique int64 build keys (the no-chain probe is not used with a filter)
    and a single-match left outer join, whose error follows the filtered
    matches: two key matches of which one passes the filter are fine."""
    rng = np.random.default_rng(5)
    n = 4000
    build = side(rng, n, 10, null_key=0.0)
    build["k"] = (rng.permutation(n).astype(np.int64), np.ones(n, bool))
    probe = side(rng, 20000, n)
    filt = [(("probe", "a"), "<", ("build", "a"))]
    for jt in ("inner", "left_outer"):
        assert gpu_pairs(kb, rt, jt, probe, build, filt) == oracle_pairs(oracle, jt, probe, build, filt)
    # single match: build key 1 twice, one row passing the filter
    b = batch(k=pa.array([1, 1, 2], type=pa.int64()), a=pa.array([5, 50, 0], type=pa.int64()))
    p = batch(k=pa.array([1, 2, 3], type=pa.int64()), a=pa.array([10, 0, 0], type=pa.int64()))
    j = kb.HashJoin(rt, kb.join_spec("left_outer", single_match=True), filter=[(("probe", 1), "<", ("build", 1))])
    j.build_push(b)
    j.build_finish()
    out = concat(j.probe(p))
    assert sorted(zip(out.column(0).to_pylist(), out.column(3).to_pylist())) == [(1, 50), (2, None), (3, None)]
    j = kb.HashJoin(rt, kb.join_spec("left_outer", single_match=True), filter=[(("probe", 1), ">", 1)])
    j.build_push(b)
    j.build_finish()
    with pytest.raises(kb.KrvError) as e:
        j.probe(p)
    assert e.value.status == kb.TOO_MANY_ROWS


def test_filter_rejections(kb, rt):
    import pyarrow as pa
    # a string column in a filter
    j = kb.HashJoin(rt, kb.join_spec("inner"), filter=[(("probe", 1), "=", ("build", 1))])
    j.build_push(batch(k=pa.array([1], type=pa.int64()), s=pa.array([2], type=pa.int64())))
    j.build_finish()
    with pytest.raises(kb.KrvError) as e:
        j.probe(batch(k=pa.array([1], type=pa.int64()), s=pa.array([True])))
    assert e.value.status == kb.UNSUPPORTED
    # column out of range
    j = kb.HashJoin(rt, kb.join_spec("inner"), filter=[(("probe", 7), "=", 1)])
    j.build_push(batch(k=pa.array([1], type=pa.int64())))
    j.build_finish()
    with pytest.raises(kb.KrvError) as e:
        j.probe(batch(k=pa.array([1], type=pa.int64())))
    assert e.value.status == kb.INVALID_ARGUMENT
    # a partitioned join
    with pytest.raises(kb.KrvError) as e:
        kb.HashJoin(rt, kb.join_spec("inner"), partitioned=True, filter=[(("probe", 0), ">", 0)])
    assert e.value.status == kb.UNSUPPORTED
