"""String and binary payload columns in join output: probe-side columns
gathered by probe row, build-side columns from the build arena's byte heap
by build row (the reference decodes build payloads for the matched rows,
crates/krishiv-exec/src/join/mod.rs:907-927), NULLs for the padded side of
outer joins, across every join type that emits rows. Checked against the
oracle's (probe row, build row) pairs: each output row's strings must be
those of its rows."""
import collections

import numpy as np
import pyarrow as pa
import pytest

from helpers import concat

pytestmark = pytest.mark.gpu

TYPES = {"inner": 0, "left_outer": 1, "left_semi": 2, "left_anti": 3, "existence": 5, "right_semi": 6,
         "right_anti": 7, "right_outer": 8, "full_outer": 9}


def strings(rng, n, prefix):
    lens = rng.integers(0, 40, n)
    vals = [prefix + "".join(chr(97 + int(c)) for c in rng.integers(0, 26, L)) for L in lens]
    vals[::17] = [""] * len(vals[::17])  # empty strings
    if n > 5:
        vals[3] = prefix + "é" * 30  # multi-byte UTF-8
    return vals


def side(rng, n, key_hi, prefix, idname):
    k = rng.integers(0, key_hi, n).astype(np.int64)
    kv = rng.random(n) > 0.03
    s = strings(rng, n, prefix)
    sv = rng.random(n) > 0.1
    b = [bytes(rng.integers(0, 256, int(rng.integers(0, 12))).astype(np.uint8)) for _ in range(n)]
    return pa.RecordBatch.from_arrays(
        [pa.array(k, mask=~kv), pa.array(s, type=pa.string(), mask=~sv), pa.array(b, type=pa.binary()),
         pa.array(np.arange(n, dtype=np.int64))], names=["k", "s", "b", idname]), (k, kv)


@pytest.mark.parametrize("jt", list(TYPES))
def test_string_payloads(kb, rt, oracle, jt):
    rng = np.random.default_rng(TYPES[jt] + 40)
    probe, (pk, pv) = side(rng, 5000, 700, "p", "pid")
    build, (bk, bv) = side(rng, 2000, 700, "b", "bid")
    j = kb.HashJoin(rt, kb.join_spec(jt))
    j.build_push(build.slice(0, 700))
    j.build_push(build.slice(700))  # two batches: the heap grows, offsets rebased
    j.build_finish()
    outs = j.probe(probe.slice(0, 2501)) + j.probe(probe.slice(2501))
    outs += j.finish()
    t = concat(outs)
    p, b = oracle.hash_join(TYPES[jt], [(bk, bv.astype(np.uint8), False)], [(pk, pv.astype(np.uint8), False)])
    want = collections.Counter(zip(p.tolist(), b.tolist()))
    names = t.column_names
    ps, pb = probe.column("s").to_pylist(), probe.column("b").to_pylist()
    bs, bb = build.column("s").to_pylist(), build.column("b").to_pylist()
    got = collections.Counter()
    for r in range(t.num_rows):
        pid = t.column("pid")[r].as_py() if "pid" in names else None
        bid = t.column("bid")[r].as_py() if "bid" in names else None
        # the strings of each side are the strings of that side's row
        if "pid" in names:
            s_col = names.index("s")
            if pid is None:
                assert t.column(s_col)[r].as_py() is None
            else:
                assert t.column(s_col)[r].as_py() == ps[pid] and t.column(names.index("b"))[r].as_py() == pb[pid]
        if "bid" in names:
            s_col = len(names) - 1 - names[::-1].index("s")
            b_col = len(names) - 1 - names[::-1].index("b")
            if bid is None:
                assert t.column(s_col)[r].as_py() is None and t.column(b_col)[r].as_py() is None
            else:
                assert t.column(s_col)[r].as_py() == bs[bid] and t.column(b_col)[r].as_py() == bb[bid]
        if jt == "existence":
            got[(pid, int(t.column("exists")[r].as_py()))] += 1
        else:
            got[(-1 if pid is None else pid, -1 if bid is None else bid)] += 1
    assert got == want


def test_string_payloads_with_duplicate_build_keys(kb, rt):
    """Several build rows per key: each probe row gets every build string of
    its key once."""
    j = kb.HashJoin(rt, kb.join_spec("inner"))
    j.build_push(pa.RecordBatch.from_arrays([pa.array([2, 3, 3], type=pa.int64()),
                                             pa.array(["x", "yy", "zzz"])], names=["k", "s"]))
    j.build_finish()
    out = concat(j.probe(pa.RecordBatch.from_arrays([pa.array([1, 2, 3], type=pa.int64())], names=["k"])))
    got = sorted(zip(out.column(0).to_pylist(), out.column(out.num_columns - 1).to_pylist()))
    assert got == [(2, "x"), (3, "yy"), (3, "zzz")]
