"""Generates the golden vectors under tests/golden/ (run in a checkout that
has the Krishiv engine reference tree; the outputs are committed, so tests
never read the reference).

    python tests/golden/make_golden.py /path/to/krishiv-engine

Writes:
  known_answers.json  -- the reference's own known-answer assertions for the
                         path (crates/krishiv-exec/src/join/keys.rs:345-370),
                         XXH64 (seed 0) vectors from python-xxhash, an
                         independent XXH64 implementation, for the widths of
                         crates/krishiv-io/src/runtime_filter/hash.rs:56-65.
  tpch_q13.npz / tpch_q18.npz -- the aggregate inputs of
                         crates/krishiv-exec/tests/aggregate_tpch.rs (Q13,
                         Q18) with Spark 4.2.0's expected answers, from
                         crates/krishiv-exec/tests/fixtures/tpch-sf0.01/.
  tpch_q1.npz / tpch_q18_keys.npz -- the inputs of Q1 (two string keys,
                         decimal sums and averages) and of Q18's outer
                         aggregate over all five keys (string, integers,
                         date, decimal), column by column (strings as
                         fixed-width unicode, decimals as unscaled (lo, hi)
                         int64 words), with Spark's expected rows as text.
"""
import csv
import json
import os
import sys

import numpy as np
import pyarrow as pa
import pyarrow.ipc as ipc
import xxhash

HERE = os.path.dirname(os.path.abspath(__file__))


def read_arrow(path):
    try:
        return ipc.open_file(path).read_all()
    except pa.ArrowInvalid:
        return ipc.open_stream(path).read_all()


def main(ref):
    fx = os.path.join(ref, "crates/krishiv-exec/tests/fixtures/tpch-sf0.01")
    # XXH64 of the little-endian bytes of signed values, per key width.
    values = [0, 1, -1, 2, 7, 42, 255, -128, 65535, -32768, 2**31 - 1, -2**31, 2**32, 2**53 + 1,
              2**62, -2**62, 2**63 - 1, -2**63, 123456789012345, -987654321098]
    xx = []
    for w in (1, 2, 4, 8):
        for v in values:
            b = (v & ((1 << (8 * w)) - 1)).to_bytes(w, "little")
            xx.append({"value": v, "width": w, "hash": xxhash.xxh64_intdigest(b, seed=0)})
    known = {
        "source": "crates/krishiv-exec/src/join/keys.rs:345-370; python-xxhash " + xxhash.VERSION,
        # keys.rs:348: h of the row (Float64 0.0, Int32 NULL), null_safe [false, true]
        "row_hash_f64_0_i32_null_nullsafe": 4733552696251797926,
        # keys.rs:362-368: level-0 partitions are the top radix bits of h
        "partition_cases": [
            {"h": 5 << 59, "radix": 5, "depth": 0, "partition": 5},
            {"h": 5 << 61, "radix": 3, "depth": 0, "partition": 5},
            {"h": (1 << 64) - 1, "radix": 3, "depth": 0, "partition": 7},
            {"h": (1 << 64) - 1, "radix": 6, "depth": 0, "partition": 63},
        ],
        "xxh64": xx,
    }
    with open(os.path.join(HERE, "known_answers.json"), "w") as f:
        json.dump(known, f, indent=1)

    # Q13: GROUP BY c_custkey COUNT(o_orderkey), then GROUP BY that count COUNT(*)
    t = read_arrow(os.path.join(fx, "q13_input.arrow"))
    cust = t.column("c_custkey").to_numpy(zero_copy_only=False)
    ok = t.column("o_orderkey")
    order = ok.fill_null(0).to_numpy(zero_copy_only=False)
    valid = ok.is_valid().to_numpy(zero_copy_only=False).astype(np.uint8)
    exp = [tuple(int(x) for x in r) for r in csv.reader(open(os.path.join(fx, "q13_expected.csv")))]
    np.savez_compressed(os.path.join(HERE, "tpch_q13.npz"), c_custkey=cust, o_orderkey=order,
                        o_orderkey_valid=valid, expected=np.array(sorted(exp), dtype=np.int64))
    # Q18: one group per order (o_orderkey determines the other four keys); SUM(l_quantity)
    t = read_arrow(os.path.join(fx, "q18_input.arrow"))
    okey = t.column("o_orderkey").to_numpy(zero_copy_only=False)
    qty = t.column("l_quantity")
    unscaled = np.array([int(v.as_py().scaleb(2)) for v in qty], dtype=np.int64)
    exp = []
    for r in csv.reader(open(os.path.join(fx, "q18_expected.csv"))):
        exp.append((int(r[2]), int(round(float(r[5]) * 100))))
    np.savez_compressed(os.path.join(HERE, "tpch_q18.npz"), o_orderkey=okey, l_quantity_unscaled=unscaled,
                        precision=np.int64(qty.type.precision), scale=np.int64(qty.type.scale),
                        expected=np.array(sorted(exp), dtype=np.int64))


def columns_of(t):
    """name -> numpy arrays of one Arrow table's columns (see the docstring)."""
    out = {}
    for f in t.schema:
        c = t.column(f.name).combine_chunks()
        out[f.name + "__valid"] = c.is_valid().to_numpy(zero_copy_only=False).astype(np.uint8)
        if pa.types.is_string(f.type):
            out[f.name + "__str"] = np.array([v if v is not None else "" for v in c.to_pylist()])
        elif pa.types.is_decimal(f.type):
            words = np.frombuffer(c.buffers()[1], dtype=np.int64)[2 * c.offset: 2 * (c.offset + len(c))]
            out[f.name + "__dec_lo"] = words[0::2].copy()
            out[f.name + "__dec_hi"] = words[1::2].copy()
            out[f.name + "__dec_ps"] = np.array([f.type.precision, f.type.scale], dtype=np.int64)
        elif pa.types.is_date32(f.type):
            out[f.name + "__date32"] = c.cast(pa.int32()).fill_null(0).to_numpy(zero_copy_only=False)
        else:
            out[f.name + "__" + str(f.type)] = c.fill_null(0).to_numpy(zero_copy_only=False)
    out["__order"] = np.array([f.name for f in t.schema])
    return out


def extra(ref):
    fx = os.path.join(ref, "crates/krishiv-exec/tests/fixtures/tpch-sf0.01")
    for q, name in (("q1", "tpch_q1.npz"), ("q18", "tpch_q18_keys.npz")):
        t = read_arrow(os.path.join(fx, q + "_input.arrow"))
        rows = [line.strip() for line in open(os.path.join(fx, q + "_expected.csv")) if line.strip()]
        np.savez_compressed(os.path.join(HERE, name), expected=np.array(sorted(rows)), **columns_of(t))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the reference checkout>")
    ref = sys.argv[1]
    main(ref)
    extra(ref)
