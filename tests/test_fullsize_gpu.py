"""The plain join and the grouped aggregate at their full benchmark sizes,
checked through size-independent properties and exact multiset equality
computed on the device, plus the CPU oracle on a sample of groups.

Join: build 1,000,000 rows (k a permutation of [0, 1M), v int64), probe
10,000,000 rows (k uniform [0, 2M), w int32); the inner join's output is
exactly {(k, w, v_of(k)) : probe rows with k < 1M}.
Aggregate: 100,000,000 rows, Zipf(1.1) keys over 1M values, decimal(15,2),
float64 and int32 columns with 2% NULLs, SUM/COUNT/MIN/MAX/AVG of each:
every one of the ~1M groups against the CPU oracle over all 100M rows
(integers and decimals exact, float64 SUM/AVG within 1e-12 relative of the
oracle's compensated sums, the Zipf head keys with millions of rows each
included), in both aggregation modes."""
import importlib

import numpy as np
import pytest

from helpers import rel_err

pytestmark = pytest.mark.gpu


def W():
    return importlib.import_module("krishiv-engine_b200.workloads")


def test_join_full_size_multiset(kb, rt):
    import torch
    build, probe = W().join(rt, scale=1.0)
    (_, bk, _), (_, bv, _) = build
    (_, pk, _), (_, pw, _) = probe
    nb = bk.shape[0]
    j = kb.HashJoin(rt, kb.join_spec("inner", probe_out=[0, 1], build_out=[1], build_rows_hint=nb))
    j.build_push_device(kb.DeviceBatch(build))
    j.build_finish()
    out = j.probe_device(kb.DeviceBatch(probe))
    rt.synchronize()
    ok, ow, ov = out.columns
    v_of = torch.empty(nb, dtype=torch.int64, device="cuda")
    v_of[bk] = bv
    m = pk < nb
    ek, ew = pk[m], pw[m]
    ev = v_of[ek]
    assert out.rows == int(m.sum())

    def order(k, w):
        return torch.argsort(k * (1 << 32) + (w.to(torch.int64) + (1 << 31)))
    a, b = order(ok, ow), order(ek, ew)
    assert torch.equal(ok[a], ek[b]) and torch.equal(ow[a], ew[b]) and torch.equal(ov[a], ev[b])


def unpack_valid(bitmap, n):
    import torch
    bits = (bitmap[: (n + 7) // 8].unsqueeze(1) >> torch.arange(8, device=bitmap.device, dtype=torch.uint8)) & 1
    return bits.reshape(-1)[:n].bool()


@pytest.mark.parametrize("mode", [1, 2])
def test_aggregate_full_size_properties(kb, rt, oracle, mode):
    import torch
    cols = W().agg(rt, scale=1.0)
    n = cols[0][1].shape[0]
    aggs = [(f, c) for c in (1, 2, 3) for f in ("sum", "count", "min", "max", "avg")]
    a = kb.HashAggregate(rt, kb.agg_spec(0, aggs, mode=mode, expected_groups=1_000_000))
    a.push_device(kb.DeviceBatch(cols))
    a.finish()
    res = a.result_device()
    rt.synchronize()
    keys = res.columns[0]
    k = cols[0][1]
    distinct = torch.unique(k)
    assert res.rows == distinct.numel()
    assert torch.equal(torch.sort(keys).values, distinct)
    def col_valid(i):
        vb = res.valid[i]
        return unpack_valid(vb, res.rows) if vb is not None else torch.ones(res.rows, dtype=torch.bool, device="cuda")

    # per value column: sum of COUNT = valid rows; SUM totals; MIN / MAX extremes
    for (name, t, vbits, *_), base in ((cols[1], 1), (cols[2], 6), (cols[3], 11)):
        valid = unpack_valid(vbits, n)
        cnt = res.columns[base + 1]
        assert int(cnt.sum()) == int(valid.sum())
        vals = t[valid]
        sv = col_valid(base)
        assert int(sv.sum()) == int((cnt > 0).sum())  # SUM is NULL exactly where no value was valid
        if name == "dec":  # decimal(25,2) sums as (lo, hi) int64 pairs
            s = res.columns[base].view(-1, 2)[sv].cpu().numpy()
            got = sum(int(x) for x in s[:, 1]) * 2**64 + sum(int(x) & (2**64 - 1) for x in s[:, 0])
            assert got == int(vals.sum())
        elif name == "f":
            # both totals in extended precision, so the check is as tight as the per-group one
            got = np.sum(res.columns[base][sv].cpu().numpy().astype(np.longdouble))
            want = np.sum(vals.cpu().numpy().astype(np.longdouble))
            assert rel_err(got, want) <= 1e-12
        else:
            assert int(res.columns[base][sv].sum()) == int(vals.sum())
        mn, mx = res.columns[base + 2][col_valid(base + 2)], res.columns[base + 3][col_valid(base + 3)]
        if name == "f":
            assert float(mn.min()) == float(vals.min()) and float(mx.max()) == float(vals.max())
        else:
            assert int(mn.min()) == int(vals.min()) and int(mx.max()) == int(vals.max())


AGGS = [(f, c) for c in (1, 2, 3) for f in ("sum", "count", "min", "max", "avg")]
_ORACLE = {}


def oracle_full(oracle, cols):
    """The oracle's aggregate over every row of the workload (computed once)."""
    if "res" not in _ORACLE:
        n = cols[0][1].shape[0]
        k = cols[0][1].cpu().numpy()
        sub = []
        for (name, t, vbits, *_), typ in zip(cols[1:], (oracle.T_DEC64, oracle.T_F64, oracle.T_I32)):
            c = {"values": t.cpu().numpy(), "valid": unpack_valid(vbits, n).cpu().numpy().astype(np.uint8),
                 "type": typ}
            if name == "dec":
                c.update(precision=15, scale=2)
            sub.append(c)
        F = {"sum": oracle.SUM, "count": oracle.COUNT, "min": oracle.MIN, "max": oracle.MAX, "avg": oracle.AVG}
        wk, _, wr = oracle.hash_aggregate(k, None, sub, [(F[f], c - 1) for f, c in AGGS])
        counts = np.bincount(np.searchsorted(np.sort(wk), k), minlength=len(wk))
        _ORACLE["res"] = (wk, wr, counts)
    return _ORACLE["res"]


@pytest.mark.parametrize("mode", [1, 2])
def test_aggregate_full_size_every_group(kb, rt, oracle, mode):
    """All ~1M groups against the oracle over all 100M rows."""
    cols = W().agg(rt, scale=1.0)
    a = kb.HashAggregate(rt, kb.agg_spec(0, AGGS, mode=mode, expected_groups=1_000_000))
    a.push_device(kb.DeviceBatch(cols))
    a.finish()
    res = a.result_device()
    rt.synchronize()
    wk, wr, rows_per_key = oracle_full(oracle, cols)
    keys = res.columns[0].cpu().numpy()
    assert len(keys) == len(wk)
    go, wo = np.argsort(keys), np.argsort(wk)
    assert np.array_equal(keys[go], wk[wo])
    # the heaviest keys (each with millions of rows) are among the groups checked
    assert rows_per_key.max() > 5_000_000
    for e, (f, c) in enumerate(AGGS):
        name = cols[c][0]
        w = wr[e]
        vb = res.valid[1 + e]
        gv = (unpack_valid(vb, res.rows).cpu().numpy() if vb is not None else np.ones(res.rows, bool))[go]
        wv = w["valid"][wo]
        assert np.array_equal(gv, wv), (f, name)
        col = res.columns[1 + e].cpu().numpy()
        if f == "count":
            assert np.array_equal(col[go], w["i64"][wo]), (f, name)
        elif name == "dec" and f in ("sum", "avg"):
            pair = col.reshape(-1, 2)[go]
            assert np.array_equal(pair[:, 0][gv].view(np.uint64), w["lo"][wo][wv].view(np.uint64)), (f, name)
            assert np.array_equal(pair[:, 1][gv], w["hi"][wo][wv]), (f, name)
        elif (name == "f" and f in ("sum", "avg")) or (name == "q" and f == "avg"):
            got, want = col[go][gv].astype(np.float64), w["f64"][wo][wv]
            rel = np.abs(got - want) / np.maximum(np.abs(want), 1e-300)
            worst = int(np.argmax(rel))
            assert rel[worst] <= 1e-12, (f, name, float(got[worst]), float(want[worst]))
        elif name == "f":
            assert np.array_equal(col[go][gv], w["f64"][wo][wv]), (f, name)
        else:
            assert np.array_equal(col[go][gv].astype(np.int64), w["i64"][wo][wv]), (f, name)
