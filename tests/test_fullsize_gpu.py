"""The plain join and the grouped aggregate at their full benchmark sizes,
checked through size-independent properties and exact multiset equality
computed on the device, plus the CPU oracle on a sample of groups.

Join: build 1,000,000 rows (k a permutation of [0, 1M), v int64), probe
10,000,000 rows (k uniform [0, 2M), w int32); the inner join's output is
exactly {(k, w, v_of(k)) : probe rows with k < 1M}.
Aggregate: 100,000,000 rows, Zipf(1.1) keys over 1M values, decimal(15,2),
float64 and int32 columns with 2% NULLs, SUM/COUNT/MIN/MAX/AVG of each."""
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
            got = float(np.sum(res.columns[base][sv].cpu().numpy()))
            assert rel_err(got, float(np.sum(vals.cpu().numpy()))) <= 1e-11
        else:
            assert int(res.columns[base][sv].sum()) == int(vals.sum())
        mn, mx = res.columns[base + 2][col_valid(base + 2)], res.columns[base + 3][col_valid(base + 3)]
        if name == "f":
            assert float(mn.min()) == float(vals.min()) and float(mx.max()) == float(vals.max())
        else:
            assert int(mn.min()) == int(vals.min()) and int(mx.max()) == int(vals.max())
    # 300 sampled groups against the oracle, exactly (float within 1e-12)
    rng = np.random.default_rng(1)
    pick = torch.tensor(rng.choice(distinct.cpu().numpy(), 300, replace=False), device="cuda")
    rows = torch.isin(k, pick)
    sub_k = k[rows].cpu().numpy()
    sub = []
    for (name, t, vbits, *_), typ in zip(cols[1:], (oracle.T_DEC64, oracle.T_F64, oracle.T_I32)):
        v = t[rows].cpu().numpy()
        m = unpack_valid(vbits, n)[rows].cpu().numpy().astype(np.uint8)
        c = {"values": v, "valid": m, "type": typ}
        if name == "dec":
            c.update(precision=15, scale=2)
        sub.append(c)
    F = {"sum": oracle.SUM, "count": oracle.COUNT, "min": oracle.MIN, "max": oracle.MAX, "avg": oracle.AVG}
    wk, _, wr = oracle.hash_aggregate(sub_k, None, sub, [(F[f], c - 1) for f, c in aggs])
    pos = {int(x): i for i, x in enumerate(keys.cpu().numpy())}
    idx = [pos[int(x)] for x in wk]
    for e, (f, c) in enumerate(aggs):
        col = res.columns[1 + e].cpu().numpy()
        cv = col_valid(1 + e).cpu().numpy()
        name = cols[c][0]
        w = wr[e]
        assert [bool(cv[i]) for i in idx] == [bool(x) for x in w["valid"]], (f, c)
        for j, i in enumerate(idx):
            if not w["valid"][j]:
                continue
            if f == "count":
                assert int(col[i]) == int(w["i64"][j]), (f, c)
            elif name == "dec" and f in ("sum", "avg"):
                pair = col.reshape(-1, 2)[i]
                assert int(pair[1]) * 2**64 + (int(pair[0]) & (2**64 - 1)) == int(w["i128"][j]), (f, c)
            elif (name == "f" and f in ("sum", "avg")) or (name == "q" and f == "avg"):
                assert rel_err(float(col[i]), float(w["f64"][j])) <= 1e-12, (f, c)
            elif name == "f":
                assert float(col[i]) == float(w["f64"][j]), (f, c)
            else:
                assert int(col[i]) == int(w["i64"][j]), (f, c)
