"""The star-join pipeline (runtime filters + two joins + grouped sum), fused
and plain, against the CPU oracle on the same seeded inputs: the rows passing
the filters and the joined rows are counted exactly; each group's sum is
within 1e-12 relative of the oracle's compensated sum."""
import importlib

import numpy as np
import pytest

from helpers import rel_err

pytestmark = pytest.mark.gpu
FLOAT_TOL = 1e-12


def unpack(valid, n):
    """A device validity bitmap as a boolean array (all True when None)."""
    if valid is None:
        return np.ones(n, dtype=bool)
    return np.unpackbits(valid.cpu().numpy(), bitorder="little")[:n].astype(bool)


def oracle_star(oracle, data, group_by=0):
    fk_a, fk_b, price, disc = [c[1].cpu().numpy() for c in data.fact]
    va, vb, vp, vd = [unpack(c[2], data.fact_rows) for c in data.fact]
    dims = []
    for d in (data.dim_a, data.dim_b):
        key, pred, attr = [c[1].cpu().numpy() for c in d]
        sel = pred == 7
        dims.append((key[sel], attr[sel]))
    (ka, aa), (kb_, ab) = dims
    fa, fb = oracle.KeyFilter(ka), oracle.KeyFilter(kb_)
    passed = fa.evaluate(fk_a, va) & fb.evaluate(fk_b, vb)
    oa, ob = np.argsort(ka), np.argsort(kb_)
    ia = np.searchsorted(ka, fk_a, sorter=oa)
    ib = np.searchsorted(kb_, fk_b, sorter=ob)
    ia = np.minimum(ia, len(ka) - 1)
    ib = np.minimum(ib, len(kb_) - 1)
    # a NULL key never joins (join/keys.rs:17-19)
    hit = (ka[oa[ia]] == fk_a) & (kb_[ob[ib]] == fk_b) & va & vb
    assert not (hit & ~passed).any(), "a runtime filter dropped a joining row"
    group = (aa[oa[ia]] if group_by == 0 else ab[ob[ib]])[hit].astype(np.int64)
    value = price[hit].astype(np.float64) * (1.0 - disc[hit])
    value_valid = (vp & vd)[hit]  # a NULL price or discount: a NULL value, skipped by SUM
    keys, _, res = oracle.hash_aggregate(group, None,
                                         [{"values": value, "valid": value_valid.astype(np.uint8), "type": oracle.T_F64}],
                                         [(oracle.SUM, 0), (oracle.COUNT_STAR, 0)])
    return int(passed.sum()), int(hit.sum()), {int(k): (s if ok else None, c) for k, s, ok, c in
                                               zip(keys, res[0]["f64"], res[0]["valid"], res[1]["i64"])}, (fa, fb)


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("group_by", [0, 1])
def test_star_matches_oracle(kb, rt, oracle, mode, group_by):
    W = importlib.import_module("krishiv-engine_b200.workloads")
    import torch
    data = W.star(rt, scale=0.01)
    torch.cuda.synchronize()
    s = kb.StarPipeline(rt, kb.star_spec(7, 7, group_by=group_by, mode=mode))
    s.build_device(kb.DeviceBatch(data.dim_a), kb.DeviceBatch(data.dim_b))
    half = data.fact_rows // 2
    for lo, hi in ((0, half), (half, data.fact_rows)):
        s.probe_device(kb.DeviceBatch([(n, t[lo:hi], v) for n, t, v in data.fact]))
    out = s.result()
    c = s.counters()
    passed, joined, want, (fa, fb) = oracle_star(oracle, data, group_by)
    assert c["fact_rows"] == data.fact_rows
    assert c["filter_a_form"] == fa.form and c["filter_b_form"] == fb.form
    assert c["filter_a_bytes"] == fa.f.bloom_bytes and c["filter_b_bytes"] == fb.f.bloom_bytes
    assert c["passed_filters"] == passed
    assert c["joined_rows"] == joined
    got = dict(zip(out.column(0).to_pylist(), out.column(1).to_pylist()))
    assert sorted(got) == sorted(want)
    for k, (ws, _) in want.items():
        assert rel_err(got[k], ws) <= FLOAT_TOL, (k, got[k], ws)


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("group_by", [0, 1])
def test_star_with_null_fact_columns(kb, rt, oracle, mode, group_by):
    """2% NULLs in every fact column: NULL keys never join, a NULL price or
    discount makes the row's value NULL (the row still joins; SUM skips it).
    Fused and plain forms against the oracle, in two device probe batches
    (the second cut at an odd row)."""
    W = importlib.import_module("krishiv-engine_b200.workloads")
    import torch
    data = W.star(rt, scale=0.01, fact_nulls=0.02)
    torch.cuda.synchronize()
    assert all(c[2] is not None for c in data.fact)
    s = kb.StarPipeline(rt, kb.star_spec(7, 7, group_by=group_by, mode=mode))
    s.build_device(kb.DeviceBatch(data.dim_a), kb.DeviceBatch(data.dim_b))
    n = data.fact_rows
    cut = n // 2 + 3
    full = [(name, t, v) for name, t, v in data.fact]
    # the second part as its own device columns: values and bitmaps realigned at row 0
    second = []
    for name, t, v in full:
        bits = np.unpackbits(v.cpu().numpy(), bitorder="little")[cut:n]
        packed = torch.tensor(np.packbits(bits, bitorder="little"), device="cuda")
        second.append((name, t[cut:].contiguous(), packed))
    first = [(name, t[:cut], v) for name, t, v in full]
    s.probe_device(kb.DeviceBatch(first))
    s.probe_device(kb.DeviceBatch(second))
    out = s.result()
    c = s.counters()
    passed, joined, want, _ = oracle_star(oracle, data, group_by)
    if mode == 0:
        assert c["passed_filters"] == passed
    assert c["joined_rows"] == joined
    got = dict(zip(out.column(0).to_pylist(), out.column(1).to_pylist()))
    assert sorted(got) == sorted(want)
    for k, (ws, _) in want.items():
        if ws is None:
            assert got[k] is None, k
        else:
            assert rel_err(got[k], ws) <= FLOAT_TOL, (k, got[k], ws)


def test_star_same_alone_and_after_reset(kb, rt):
    W = importlib.import_module("krishiv-engine_b200.workloads")
    data = W.star(rt, scale=0.004)
    s = kb.StarPipeline(rt, kb.star_spec(7, 7))
    s.build_device(kb.DeviceBatch(data.dim_a), kb.DeviceBatch(data.dim_b))
    s.probe_device(kb.DeviceBatch(data.fact))
    first = s.result().to_pydict()
    s.reset()
    s.probe_device(kb.DeviceBatch(data.fact))
    second = s.result().to_pydict()
    assert sorted(first["attr"]) == sorted(second["attr"])
    a = dict(zip(first["attr"], first["sum"]))
    b = dict(zip(second["attr"], second["sum"]))
    for k in a:
        assert rel_err(a[k], b[k]) <= FLOAT_TOL


@pytest.mark.parametrize("pinned", [True, False])
def test_star_host_batches(kb, rt, oracle, pinned):
    """Host Arrow batches through krv_star_build / krv_star_probe: page-locked
    columns are read in place by the kernels, pageable ones are copied; both
    give the oracle's answer, and the caller may overwrite its buffers as soon
    as the calls return."""
    import pyarrow as pa
    import torch
    W = importlib.import_module("krishiv-engine_b200.workloads")
    data = W.star(rt, scale=0.01)
    torch.cuda.synchronize()
    passed, joined, want, _ = oracle_star(oracle, data, 0)
    keep = []

    def host(cols):
        arrays = []
        for name, t, _ in cols:
            h = torch.empty(t.shape, dtype=t.dtype, pin_memory=pinned)
            h.copy_(t)
            keep.append(h)
            arrays.append(pa.array(h.numpy()))
        return pa.RecordBatch.from_arrays(arrays, names=[n for n, _, _ in cols])

    fact, dim_a, dim_b = host(data.fact), host(data.dim_a), host(data.dim_b)
    s = kb.StarPipeline(rt, kb.star_spec(7, 7, group_by=0, mode=kb.STAR_FUSED))
    s.build(dim_a, dim_b)
    half = data.fact_rows // 2
    for lo, hi in ((0, half), (half, data.fact_rows)):
        s.probe(fact.slice(lo, hi - lo))
    for h in keep:  # the library no longer reads the caller's buffers
        h.fill_(-1)
    out = s.result()
    c = s.counters()
    assert c["passed_filters"] == passed and c["joined_rows"] == joined
    got = dict(zip(out.column(0).to_pylist(), out.column(1).to_pylist()))
    assert sorted(got) == sorted(want)
    for k, (ws, _) in want.items():
        assert rel_err(got[k], ws) <= FLOAT_TOL, (k, got[k], ws)


def test_star_host_batch_streamed(kb, rt, oracle):
    """A page-locked fact batch of 36M rows: fk_b crosses the host link in
    bulk copies of 8M rows, three in flight, while the kernels read the
    other columns in place. Probed as one row and the rest (an odd Arrow
    offset, five chunks, the last one ragged), then again after a reset:
    the oracle's answer both times."""
    import pyarrow as pa
    import torch
    W = importlib.import_module("krishiv-engine_b200.workloads")
    data = W.star(rt, scale=0.12)
    torch.cuda.synchronize()
    assert data.fact_rows > 4 * (8 << 20)
    passed, joined, want, _ = oracle_star(oracle, data, 0)
    keep = []

    def host(cols):
        arrays = []
        for name, t, _ in cols:
            h = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
            h.copy_(t)
            keep.append(h)
            arrays.append(pa.array(h.numpy()))
        return pa.RecordBatch.from_arrays(arrays, names=[n for n, _, _ in cols])

    fact, dim_a, dim_b = host(data.fact), host(data.dim_a), host(data.dim_b)
    s = kb.StarPipeline(rt, kb.star_spec(7, 7, group_by=0, mode=kb.STAR_FUSED))
    s.build(dim_a, dim_b)
    for parts in (((0, 1), (1, data.fact_rows - 1)), ((0, data.fact_rows),)):
        s.reset()
        for lo, n in parts:
            s.probe(fact.slice(lo, n))
        out = s.result()
        c = s.counters()
        assert c["fact_rows"] == data.fact_rows
        assert c["passed_filters"] == passed and c["joined_rows"] == joined
        got = dict(zip(out.column(0).to_pylist(), out.column(1).to_pylist()))
        assert sorted(got) == sorted(want)
        for k, (ws, _) in want.items():
            assert rel_err(got[k], ws) <= FLOAT_TOL, (k, got[k], ws)


def test_star_host_batch_streamed_with_nulls(kb, rt, oracle):
    """Page-locked host columns with 2% NULLs each, 36M fact rows: fk_b moves
    in bulk copies of 8M rows, the other values are read in place, and the
    validity bitmaps (copied to the device) are read at the bit offset of an
    Arrow slice that starts at row 5 plus that of each chunk."""
    import pyarrow as pa
    import torch
    W = importlib.import_module("krishiv-engine_b200.workloads")
    data = W.star(rt, scale=0.12, fact_nulls=0.02)
    torch.cuda.synchronize()
    passed, joined, want, _ = oracle_star(oracle, data, 0)
    keep = []
    n = data.fact_rows

    def pinned(t):
        h = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
        h.copy_(t)
        keep.append(h)
        return h

    arrays = []
    for name, t, v in data.fact:
        ht, hv = pinned(t), pinned(v)
        typ = pa.float64() if t.dtype == torch.float64 else pa.int64()
        arrays.append(pa.Array.from_buffers(typ, n, [pa.foreign_buffer(hv.data_ptr(), hv.numel()),
                                                     pa.foreign_buffer(ht.data_ptr(), ht.numel() * 8)]))
    fact = pa.RecordBatch.from_arrays(arrays, names=[c[0] for c in data.fact])

    def host(cols):
        return pa.RecordBatch.from_arrays([pa.array(pinned(t).numpy()) for _, t, _ in cols], names=[c[0] for c in cols])

    s = kb.StarPipeline(rt, kb.star_spec(7, 7, group_by=0, mode=kb.STAR_FUSED))
    s.build(host(data.dim_a), host(data.dim_b))
    s.probe(fact.slice(0, 5))
    s.probe(fact.slice(5, n - 5))
    out = s.result()
    c = s.counters()
    assert c["passed_filters"] == passed and c["joined_rows"] == joined
    got = dict(zip(out.column(0).to_pylist(), out.column(1).to_pylist()))
    assert sorted(got) == sorted(want)
    for k, (ws, _) in want.items():
        if ws is None:
            assert got[k] is None, k
        else:
            assert rel_err(got[k], ws) <= FLOAT_TOL, (k, got[k], ws)
