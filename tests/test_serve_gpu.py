"""The request server (krv_server_*) against the CPU oracle: each request's
groups, SUMs and COUNTs are exact (int64), compared as sorted multisets, in
batched mode (ticks that split requests, shared-memory and global
aggregation, duplicate build keys, NULL probe keys), in plain mode, alone and
in the mix; admission by the HBM budget; ANSI overflow."""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def W():
    return importlib.import_module("krishiv-engine_b200.workloads")


def expected(oracle, build_k, build_g, probe_k, probe_x, probe_valid=None):
    """GROUP BY g: SUM(x), COUNT(*) over probe JOIN build USING (k), by the
    oracle's join (all duplicate matches, NULL keys never match)."""
    pv = None if probe_valid is None else probe_valid.astype(np.uint8)
    pi, bi = oracle.hash_join(0, [(build_k, None)], [(probe_k, pv)])
    g = build_g[bi]
    x = probe_x[pi]
    out = {}
    for gg, xx in zip(g.tolist(), x.tolist()):
        s, c = out.get(gg, (0, 0))
        out[gg] = (s + xx, c + 1)
    return {k: (((s + 2**63) % 2**64) - 2**63, c) for k, (s, c) in out.items()}


def got_of(res):
    if res is None or res.rows == 0:
        return {}
    g, s, c = (t.cpu().numpy().tolist() for t in res.columns)
    d = dict(zip(g, zip(s, c)))
    assert len(d) == res.rows
    return d


def run_all(kb, srv, submits):
    ids = [srv.submit(t, db) for t, db in submits]
    results = {}
    for _ in range(100000):
        n = srv.step(wait=True)
        while True:
            p = srv.poll()
            if p is None:
                break
            rid, st, res = p
            results[rid] = (st, got_of(res))
        if n == 0 and len(results) == len(ids):
            break
    assert len(results) == len(ids)
    return [results[i] for i in ids]


def make_case(kb, rt, seed=5):
    """Five tables and 24 probes of uneven sizes, some with NULL keys, one
    empty. The tables cover every lookup layout and both aggregations:
    dense unique keys (direct array) with few and with many groups, sparse
    unique keys (records) with many and with few groups, duplicate keys
    (chains)."""
    rng = np.random.default_rng(seed)
    tables = []
    specs = [(5000, 40), (20000, 6000), (3000, 300), (8000, 3000), (6000, 500)]
    for i, (nb, G) in enumerate(specs):
        if i == 2:  # duplicate keys: every key three times
            k = np.repeat(rng.permutation(nb // 3), 3).astype(np.int64)
        elif i in (0, 3):  # dense keys
            k = rng.permutation(nb).astype(np.int64) + 12345 - 4000 * i
        else:
            k = rng.permutation(nb).astype(np.int64) * 7 - 1000
        g = rng.integers(-(2**40), 2**40, G)[rng.integers(0, G, k.size)].astype(np.int64)
        tables.append((k, g))
    probes = []
    for j in range(24):
        ti = j % 5
        bk = tables[ti][0]
        n = 0 if j == 5 else int(rng.integers(1, 60000))
        hit = rng.random(n) < rng.uniform(0.1, 1.0)
        pk = np.where(hit, bk[rng.integers(0, bk.size, n)] if bk.size else 0, rng.integers(2**41, 2**42, n))
        px = rng.integers(-10**9, 10**9, n)
        valid = (rng.random(n) > 0.05) if j % 4 == 1 else None
        probes.append((ti, pk.astype(np.int64), px.astype(np.int64), valid))
    return tables, probes


def device_batch(kb, cols):
    import torch
    out = []
    for name, a, valid in cols:
        t = torch.tensor(a, device="cuda")
        v = None
        if valid is not None:
            bits = np.packbits(valid.astype(np.uint8), bitorder="little")
            bits = np.concatenate([bits, np.zeros(8, np.uint8)])
            v = torch.tensor(bits, device="cuda")
        out.append((name, t, v))
    return kb.DeviceBatch(out)


def load(kb, srv, tables):
    tids, keep = [], []
    for k, g in tables:
        db = device_batch(kb, [("k", k, None), ("g", g, None)])
        keep.append(db)
        tids.append(srv.add_table(db))
    return tids, keep


def submits_of(kb, tids, probes):
    return [(tids[ti], device_batch(kb, [("k", pk, valid), ("x", px, None)])) for ti, pk, px, valid in probes]


@pytest.mark.parametrize("mode", [0, 1])
def test_requests_match_the_oracle(kb, rt, oracle, mode):
    import torch
    tables, probes = make_case(kb, rt)
    srv = kb.Server(rt, kb.server_options(mode=mode, tick_rows=50_000, max_tick_requests=5, autotune=1))
    tids, _keep = load(kb, srv, tables)
    torch.cuda.synchronize()
    got = run_all(kb, srv, submits_of(kb, tids, probes))
    for (ti, pk, px, valid), (st, res) in zip(probes, got):
        assert st == kb.OK
        want = expected(oracle, tables[ti][0], tables[ti][1], pk, px, valid)
        assert res == want
    s = srv.stats()
    assert s["requests_done"] == len(probes)
    if mode == 0:
        assert s["ticks"] >= 10  # requests were split over ticks


def test_same_alone_and_in_the_mix(kb, rt):
    """Each request's result is the same run alone on a fresh server and run
    among all the others (exact integers)."""
    import torch
    tables, probes = make_case(kb, rt, seed=11)
    srv = kb.Server(rt, kb.server_options(tick_rows=80_000, max_tick_requests=8))
    tids, _keep = load(kb, srv, tables)
    mix = run_all(kb, srv, submits_of(kb, tids, probes))
    for j in (0, 4, 7, 13):
        alone_srv = kb.Server(rt, kb.server_options(tick_rows=80_000))
        atids, _k2 = load(kb, alone_srv, tables)
        alone = run_all(kb, alone_srv, submits_of(kb, atids, [probes[j]]))[0]
        assert alone == mix[j]
        alone_srv.close()
    torch.cuda.synchronize()


def test_admission_by_hbm_budget(kb, rt, oracle):
    tables, probes = make_case(kb, rt, seed=3)
    # table 1 has ~6000 groups: 48 bytes each per running request
    budget = 48 * 6000 * 2 + 48 * 400
    srv = kb.Server(rt, kb.server_options(tick_rows=30_000, hbm_budget_bytes=budget))
    tids, _keep = load(kb, srv, tables)
    subs = submits_of(kb, tids, probes)
    ids = [srv.submit(t, db) for t, db in subs]
    seen_max = 0
    results = {}
    while len(results) < len(ids):
        srv.step(wait=True)
        seen_max = max(seen_max, srv.stats()["budget_in_use"])
        while (p := srv.poll()) is not None:
            results[p[0]] = (p[1], got_of(p[2]))
    assert 0 < seen_max <= budget
    for (ti, pk, px, valid), rid in zip(probes, ids):
        assert results[rid] == (kb.OK, expected(oracle, tables[ti][0], tables[ti][1], pk, px, valid))
    # a request whose state alone exceeds the budget is refused at submit
    small = kb.Server(rt, kb.server_options(hbm_budget_bytes=1000))
    t2, _k3 = load(kb, small, tables[1:2])
    with pytest.raises(kb.KrvError) as e:
        small.submit(t2[0], subs[1][1])
    assert e.value.status == kb.NEED_MEMORY


@pytest.mark.parametrize("mode", [0, 1])
def test_ansi_overflow_fails_only_that_request(kb, rt, mode):
    k = np.arange(10, dtype=np.int64)
    g = np.zeros(10, dtype=np.int64)
    srv = kb.Server(rt, kb.server_options(mode=mode))
    tids, _keep = load(kb, srv, [(k, g)])
    big = device_batch(kb, [("k", np.array([1, 2, 3], np.int64), None), ("x", np.full(3, 2**62, np.int64), None)])
    ok = device_batch(kb, [("k", np.array([1, 2], np.int64), None), ("x", np.array([5, 6], np.int64), None)])
    got = run_all(kb, srv, [(tids[0], big), (tids[0], ok)])
    assert got[0][0] == kb.ARITHMETIC_OVERFLOW
    assert got[1] == (kb.OK, {0: (11, 2)})
    srv2 = kb.Server(rt, kb.server_options(mode=mode, ansi=0))
    t2, _k2 = load(kb, srv2, [(k, g)])
    big2 = device_batch(kb, [("k", np.array([1, 2, 3], np.int64), None), ("x", np.full(3, 2**62, np.int64), None)])
    assert run_all(kb, srv2, [(t2[0], big2)])[0] == (kb.OK, {0: (3 * 2**62 - 2**64, 3)})


def test_autotuner_settles(kb, rt):
    tables, probes = make_case(kb, rt, seed=9)
    srv = kb.Server(rt, kb.server_options(tick_rows=20_000, autotune=1))
    tids, _keep = load(kb, srv, tables)
    run_all(kb, srv, submits_of(kb, tids, probes * 2))
    s = srv.stats()
    assert s["tuned"] == 1 and s["threads"] in (256, 512) and s["smem_groups"] in (0, 2048)


def test_serve_templates_generate(kb, rt):
    ts = W().serve_templates(rt, 3, scale=0.001)
    for t in ts:
        assert t.probe_rows == 10 * t.build_rows
        k = t.build[0][1].cpu().numpy()
        assert np.array_equal(np.sort(k), np.arange(t.build_rows))
