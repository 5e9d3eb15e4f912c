"""krv_agg_sum_i64_scratch, the grouped SUM/COUNT that allocates no device
memory (its hash table is a fixed array of the library), against the
krv_agg_create/push/finish entry points and the CPU oracle on the same inputs.
Integer results, so the comparisons are exact. Collected last so that it also
runs after every other test in one process."""
import time

import numpy as np
import pytest

I64_MIN = -(2**63)


def test_rejects_max_groups_beyond_the_scratch(kb):
    """The C entry point refuses a max_groups beyond its fixed table before
    any device work (so this needs no GPU)."""
    st = kb.lib().krv_agg_sum_i64_scratch(None, None, 0, kb.SCRATCH_MAX_GROUPS + 1, None, None, None, None, None)
    assert st == kb.INVALID_ARGUMENT
    assert b"max_groups 65537" in kb.lib().krv_last_error()


def test_python_binding_rejects_bad_tensors(kb):
    """Checks made before any call into the library: dtype, device, layout
    and output lengths (a short or mistyped output would be written out of
    bounds by the device)."""
    import torch
    ok = torch.zeros(4, dtype=torch.int64)
    info = torch.zeros(2, dtype=torch.int64)
    with pytest.raises(ValueError, match="int64"):
        kb.agg_sum_i64_scratch(ok.int(), ok, ok, ok, ok, info)
    with pytest.raises(ValueError, match="CUDA"):
        kb.agg_sum_i64_scratch(ok, ok, ok, ok, ok, info)


def oracle_groups(oracle, key, v):
    """GROUP BY key SUM(v), COUNT(*) by the CPU oracle (ANSI off: wraps)."""
    k, _, res = oracle.hash_aggregate(key, None, [{"values": v, "type": oracle.T_I64}],
                                      [(oracle.SUM, 0), (oracle.COUNT_STAR, 0)], ansi=False)
    return {int(kk): (int(s), int(c)) for kk, s, c in zip(k, res[0]["i64"], res[1]["i64"])}


def existing(kb, rt, kt, vt):
    """The same query through the krv_agg_* entry points (ANSI off: wraps)."""
    a = kb.HashAggregate(rt, kb.agg_spec(0, [("sum", 1), ("count_star", 0)], ansi=False))
    a.push_device(kb.DeviceBatch([("k", kt, None), ("v", vt, None)]))
    a.finish()
    res = a.result_device()
    rt.synchronize()
    k = res.columns[0].cpu().numpy().tolist()
    s = res.columns[1].cpu().numpy().tolist()
    c = res.columns[2].cpu().numpy().tolist()
    return {kk: (ss, cc) for kk, ss, cc in zip(k, s, c)}


def scratch(kb, kt, vt, max_groups):
    import torch
    ok = torch.empty(max_groups, dtype=torch.int64, device="cuda")
    osum = torch.empty(max_groups, dtype=torch.int64, device="cuda")
    ocnt = torch.empty(max_groups, dtype=torch.int64, device="cuda")
    info = torch.full((2,), 7, dtype=torch.int64, device="cuda")
    kb.agg_sum_i64_scratch(kt, vt, ok, osum, ocnt, info, stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    g, wrapped = info.cpu().tolist()
    if g < 0:
        return g, wrapped, None
    got = dict(zip(ok[:g].cpu().tolist(), zip(osum[:g].cpu().tolist(), ocnt[:g].cpu().tolist())))
    assert len(got) == g  # every group once
    return g, wrapped, got


@pytest.mark.gpu
def test_two_calls_in_a_row_match_the_aggregate(kb, rt, oracle):
    import torch
    rng = np.random.default_rng(2024)
    # First call: 2M rows over 50,000 keys, with the table's marker key.
    n1 = 2_000_000
    k1 = rng.integers(-(2**40), 2**40, 50_000, dtype=np.int64)
    k1[17] = I64_MIN
    key1 = k1[rng.integers(0, k1.size, n1)]
    v1 = rng.integers(-10**12, 10**12, n1, dtype=np.int64)
    # Second call: fewer keys (none of the first call's may survive), one
    # group whose sum wraps.
    n2 = 300_001
    key2 = rng.integers(0, 999, n2, dtype=np.int64)
    v2 = rng.integers(-1000, 1000, n2, dtype=np.int64)
    key2[:3] = 5000
    v2[:3] = 2**62
    for key, v, wraps in ((key1, v1, 0), (key2, v2, 1)):
        kt = torch.tensor(key, device="cuda")
        vt = torch.tensor(v, device="cuda")
        torch.cuda.synchronize()
        want = existing(kb, rt, kt, vt)
        g, wrapped, got = scratch(kb, kt, vt, kb.SCRATCH_MAX_GROUPS)
        assert g == len(want)
        assert got == want
        assert got == oracle_groups(oracle, key, v)
        assert wrapped == wraps


@pytest.mark.gpu
def test_more_keys_than_max_groups_voids_the_answer(kb, rt):
    import torch
    key = torch.arange(1000, dtype=torch.int64, device="cuda")
    v = torch.ones(1000, dtype=torch.int64, device="cuda")
    g, _, _ = scratch(kb, key, v, 100)
    assert g == -1
    g, wrapped, got = scratch(kb, key, v, 1000)  # the next call starts clean
    assert g == 1000 and wrapped == 0 and got == {i: (1, 1) for i in range(1000)}


@pytest.mark.gpu
def test_empty_input(kb, rt):
    import torch
    e = torch.zeros(0, dtype=torch.int64, device="cuda")
    g, wrapped, got = scratch(kb, e, e, 16)
    assert (g, wrapped, got) == (0, 0, {})


@pytest.mark.gpu
def test_many_more_keys_than_the_table_stops_early(kb, rt):
    """About ten times KRV_SCRATCH_MAX_GROUPS distinct keys over 8M rows: the
    answer is void (-1), and the call gives up soon after the table has no
    room instead of walking long probe runs for every remaining row."""
    import torch
    n = 8_000_000
    key = torch.randint(0, 10 * kb.SCRATCH_MAX_GROUPS, (n,), dtype=torch.int64, device="cuda")
    v = torch.ones(n, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    g, _, _ = scratch(kb, key, v, kb.SCRATCH_MAX_GROUPS)
    dt = time.perf_counter() - t0
    assert g == -1
    assert dt < 2.0, dt
    # and a fitting call right after it is exact again
    small = torch.arange(100, dtype=torch.int64, device="cuda").repeat(3)
    g, wrapped, got = scratch(kb, small, torch.ones_like(small), 100)
    assert (g, wrapped) == (100, 0) and got == {i: (3, 3) for i in range(100)}
