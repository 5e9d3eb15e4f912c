"""krv_agg_sum_i64_scratch, the grouped SUM/COUNT that allocates no device
memory (its hash table is a fixed array of the library), against the
krv_agg_create/push/finish entry points on the same inputs. Integer results,
so the comparison is exact. Collected last so that it also runs after every
other test in one process."""
import numpy as np
import pytest

I64_MIN = -(2**63)


def test_rejects_max_groups_beyond_the_scratch(kb):
    import torch
    e = torch.zeros(0, dtype=torch.int64)
    info = torch.zeros(2, dtype=torch.int64)
    too_many = torch.zeros(kb.SCRATCH_MAX_GROUPS + 1, dtype=torch.int64)
    with pytest.raises(kb.KrvError) as err:
        kb.agg_sum_i64_scratch(e, e, too_many, too_many, too_many, info)
    assert err.value.status == kb.INVALID_ARGUMENT
    assert b"max_groups 65537" in kb.lib().krv_last_error()


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
def test_two_calls_in_a_row_match_the_aggregate(kb, rt):
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
