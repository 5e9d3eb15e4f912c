"""The key hash on the device, bit for bit against the oracle: the seedless
row hash h of one or several key columns (NULLs skipped or mixed as NULL_HASH
by null safety, float64 keys normalised), g = fin(h ^ seed) and the partition
ids of level 0 (top radix bits of h) and of the grace levels 1..6 (bits
[48-3d, 51-3d) of g). The oracle itself is pinned to the reference's known
answer for h (crates/krishiv-exec/src/join/keys.rs:348) and its partition
cases (hash.rs:139-148) by the CPU tests."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
MASK = (1 << 64) - 1


def _bitmap(valid):
    return np.packbits(valid.astype(np.uint8), bitorder="little")


def _device(kb, cols):
    import torch
    out = []
    for name, values, valid in cols:
        t = torch.tensor(values, device="cuda")
        v = torch.tensor(_bitmap(valid), device="cuda") if valid is not None else None
        out.append((name, t, v))
    return kb.DeviceBatch(out)


def _u64(t):
    return t.cpu().numpy().view(np.uint64)


@pytest.mark.parametrize("n", [0, 1, 1000, 300_001])
def test_single_int64_key(kb, rt, oracle, n):
    rng = np.random.default_rng(n)
    k = rng.integers(-(2**63), 2**63 - 1, n, dtype=np.int64)
    if n:
        k[: min(n, 4)] = [0, -1, 2**63 - 1, -(2**63)][: min(n, 4)]
    seed = 0x4B52565F4A4F494E
    db = _device(kb, [("k", k, None)])
    h, g, p = kb.hash_rows(rt, db, seed=seed, depth=0, radix=6)
    rt.synchronize()
    want_h = oracle.row_hash([(k, None, False)])
    assert np.array_equal(_u64(h), want_h)
    L = oracle.lib()
    want_g = np.array([L.orc_finalize(int(x), seed) for x in want_h], dtype=np.uint64)
    assert np.array_equal(_u64(g), want_g)
    want_p = np.array([L.orc_partition(int(x), 0, 6, seed) for x in want_h], dtype=np.int32)
    assert np.array_equal(p.cpu().numpy(), want_p)


@pytest.mark.parametrize("null_safe", [(0, 0, 0), (1, 0, 1), (1, 1, 1)])
def test_composite_keys_with_nulls(kb, rt, oracle, null_safe):
    rng = np.random.default_rng(7)
    n = 50_000
    a = rng.integers(-1000, 1000, n, dtype=np.int64)
    b = rng.integers(-(2**31), 2**31 - 1, n, dtype=np.int64).astype(np.int32)
    f = rng.standard_normal(n)
    f[::97] = -0.0
    f[1::97] = 0.0
    f[2::97] = np.nan
    f[3::97] = -np.nan
    va = rng.random(n) > 0.1
    vb = rng.random(n) > 0.1
    vf = rng.random(n) > 0.1
    db = _device(kb, [("a", a, va), ("b", b, vb), ("f", f, vf)])
    seed = 0x1234567887654321
    want_h = oracle.row_hash([(a, va, False), (b, vb, False), (f, vf, True)], list(null_safe))
    L = oracle.lib()
    for depth in range(0, 8):
        radix = 3 + depth % 4
        h, g, p = kb.hash_rows(rt, db, key_columns=(0, 1, 2), null_safe=list(null_safe), seed=seed, depth=depth,
                               radix=radix)
        rt.synchronize()
        assert np.array_equal(_u64(h), want_h)
        got_p = p.cpu().numpy()
        want_p = np.array([L.orc_partition(int(x), depth, radix, seed) for x in want_h[:5000]], dtype=np.int32)
        assert np.array_equal(got_p[:5000], want_p), depth
        if depth == 1:
            want_g = np.array([L.orc_finalize(int(x), seed) for x in want_h[:5000]], dtype=np.uint64)
            assert np.array_equal(_u64(g)[:5000], want_g)


def test_known_answer_row(kb, rt, oracle):
    """The reference's known answer (join/keys.rs:348): the row (Float64 0.0,
    Int32 NULL) with null_safe = [false, true] hashes to 4733552696251797926."""
    f = np.array([0.0, -0.0])
    i = np.array([5, 5], dtype=np.int32)
    db = _device(kb, [("f", f, None), ("i", i, np.array([False, False]))])
    h, _, _ = kb.hash_rows(rt, db, key_columns=(0, 1), null_safe=[0, 1])
    rt.synchronize()
    assert _u64(h).tolist() == [4_733_552_696_251_797_926] * 2
