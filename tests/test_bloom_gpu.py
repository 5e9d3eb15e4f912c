"""GPU runtime key filter parity: the same form, the same Bloom bits and the
same pass/fail answer for every row as the CPU oracle's restatement of the
reference's KeyFilter (bit-exact), and zero false negatives."""
import numpy as np
import pyarrow as pa
import pytest

from helpers import batch

pytestmark = pytest.mark.gpu


def build_both(kb, rt, oracle, keys, valid=None):
    b = batch(k=pa.array(keys, mask=None if valid is None else ~valid.astype(bool)))
    g = kb.KeyFilter.build(rt, b, 0)
    o = oracle.KeyFilter(keys, None if valid is None else valid.astype(np.uint8))
    return g, o


def evaluate_both(g, o, probe, pvalid=None):
    b = batch(k=pa.array(probe, mask=None if pvalid is None else ~pvalid.astype(bool)))
    got = np.array(g.evaluate(b, 0).to_pylist(), dtype=bool)
    want = o.evaluate(probe, None if pvalid is None else pvalid.astype(np.uint8))
    return got, want


@pytest.mark.parametrize("n_keys", [1, 100, 4096, 4097, 50_000, 1_000_000])
def test_forms_bits_and_answers(kb, rt, oracle, n_keys):
    rng = np.random.default_rng(n_keys)
    keys = rng.permutation(20 * max(n_keys, 10))[:n_keys].astype(np.int64)
    g, o = build_both(kb, rt, oracle, keys)
    info = g.info()
    assert info["form"] == o.form
    assert (info["lo"], info["hi"], info["keys"]) == (o.f.lo, o.f.hi, o.f.keys)
    if o.form == oracle.FORM_BLOOM:
        assert info["bloom_bytes"] == o.f.bloom_bytes
        assert np.array_equal(np.frombuffer(g.bloom_bytes(), dtype=np.uint32), o.words)
    probe = np.concatenate([keys, rng.integers(-10, 25 * max(n_keys, 10), 2_000_000)]).astype(np.int64)
    got, want = evaluate_both(g, o, probe)
    assert np.array_equal(got, want)
    assert got[: len(keys)].all()  # no false negatives


def test_dense_range_and_nulls(kb, rt, oracle):
    keys = np.arange(1000, 3000, dtype=np.int64)
    valid = np.ones(len(keys), dtype=bool)
    valid[::7] = False  # NULL build keys are not kept
    g, o = build_both(kb, rt, oracle, keys, valid)
    assert g.info()["form"] == o.form
    probe = np.arange(0, 4000, dtype=np.int64)
    pvalid = np.ones(len(probe), dtype=bool)
    pvalid[::5] = False
    got, want = evaluate_both(g, o, probe, pvalid)
    assert np.array_equal(got, want)


def test_empty_filter(kb, rt, oracle):
    keys = np.zeros(10, dtype=np.int64)
    g, o = build_both(kb, rt, oracle, keys, np.zeros(10, dtype=bool))
    assert g.info()["form"] == kb.FILTER_EMPTY == o.form
    got, want = evaluate_both(g, o, np.arange(5, dtype=np.int64))
    assert not got.any() and np.array_equal(got, want)


def test_join_publishes_the_same_filter(kb, rt, oracle):
    rng = np.random.default_rng(5)
    keys = rng.permutation(10_000_000)[:300_000].astype(np.int64)
    j = kb.HashJoin(rt, kb.join_spec("inner", runtime_filter=True))
    j.build_push(batch(k=pa.array(keys)))
    j.build_finish()
    f = j.key_filter()
    o = oracle.KeyFilter(keys)
    assert f.info()["form"] == kb.FILTER_BLOOM == o.form
    assert np.array_equal(np.frombuffer(f.bloom_bytes(), dtype=np.uint32), o.words)


def test_over_the_item_cap_keeps_the_range(kb, rt, oracle):
    keys = np.random.default_rng(6).permutation(50_000_000)[:4_000_001].astype(np.int64)
    g, o = build_both(kb, rt, oracle, keys)
    assert g.info()["form"] == kb.FILTER_RANGE == o.form
