"""The fused star plan built from an operator chain (krv_star_from_joins):
two inner joins whose build sides hold the dimensions' rows after their
predicates, probed in turn by the fact batch, then a grouped
SUM(price * (1 - discount)). The fused plan (and its plain form) must give
the oracle's answer for the same query, and a chain of another shape must be
refused with KRV_UNSUPPORTED so that the caller runs the operators."""
import importlib

import pytest

from helpers import rel_err
from test_star_gpu import FLOAT_TOL, oracle_star

pytestmark = pytest.mark.gpu


def dim_joins(kb, rt, data, join_type="inner", filters=True):
    """The chain's two joins: join_a on fk_a (fact column 0) keeps fk_b,
    price and discount and adds dim a's attribute; join_b on fk_b (column 0
    of join_a's output) keeps all four and adds dim b's attribute. Each build
    side is its dimension's rows with pred == 7 (key, attr)."""
    import torch
    joins = []
    probe_out = ([1, 2, 3], [0, 1, 2, 3])
    for d, dim in enumerate((data.dim_a, data.dim_b)):
        (kn, key, _), (_, pred, _), (an, attr, _) = dim
        sel = pred == 7
        j = kb.HashJoin(rt, kb.join_spec(join_type if d == 0 else "inner", probe_keys=(0,), build_keys=(0,),
                                         probe_out=probe_out[d], build_out=[1], runtime_filter=filters))
        j.build_push_device(kb.DeviceBatch([(kn, key[sel].contiguous(), None), (an, attr[sel].contiguous(), None)]))
        j.build_finish()
        joins.append(j)
    torch.cuda.synchronize()
    return joins


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("group_by", [0, 1])
def test_chain_matches_oracle(kb, rt, oracle, mode, group_by):
    W = importlib.import_module("krishiv-engine_b200.workloads")
    data = W.star(rt, scale=0.01)
    ja, jb = dim_joins(kb, rt, data)
    # join_b's output: fk_b, price, discount, attr_a, attr_b
    s = kb.StarPipeline.from_joins(rt, ja, jb, n_fact_columns=4, group_col=3 + group_by, price_col=1,
                                   discount_col=2, mode=mode)
    del ja, jb  # the plan keeps its own copy of the dimensions
    half = data.fact_rows // 2
    for lo, hi in ((0, half), (half, data.fact_rows)):
        s.probe_device(kb.DeviceBatch([(n, t[lo:hi], v) for n, t, v in data.fact]))
    out = s.result()
    c = s.counters()
    passed, joined, want, _ = oracle_star(oracle, data, group_by)
    assert c["fact_rows"] == data.fact_rows
    assert c["passed_filters"] == passed
    assert c["joined_rows"] == joined
    got = dict(zip(out.column(0).to_pylist(), out.column(1).to_pylist()))
    assert sorted(got) == sorted(want)
    for k, (ws, _) in want.items():
        assert rel_err(got[k], ws) <= FLOAT_TOL, (k, got[k], ws)


def test_chain_without_filters_joins_the_same_rows(kb, rt, oracle):
    W = importlib.import_module("krishiv-engine_b200.workloads")
    data = W.star(rt, scale=0.005)
    ja, jb = dim_joins(kb, rt, data, filters=False)
    s = kb.StarPipeline.from_joins(rt, ja, jb, n_fact_columns=4, group_col=3, price_col=1, discount_col=2)
    s.probe_device(kb.DeviceBatch(data.fact))
    out = s.result()  # the fused plan's counters are read with its result
    c = s.counters()
    _, joined, want, _ = oracle_star(oracle, data, 0)
    assert c["filter_a_form"] == -1 and c["filter_b_form"] == -1  # no runtime filter was built
    assert c["joined_rows"] == joined
    got = dict(zip(out.column(0).to_pylist(), out.column(1).to_pylist()))
    assert sorted(got) == sorted(want)


def test_other_chains_are_refused(kb, rt):
    W = importlib.import_module("krishiv-engine_b200.workloads")
    data = W.star(rt, scale=0.001)
    ja, jb = dim_joins(kb, rt, data, join_type="left_outer")
    with pytest.raises(kb.KrvError) as e:
        kb.StarPipeline.from_joins(rt, ja, jb, n_fact_columns=4, group_col=3, price_col=1, discount_col=2)
    assert e.value.status == kb.UNSUPPORTED
    ja, jb = dim_joins(kb, rt, data)
    with pytest.raises(kb.KrvError) as e:  # grouped by a fact column
        kb.StarPipeline.from_joins(rt, ja, jb, n_fact_columns=4, group_col=0, price_col=1, discount_col=2)
    assert e.value.status == kb.UNSUPPORTED
