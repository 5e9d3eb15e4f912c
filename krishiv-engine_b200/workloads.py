"""Synthetic workloads of the benchmarks, generated on the device with the
library's counter-based generators (krv_gen_fill), so every run and every
row range is reproducible and the CPU oracle can regenerate any sample.

Shapes (rows at scale 1.0):
  star:   fact 300,000,000 {fk_a uniform [0, 20M), fk_b uniform [0, 1M),
          price int64 uniform [1,000, 10,000,000], discount float64 uniform
          [0, 0.1)}; dim_a 20,000,000 and dim_b 1,000,000 rows {key: a
          permutation of [0, rows), pred int32 uniform [0, 20) (pred = 7
          selects 5%), attr int32 uniform [0, 25)}.
  join:   build 1,000,000 {k: a permutation of [0, 1M), v int64 uniform};
          probe 10,000,000 {k uniform [0, 2M) (about half match), w int32}.
  agg:    100,000,000 rows {k: Zipf(1.1) over 1,000,000 values, dec
          decimal(15,2) unscaled uniform [100, 1e7], f float64 uniform [0, 1),
          q int32 uniform [1, 50]; 2% NULLs per value column}.
  serve:  request templates, each a resident build table {k: a permutation
          of [0, nb) (unique), g int64 uniform [0, G)} and a probe of 10 * nb
          rows {k: with probability r uniform over the build keys, else
          uniform over the disjoint range [2^40, 2^41); x int64 uniform
          [-1e9, 1e9]}; nb log-uniform over [1e3, 5e7 * scale], G log-uniform
          over [10, 1e6] (at most nb), r uniform over [0.1, 1.0]; requests
          pick templates uniformly and arrive as a Poisson process.
  grace:  build 500,000,000 {k int64 uniform [0, 1e9), p1, p2 int64}; probe
          2,000,000,000 {k int64: 90% uniform [0, 1e9), 10% one of 100 heavy
          keys; p int64}; 1% NULL keys on both sides (the key domain scales
          with the rows).
"""
from __future__ import annotations

import importlib
from dataclasses import dataclass

STAR_SEED = 0x4B52560003
JOIN_SEED = 0x4B52560001
AGG_SEED = 0x4B52560002
SERVE_SEED = 0x4B52560005
GRACE_SEED = 0x4B52560004
PRED_VALUE = 7


def _kb():
    return importlib.import_module("krishiv-engine_b200")


def _col(rt, n, dtype, kind, seed, column, **kw):
    import torch
    t = torch.empty(n, dtype=dtype, device=f"cuda:{rt.device}")
    valid = None
    if kw.get("null_fraction", 0.0) > 0:
        valid = torch.empty((n + 31) // 32 * 4, dtype=torch.uint8, device=t.device)
    _kb().gen_fill(rt, t, kind, seed, column, valid=valid, **kw)
    return t, valid


@dataclass
class StarData:
    fact: list      # [(name, tensor, valid)]
    dim_a: list
    dim_b: list
    fact_rows: int
    dim_a_rows: int
    dim_b_rows: int


def star(rt, scale: float = 1.0, seed: int = STAR_SEED, fact_row0: int = 0, fact_scale=None,
         fact_nulls: float = 0.0) -> StarData:
    """The star-join inputs; `fact_row0` selects which fact rows (a shard of
    the fact stream for one of several devices); `fact_scale` (default
    `scale`) sizes the fact table alone, the dimensions keep `scale`;
    `fact_nulls` > 0 makes that fraction of each fact column NULL
    (independently per column)."""
    import torch
    kb = _kb()
    fs = scale if fact_scale is None else fact_scale
    nf, na, nb = int(300_000_000 * fs), int(20_000_000 * scale), int(1_000_000 * scale)
    r0 = dict(row0=fact_row0, null_fraction=fact_nulls)
    fk_a, v1 = _col(rt, nf, torch.int64, kb.GEN_UNIFORM_I64, seed, 1, lo=0, hi=na - 1, **r0)
    fk_b, v2 = _col(rt, nf, torch.int64, kb.GEN_UNIFORM_I64, seed, 2, lo=0, hi=nb - 1, **r0)
    price, v3 = _col(rt, nf, torch.int64, kb.GEN_UNIFORM_I64, seed, 3, lo=1000, hi=10_000_000, **r0)
    disc, v4 = _col(rt, nf, torch.float64, kb.GEN_UNIT_F64, seed, 4, x0=0.0, x1=0.1, **r0)
    dims = []
    for base, n in ((10, na), (20, nb)):
        key, _ = _col(rt, n, torch.int64, kb.GEN_PERMUTATION, seed + base, base + 1, lo=0, hi=n)
        pred, _ = _col(rt, n, torch.int32, kb.GEN_UNIFORM_I32, seed, base + 2, lo=0, hi=19)
        attr, _ = _col(rt, n, torch.int32, kb.GEN_UNIFORM_I32, seed, base + 3, lo=0, hi=24)
        dims.append([("key", key, None), ("pred", pred, None), ("attr", attr, None)])
    fact = [("fk_a", fk_a, v1), ("fk_b", fk_b, v2), ("price", price, v3), ("discount", disc, v4)]
    return StarData(fact, dims[0], dims[1], nf, na, nb)


def join(rt, scale: float = 1.0, seed: int = JOIN_SEED):
    import torch
    kb = _kb()
    nb, np_ = int(1_000_000 * scale), int(10_000_000 * scale)
    bk, _ = _col(rt, nb, torch.int64, kb.GEN_PERMUTATION, seed, 1, lo=0, hi=nb)
    bv, _ = _col(rt, nb, torch.int64, kb.GEN_UNIFORM_I64, seed, 2, lo=-(2**62), hi=2**62)
    pk, _ = _col(rt, np_, torch.int64, kb.GEN_UNIFORM_I64, seed, 3, lo=0, hi=2 * nb - 1)
    pw, _ = _col(rt, np_, torch.int32, kb.GEN_UNIFORM_I32, seed, 4, lo=-(2**31), hi=2**31 - 1)
    return [("k", bk, None), ("v", bv, None)], [("k", pk, None), ("w", pw, None)]


def agg(rt, scale: float = 1.0, seed: int = AGG_SEED, domain: int = 1_000_000):
    import pyarrow as pa
    import torch
    kb = _kb()
    n = int(100_000_000 * scale)
    k, _ = _col(rt, n, torch.int64, kb.GEN_ZIPF, seed, 1, lo=0, hi=domain, x0=1.1)
    dec, dv = _col(rt, n, torch.int64, kb.GEN_UNIFORM_I64, seed, 2, lo=100, hi=10_000_000, null_fraction=0.02)
    f, fv = _col(rt, n, torch.float64, kb.GEN_UNIT_F64, seed, 3, x0=0.0, x1=1.0, null_fraction=0.02)
    q, qv = _col(rt, n, torch.int32, kb.GEN_UNIFORM_I32, seed, 4, lo=1, hi=50, null_fraction=0.02)
    return [("k", k, None), ("dec", dec, dv, pa.decimal64(15, 2)), ("f", f, fv), ("q", q, qv)]


@dataclass
class ServeTemplate:
    build: list        # [(name, tensor, valid)]: k, g
    probe: list        # [(name, tensor, valid)]: k, x
    build_rows: int
    probe_rows: int
    groups: int        # G of the generator (distinct groups <= G)
    match: float       # r


def serve_templates(rt, count: int, scale: float = 1.0, seed: int = SERVE_SEED, max_build=None):
    """`count` request templates of the served request stream (see the module
    docstring); template j is generated from (seed, j) alone. `scale` scales
    the largest build (5e7 rows); the smallest stays 1e3 rows."""
    import math

    import numpy as np
    import torch
    kb = _kb()
    rng = np.random.default_rng(seed)
    lo_b, hi_b = 1e3, max(1e3, 5e7 * scale)
    if max_build is not None:
        hi_b = min(hi_b, max_build)
    out = []
    for j in range(count):
        nb = max(1, int(round(math.exp(rng.uniform(math.log(max(lo_b, 1.0)), math.log(max(hi_b, 2.0)))))))
        G = max(1, min(nb, int(round(math.exp(rng.uniform(math.log(10), math.log(1e6)))))))
        r = float(rng.uniform(0.1, 1.0))
        npr = 10 * nb
        sj = seed + 0x1000 * (j + 1)
        k, _ = _col(rt, nb, torch.int64, kb.GEN_PERMUTATION, sj, 1, lo=0, hi=nb)
        g, _ = _col(rt, nb, torch.int64, kb.GEN_UNIFORM_I64, sj, 2, lo=0, hi=G - 1)
        kin, _ = _col(rt, npr, torch.int64, kb.GEN_UNIFORM_I64, sj, 3, lo=0, hi=nb - 1)
        kout, _ = _col(rt, npr, torch.int64, kb.GEN_UNIFORM_I64, sj, 4, lo=1 << 40, hi=(1 << 41) - 1)
        u, _ = _col(rt, npr, torch.int64, kb.GEN_UNIFORM_I64, sj, 5, lo=0, hi=999_999)
        x, _ = _col(rt, npr, torch.int64, kb.GEN_UNIFORM_I64, sj, 6, lo=-1_000_000_000, hi=1_000_000_000)
        pk = torch.where(u < int(r * 1_000_000), kin, kout)
        del kin, kout, u
        out.append(ServeTemplate([("k", k, None), ("g", g, None)], [("k", pk, None), ("x", x, None)], nb, npr, G, r))
    return out


def serve_arrivals(n: int, rate_per_s: float, templates: int, seed: int = SERVE_SEED):
    """Poisson arrival times (seconds from 0) and the template of each of `n`
    requests."""
    import numpy as np
    rng = np.random.default_rng(seed ^ 0x5EED)
    gaps = rng.exponential(1.0 / rate_per_s, n) if rate_per_s > 0 else np.zeros(n)
    return np.cumsum(gaps) - gaps[0], rng.integers(0, templates, n)


def grace_build(rt, scale: float = 1.0, seed: int = GRACE_SEED):
    """The partitioned join's build side: (k, p1, p2), k NULL in 1% of rows."""
    import torch
    kb = _kb()
    nb = int(500_000_000 * scale)
    dom = int(1_000_000_000 * scale)
    k, kv = _col(rt, nb, torch.int64, kb.GEN_UNIFORM_I64, seed, 1, lo=0, hi=dom - 1, null_fraction=0.01)
    p1, _ = _col(rt, nb, torch.int64, kb.GEN_UNIFORM_I64, seed, 2, lo=-(2**62), hi=2**62)
    p2, _ = _col(rt, nb, torch.int64, kb.GEN_UNIFORM_I64, seed, 3, lo=-(2**62), hi=2**62)
    return [("k", k, kv), ("p1", p1, None), ("p2", p2, None)]


def grace_probe(rt, scale: float = 1.0, seed: int = GRACE_SEED, chunk: int = 1 << 28):
    """The partitioned join's probe side: (k, p); 10% of the rows take one of
    100 heavy keys, 1% have a NULL key. Generated in chunks of `chunk` rows."""
    import torch
    kb = _kb()
    n = int(2_000_000_000 * scale)
    dom = int(1_000_000_000 * scale)
    heavy, _ = _col(rt, 100, torch.int64, kb.GEN_UNIFORM_I64, seed, 20, lo=0, hi=dom - 1)
    k, kv = _col(rt, n, torch.int64, kb.GEN_UNIFORM_I64, seed, 11, lo=0, hi=dom - 1, null_fraction=0.01)
    p, _ = _col(rt, n, torch.int64, kb.GEN_UNIFORM_I64, seed, 12, lo=-(2**62), hi=2**62)
    for r0 in range(0, n, chunk):
        m = min(chunk, n - r0)
        u, _ = _col(rt, m, torch.int64, kb.GEN_UNIFORM_I64, seed, 13, lo=0, hi=999, row0=r0)
        h, _ = _col(rt, m, torch.int64, kb.GEN_UNIFORM_I64, seed, 14, lo=0, hi=99, row0=r0)
        sl = k[r0:r0 + m]
        torch.where(u < 100, heavy[h], sl, out=sl)
        del u, h
    return [("k", k, kv), ("p", p, None)]
