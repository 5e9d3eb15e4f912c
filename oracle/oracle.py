"""ctypes binding of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: the tests, the smoke check and the benchmark's
CPU-baseline leg use this as the checker. The product library never imports
it. The C sources restate the Krishiv engine's CPU algorithms; each C function
cites the reference file:line it follows.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_NATIVE_PATH = os.path.join(_HERE, "_native", "liboracle.so")

INNER, LEFT_OUTER, LEFT_SEMI, LEFT_ANTI, NULL_AWARE_ANTI, EXISTENCE = 0, 1, 2, 3, 4, 5
RIGHT_SEMI, RIGHT_ANTI, RIGHT_OUTER, FULL_OUTER = 6, 7, 8, 9

T_I32, T_I64, T_F64, T_DEC64, T_DEC128 = 0, 1, 2, 3, 4
COUNT_STAR, COUNT, SUM, MIN, MAX, AVG = 0, 1, 2, 3, 4, 5

FORM_RANGE, FORM_EXACT, FORM_BLOOM, FORM_EMPTY = 0, 1, 2, 3


def build() -> str:
    """Compiles the oracle with its Makefile (gcc) and returns the .so path."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


class OrcCol(C.Structure):
    _fields_ = [("data", C.c_void_p), ("valid", C.c_void_p), ("width", C.c_int32),
                ("is_float", C.c_int32)]


class OrcValueCol(C.Structure):
    _fields_ = [("data", C.c_void_p), ("valid", C.c_void_p), ("type", C.c_int32),
                ("precision", C.c_int32), ("scale", C.c_int32), ("pad", C.c_int32)]


class OrcAggExpr(C.Structure):
    _fields_ = [("func", C.c_int32), ("col", C.c_int32)]


class OrcAggOut(C.Structure):
    _fields_ = [("i64", C.POINTER(C.c_int64)), ("f64", C.POINTER(C.c_double)),
                ("f64_seq", C.POINTER(C.c_double)), ("lo", C.POINTER(C.c_uint64)),
                ("hi", C.POINTER(C.c_int64)), ("valid", C.POINTER(C.c_uint8))]


class OrcKeyFilter(C.Structure):
    _fields_ = [("form", C.c_int32), ("nulls_pass", C.c_int32), ("has_range", C.c_int32),
                ("pad", C.c_int32), ("lo", C.c_int64), ("hi", C.c_int64), ("keys", C.c_int64),
                ("distinct", C.c_int64), ("bloom_bytes", C.c_int64)]


_lib = None
_lib_kind = "generic"


def use_native() -> str:
    """Loads a copy of the oracle compiled for this host (-O3 -march=native),
    built here with `make native`; falls back to the generic -O3 copy when
    that build fails. Must come before the first use. Returns which copy is
    loaded ("native" or "generic")."""
    global _lib_kind
    if _lib is not None:
        return _lib_kind
    try:
        subprocess.run(["make", "-s", "-C", _HERE, "native"], check=True, capture_output=True)
        _lib_kind = "native"
    except (OSError, subprocess.CalledProcessError):
        _lib_kind = "generic"
    return _lib_kind


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_NATIVE_PATH if _lib_kind == "native" else _LIB_PATH)
        u64, i64, i32, vp = C.c_uint64, C.c_int64, C.c_int32, C.c_void_p
        L.orc_fold.restype = u64
        L.orc_fold.argtypes = [u64, u64]
        L.orc_finalize.restype = u64
        L.orc_finalize.argtypes = [u64, u64]
        L.orc_partition.restype = i32
        L.orc_partition.argtypes = [u64, i32, i32, u64]
        L.orc_null_spread.restype = u64
        L.orc_null_spread.argtypes = [u64]
        L.orc_row_hash.argtypes = [vp, C.c_int, vp, i64, vp]
        L.orc_xxh64_fixed.restype = u64
        L.orc_xxh64_fixed.argtypes = [u64, u64, i32]
        L.orc_int_hashes.argtypes = [vp, i64, i32, vp]
        L.orc_bloom_bytes_for.restype = i64
        L.orc_bloom_bytes_for.argtypes = [u64, C.c_double]
        L.orc_bloom_insert.argtypes = [vp, i64, vp, i64]
        L.orc_bloom_check.argtypes = [vp, i64, vp, i64, vp]
        L.orc_bloom_expected_fpp.restype = C.c_double
        L.orc_bloom_expected_fpp.argtypes = [i64, u64]
        L.orc_key_filter_build.argtypes = [vp, vp, i64, vp, vp, C.POINTER(C.POINTER(C.c_int64)),
                                           C.POINTER(i64)]
        L.orc_key_filter_eval.argtypes = [vp, vp, vp, i64, vp, vp, i64, vp]
        L.orc_hash_join.restype = i64
        L.orc_hash_join.argtypes = [i32, vp, i64, vp, i64, i32, vp, i32, u64, i32,
                                    C.POINTER(C.POINTER(C.c_int64)),
                                    C.POINTER(C.POINTER(C.c_int64))]
        L.orc_free.argtypes = [vp]
        L.orc_hash_aggregate.restype = i64
        L.orc_hash_aggregate.argtypes = [vp, vp, i32, i64, vp, i32, vp, i32, i32,
                                         C.POINTER(C.POINTER(C.c_int64)),
                                         C.POINTER(C.POINTER(C.c_uint8)), vp]
        L.orc_avg_decimal.restype = i32
        L.orc_avg_decimal.argtypes = [i64, i64, i32, i64, i32, i32, C.POINTER(u64),
                                      C.POINTER(i64)]
        L.orc_rand.restype = u64
        L.orc_rand.argtypes = [u64, C.c_uint32, u64]
        L.orc_permute.restype = u64
        L.orc_permute.argtypes = [u64, u64, u64]
        L.orc_zipf_cdf.argtypes = [C.c_double, i64, vp]
        L.orc_zipf_rank.restype = i64
        L.orc_zipf_rank.argtypes = [vp, i64, C.c_double]
        L.orc_gen_column.argtypes = [u64, C.c_uint32, i32, i64, i64, C.c_double, C.c_double, i64, i64,
                                     C.c_double, vp, vp]
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data


def _col(values, valid=None, is_float=False):
    values = np.ascontiguousarray(values)
    v = None if valid is None else np.ascontiguousarray(valid, dtype=np.uint8)
    width = values.dtype.itemsize if values.ndim == 1 else values.shape[1] * values.dtype.itemsize
    return OrcCol(values.ctypes.data, _ptr(v), width, int(is_float)), (values, v)


def row_hash(cols, null_bits=None):
    """Seedless row hash h of key columns. `cols` is a list of
    (values, valid-or-None, is_float) tuples of equal length."""
    n = len(cols[0][0])
    arr = (OrcCol * len(cols))()
    keep = []
    for i, (v, m, f) in enumerate(cols):
        c, k = _col(v, m, f)
        arr[i] = c
        keep.append(k)
    nb = np.array(null_bits if null_bits is not None else [0] * len(cols), dtype=np.int32)
    out = np.empty(n, dtype=np.uint64)
    lib().orc_row_hash(C.addressof(arr), len(cols), nb.ctypes.data, n, out.ctypes.data)
    return out


def xxh64_int(values, width=8):
    values = np.ascontiguousarray(values, dtype=np.int64)
    out = np.empty(len(values), dtype=np.uint64)
    lib().orc_int_hashes(values.ctypes.data, len(values), width, out.ctypes.data)
    return out


def bloom_bytes_for(items, fpp):
    return lib().orc_bloom_bytes_for(items, fpp)


def bloom_build(hashes, nbytes):
    hashes = np.ascontiguousarray(hashes, dtype=np.uint64)
    words = np.zeros(nbytes // 4, dtype=np.uint32)
    lib().orc_bloom_insert(words.ctypes.data, nbytes, hashes.ctypes.data, len(hashes))
    return words


def bloom_check(words, hashes):
    hashes = np.ascontiguousarray(hashes, dtype=np.uint64)
    out = np.empty(len(hashes), dtype=np.uint8)
    lib().orc_bloom_check(words.ctypes.data, words.nbytes, hashes.ctypes.data, len(hashes),
                          out.ctypes.data)
    return out.astype(bool)


class KeyFilter:
    """The runtime key filter of an int64 build key column (forms and sizing
    of crates/krishiv-io/src/runtime_filter/filter.rs)."""

    def __init__(self, keys, valid=None):
        keys = np.ascontiguousarray(keys, dtype=np.int64)
        v = None if valid is None else np.ascontiguousarray(valid, dtype=np.uint8)
        self.f = OrcKeyFilter()
        self.words = np.zeros((8 << 20) // 4, dtype=np.uint32)
        es = C.POINTER(C.c_int64)()
        en = C.c_int64(0)
        lib().orc_key_filter_build(keys.ctypes.data, _ptr(v), len(keys), C.addressof(self.f),
                                   self.words.ctypes.data, C.byref(es), C.byref(en))
        self.exact = np.ctypeslib.as_array(es, shape=(en.value,)).copy() if en.value else \
            np.zeros(0, dtype=np.int64)
        if en.value:
            lib().orc_free(es)
        self.words = self.words[: max(self.f.bloom_bytes, 32) // 4].copy()

    @property
    def form(self):
        return self.f.form

    def evaluate(self, keys, valid=None):
        keys = np.ascontiguousarray(keys, dtype=np.int64)
        v = None if valid is None else np.ascontiguousarray(valid, dtype=np.uint8)
        out = np.empty(len(keys), dtype=np.uint8)
        lib().orc_key_filter_eval(C.addressof(self.f), self.words.ctypes.data,
                                  self.exact.ctypes.data, len(self.exact), keys.ctypes.data,
                                  _ptr(v), len(keys), out.ctypes.data)
        return out.astype(bool)


class OrcOperand(C.Structure):
    _fields_ = [("side", C.c_int32), ("is_float", C.c_int32), ("col", OrcCol), ("i64", C.c_int64),
                ("f64", C.c_double)]


class OrcTerm(C.Structure):
    _fields_ = [("op", C.c_int32), ("pad", C.c_int32), ("l", OrcOperand), ("r", OrcOperand)]


class OrcFilter(C.Structure):
    _fields_ = [("n", C.c_int32), ("pad", C.c_int32), ("t", OrcTerm * 8)]


CMP = {"=": 0, "!=": 1, "<": 2, "<=": 3, ">": 4, ">=": 5}


def make_filter(terms, probe_cols, build_cols):
    """A residual filter: `terms` as (left, op, right) with operands
    ("probe", i) / ("build", i) naming entries of `probe_cols` /
    `build_cols` ((values, valid-or-None) numpy pairs), an int or a float.
    Returns (OrcFilter, keep-alive list)."""
    f = OrcFilter()
    f.n = len(terms)
    keep = []

    def operand(o):
        if isinstance(o, tuple):
            values, valid = (probe_cols if o[0] == "probe" else build_cols)[o[1]]
            c, k = _col(values, valid, values.dtype == np.float64)
            keep.append(k)
            return OrcOperand(side=0 if o[0] == "probe" else 1, is_float=int(values.dtype == np.float64), col=c)
        if isinstance(o, float):
            return OrcOperand(side=2, is_float=1, f64=o)
        return OrcOperand(side=2, is_float=0, i64=int(o))
    for i, (l, op, r) in enumerate(terms):
        f.t[i] = OrcTerm(op=CMP[op], l=operand(l), r=operand(r))
    return f, keep


def hash_join(join_type, build_keys, probe_keys, null_safe=None, single_match=False, seed=7,
              radix=3, filter=None):
    """Index pairs of probe ⋈ build. `build_keys`/`probe_keys`: lists of
    (values, valid-or-None, is_float). Returns (probe_rows, build_rows) int64
    arrays with -1 for a NULL-padded side (existence: build_rows = flag).
    `filter`: a residual filter from make_filter (or None)."""
    nk = len(build_keys)
    nb = len(build_keys[0][0])
    np_ = len(probe_keys[0][0])
    ba = (OrcCol * nk)()
    pa = (OrcCol * nk)()
    keep = []
    for i in range(nk):
        c, k = _col(*build_keys[i])
        ba[i] = c
        keep.append(k)
        c, k = _col(*probe_keys[i])
        pa[i] = c
        keep.append(k)
    ns = np.array(null_safe if null_safe is not None else [0] * nk, dtype=np.int32)
    op = C.POINTER(C.c_int64)()
    ob = C.POINTER(C.c_int64)()
    L = lib()
    L.orc_hash_join_filtered.restype = C.c_int64
    L.orc_hash_join_filtered.argtypes = [C.c_int32, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int32,
                                         C.c_void_p, C.c_int32, C.c_uint64, C.c_int32, C.c_void_p,
                                         C.POINTER(C.POINTER(C.c_int64)), C.POINTER(C.POINTER(C.c_int64))]
    n = L.orc_hash_join_filtered(join_type, C.addressof(ba), nb, C.addressof(pa), np_, nk,
                                 ns.ctypes.data, int(single_match), seed, radix,
                                 C.addressof(filter[0]) if filter is not None else None, C.byref(op),
                                 C.byref(ob))
    if n == -2:
        raise RuntimeError("SCALAR_SUBQUERY_TOO_MANY_ROWS")
    if n < 0:
        raise RuntimeError(f"oracle join failed: {n}")
    if n == 0:
        return np.zeros(0, np.int64), np.zeros(0, np.int64)
    p = np.ctypeslib.as_array(op, shape=(n,)).copy()
    b = np.ctypeslib.as_array(ob, shape=(n,)).copy()
    lib().orc_free(op)
    lib().orc_free(ob)
    return p, b


def hash_aggregate(key, key_valid, cols, exprs, ansi=True):
    """GROUP BY one int64/int32 key. `cols`: list of dicts {values, valid,
    type, precision, scale}; `exprs`: list of (func, col). Returns
    (keys, key_valid, results) with results[e] a dict of numpy arrays."""
    key = np.ascontiguousarray(key)
    kv = None if key_valid is None else np.ascontiguousarray(key_valid, dtype=np.uint8)
    n = len(key)
    ca = (OrcValueCol * max(1, len(cols)))()
    keep = []
    for i, c in enumerate(cols):
        v = np.ascontiguousarray(c["values"])
        m = None if c.get("valid") is None else np.ascontiguousarray(c["valid"], dtype=np.uint8)
        keep.append((v, m))
        ca[i] = OrcValueCol(v.ctypes.data, _ptr(m), c["type"], c.get("precision", 0),
                            c.get("scale", 0), 0)
    ea = (OrcAggExpr * len(exprs))(*[OrcAggExpr(f, c) for f, c in exprs])
    outs = (OrcAggOut * len(exprs))()
    ok = C.POINTER(C.c_int64)()
    okv = C.POINTER(C.c_uint8)()
    ng = lib().orc_hash_aggregate(key.ctypes.data, _ptr(kv), key.dtype.itemsize, n,
                                  C.addressof(ca), len(cols), C.addressof(ea), len(exprs),
                                  int(ansi), C.byref(ok), C.byref(okv), C.addressof(outs))
    if ng == -3:
        raise OverflowError("ARITHMETIC_OVERFLOW")
    if ng < 0:
        raise RuntimeError(f"oracle aggregate failed: {ng}")
    m = max(ng, 1)
    keys = np.ctypeslib.as_array(ok, shape=(m,))[:ng].copy()
    kvalid = np.ctypeslib.as_array(okv, shape=(m,))[:ng].astype(bool)
    lib().orc_free(ok)
    lib().orc_free(okv)
    results = []
    for e in range(len(exprs)):
        o = outs[e]
        r = {}
        for name in ("i64", "f64", "f64_seq", "lo", "hi", "valid"):
            p = getattr(o, name)
            r[name] = np.ctypeslib.as_array(p, shape=(m,))[:ng].copy()
            lib().orc_free(p)
        r["valid"] = r["valid"].astype(bool)
        r["i128"] = [int(lo) + (int(hi) << 64) for lo, hi in zip(r["lo"], r["hi"])] \
            if ng and (r["hi"].any() or r["lo"].any()) else [0] * ng
        results.append(r)
    return keys, kvalid, results


def rand(seed, column, rows):
    L = lib()
    return np.array([L.orc_rand(seed, column, r) for r in rows], dtype=np.uint64)


def permute(seed, n, idx):
    L = lib()
    return np.array([L.orc_permute(seed, n, int(i)) for i in idx], dtype=np.int64)


GEN_DTYPE = {0: np.int64, 1: np.int32, 2: np.float64, 3: np.int64, 4: np.int64}


def gen_column(kind, seed, column, n, lo=0, hi=0, x0=0.0, x1=0.0, null_fraction=0.0, row0=0):
    """The synthetic column generator (the device generators' function)."""
    out = np.empty(n, dtype=GEN_DTYPE[kind])
    valid = np.empty(n, dtype=np.uint8) if null_fraction > 0 else None
    lib().orc_gen_column(seed, column, kind, lo, hi, x0, x1, row0, n, null_fraction, out.ctypes.data,
                         _ptr(valid))
    return out, valid


def zipf_cdf(s, n):
    cdf = np.empty(n, dtype=np.float64)
    lib().orc_zipf_cdf(s, n, cdf.ctypes.data)
    return cdf


def star_inputs(scale, seed, fact_row0=0, fact_rows=None, pred=7):
    """The star query's columns (the device generators' functions): fact rows
    [fact_row0, fact_row0 + fact_rows) and both dimensions in full."""
    nf, na, nb = int(300_000_000 * scale), int(20_000_000 * scale), int(1_000_000 * scale)
    n = nf if fact_rows is None else fact_rows
    r0 = dict(row0=fact_row0)
    fact = (gen_column(0, seed, 1, n, lo=0, hi=na - 1, **r0)[0], gen_column(0, seed, 2, n, lo=0, hi=nb - 1, **r0)[0],
            gen_column(0, seed, 3, n, lo=1000, hi=10_000_000, **r0)[0], gen_column(2, seed, 4, n, x0=0.0, x1=0.1, **r0)[0])
    dims = []
    for base, m in ((10, na), (20, nb)):
        dims.append((gen_column(3, seed + base, base + 1, m, lo=0, hi=m)[0], gen_column(1, seed, base + 2, m, lo=0, hi=19)[0],
                     gen_column(1, seed, base + 3, m, lo=0, hi=24)[0]))
    return fact, dims


def gen_column_mt(kind, seed, column, n, threads, lo=0, hi=0, x0=0.0, x1=0.0, row0=0, chunk=1 << 22):
    """gen_column over `threads` host threads (chunks of rows; the C calls
    release the interpreter lock). No NULLs."""
    from concurrent.futures import ThreadPoolExecutor
    out = np.empty(n, dtype=GEN_DTYPE[kind])
    L = lib()

    def work(a):
        b = min(n, a + chunk)
        L.orc_gen_column(seed, column, kind, lo, hi, x0, x1, row0 + a, b - a, 0.0, out[a:].ctypes.data, None)

    with ThreadPoolExecutor(max_workers=max(1, threads)) as ex:
        list(ex.map(work, range(0, n, chunk)))
    return out


def star_inputs_mt(scale, seed, threads, fact_rows=None, pred=7):
    """star_inputs with the fact columns generated on `threads` host threads."""
    nf, na, nb = int(300_000_000 * scale), int(20_000_000 * scale), int(1_000_000 * scale)
    n = nf if fact_rows is None else fact_rows
    fact = (gen_column_mt(0, seed, 1, n, threads, lo=0, hi=na - 1), gen_column_mt(0, seed, 2, n, threads, lo=0, hi=nb - 1),
            gen_column_mt(0, seed, 3, n, threads, lo=1000, hi=10_000_000),
            gen_column_mt(2, seed, 4, n, threads, x0=0.0, x1=0.1))
    dims = []
    for base, m in ((10, na), (20, nb)):
        dims.append((gen_column(3, seed + base, base + 1, m, lo=0, hi=m)[0], gen_column(1, seed, base + 2, m, lo=0, hi=19)[0],
                     gen_column(1, seed, base + 3, m, lo=0, hi=24)[0]))
    return fact, dims


def star_query(fact, dims, pred=7, group_by=0, threads=1, use_filters=True):
    """orc_star_query: {group: (sum, count)}, rows passing the filters, joined
    rows, build seconds, probe seconds."""
    L = lib()
    vp, i64, i32, dbl = C.c_void_p, C.c_int64, C.c_int32, C.c_double
    L.orc_star_query.restype = i64
    L.orc_star_query.argtypes = [vp, vp, vp, i64, i32, vp, vp, vp, i64, i32, vp, vp, vp, vp, i64, i32, i32, i32,
                                 vp, vp, C.POINTER(i64), C.POINTER(i64), C.POINTER(dbl), C.POINTER(dbl)]
    fk_a, fk_b, price, disc = fact
    (ka, pa, aa), (kb, pb, ab) = dims
    out_sum = np.zeros(4096)
    out_cnt = np.zeros(4096, dtype=np.int64)
    passed, joined, tb, tp = i64(), i64(), dbl(), dbl()
    L.orc_star_query(ka.ctypes.data, pa.ctypes.data, aa.ctypes.data, len(ka), pred, kb.ctypes.data, pb.ctypes.data,
                     ab.ctypes.data, len(kb), pred, fk_a.ctypes.data, fk_b.ctypes.data, price.ctypes.data,
                     disc.ctypes.data, len(fk_a), group_by, threads, 1 if use_filters else 0, out_sum.ctypes.data,
                     out_cnt.ctypes.data, C.byref(passed), C.byref(joined), C.byref(tb), C.byref(tp))
    groups = {int(g): (float(out_sum[g]), int(out_cnt[g])) for g in np.nonzero(out_cnt)[0]}
    return groups, passed.value, joined.value, tb.value, tp.value
