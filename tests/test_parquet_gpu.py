"""Parquet column chunks decoded on the device (krv_parquet_decode_chunk)
against pyarrow's decode of the same file, bit for bit: values and validity,
over PLAIN and dictionary-encoded pages, UNCOMPRESSED and SNAPPY chunks, data
pages v1 and v2, required and optional columns, many pages and row groups,
a dictionary that overflows into PLAIN pages, all-NULL and single-value
columns. The key filter's "pass" column, evaluated on the encoded pages
(once per dictionary entry, or per PLAIN value), equals the CPU oracle's
filter over the decoded keys (crates/krishiv-io/src/runtime_filter/
filter.rs:776-798, KeyFilter::evaluate_keys; the dictionary stage of
crates/krishiv-io/src/parquet/dict_probe.rs)."""
import numpy as np
import pyarrow as pa
import pyarrow.parquet as pq
import pytest

pytestmark = pytest.mark.gpu


def write(tmp_path, table, name="t.parquet", **kw):
    path = str(tmp_path / name)
    pq.write_table(table, path, **kw)
    return path


def bits(res, col):
    v = res.valid[col]
    if v is None:
        return np.ones(res.rows, bool)
    return np.unpackbits(v.cpu().numpy(), bitorder="little")[: res.rows].astype(bool)


def decode_all(kb, rt, path, column, key_filter=None):
    """Every row group's chunk of `column` decoded on the device: (values,
    validity, pass or None, infos) concatenated over the row groups."""
    from importlib import import_module
    S = import_module("krishiv-engine_b200.scan")
    pf = pq.ParquetFile(path)
    md = pf.metadata
    names = [md.schema.column(i).path for i in range(md.num_columns)]
    ci = names.index(column)
    t = pf.schema_arrow.field(column).type
    vals, valid, passes, infos = [], [], [], []
    with open(path, "rb") as f:
        for rg in range(md.num_row_groups):
            data, d = S.column_chunk(f, md, rg, ci)
            res, info = kb.parquet_decode_chunk(rt, data, d["physical_type"], d["codec"], d["max_def_level"],
                                                d["num_values"], S.arrow_format(t), column, key_filter)
            infos.append(info)
            assert res.rows == info["rows"] == d["num_values"]
            if res.rows == 0:
                continue
            vals.append(res.columns[0].cpu().numpy())
            valid.append(bits(res, 0))
            if key_filter is not None:
                passes.append(np.unpackbits(res.columns[1].cpu().numpy(), bitorder="little")[: res.rows].astype(bool))
    cat = lambda xs: np.concatenate(xs) if xs else np.zeros(0)
    return cat(vals), cat(valid).astype(bool), (cat(passes).astype(bool) if key_filter is not None else None), infos


def expect(path, column):
    """pyarrow's decode: (values as numpy with NULLs zeroed, validity)."""
    a = pq.read_table(path, columns=[column]).column(0).combine_chunks()
    valid = np.ones(len(a), bool) if a.null_count == 0 else np.asarray(a.is_valid())
    return a, valid


def check_same(kb, rt, path, column):
    got, gvalid, _, infos = decode_all(kb, rt, path, column)
    a, valid = expect(path, column)
    assert np.array_equal(gvalid, valid)
    t = a.type
    if pa.types.is_decimal(t):
        want = np.array([int(x.as_py().scaleb(t.scale)) if x.is_valid else 0 for x in a], dtype=np.int64)
        lo = got.reshape(-1, 2)[:, 0] if t.bit_width == 128 else got
        assert np.array_equal(lo[valid], want[valid])
        if t.bit_width == 128:
            hi = got.reshape(-1, 2)[:, 1]
            assert np.array_equal(hi[valid], np.where(want[valid] < 0, -1, 0))
    else:
        np_t = {"int32": np.int32, "int64": np.int64, "double": np.float64, "date32[day]": np.int32}[str(t)]
        want = a.cast(pa.int32() if str(t) == "date32[day]" else t).fill_null(0).to_numpy(zero_copy_only=False)
        want = want.astype(np_t)
        # bit patterns (NaN and -0.0 included)
        g = got.view(np.int64 if np_t in (np.int64, np.float64) else np.int32)
        w = want.view(np.int64 if np_t in (np.int64, np.float64) else np.int32)
        assert np.array_equal(g[valid], w[valid])
    return infos


def keys_with_nulls(n, seed=1, dom=50_000, null_frac=0.05):
    rng = np.random.default_rng(seed)
    k = rng.integers(-dom, dom, n).astype(np.int64)
    valid = rng.random(n) >= null_frac
    return pa.array(k, mask=~valid)


@pytest.mark.parametrize("compression", ["NONE", "SNAPPY"])
@pytest.mark.parametrize("use_dictionary", [True, False])
@pytest.mark.parametrize("page_version", ["1.0", "2.0"])
def test_int64_with_nulls(kb, rt, tmp_path, compression, use_dictionary, page_version):
    n = 300_000
    t = pa.table({"k": keys_with_nulls(n)})
    path = write(tmp_path, t, compression=compression, use_dictionary=use_dictionary, data_page_version=page_version,
                 row_group_size=110_000, data_page_size=64 << 10)
    infos = check_same(kb, rt, path, "k")
    assert len(infos) == 3 and sum(i["pages"] for i in infos) > 3
    assert all((i["dictionary_entries"] > 0) == use_dictionary for i in infos)


@pytest.mark.parametrize("compression", ["NONE", "SNAPPY"])
def test_types(kb, rt, tmp_path, compression):
    rng = np.random.default_rng(4)
    n = 70_001
    f = rng.standard_normal(n)
    f[:7] = [np.nan, -0.0, 0.0, np.inf, -np.inf, 1e-308, -5e-324]
    cents = rng.integers(-10**13, 10**13, n)
    t = pa.table({
        "i32": pa.array(rng.integers(-2**31, 2**31, n).astype(np.int32), mask=rng.random(n) < 0.02),
        "d": pa.array(rng.integers(-20_000, 20_000, n).astype(np.int32), type=pa.date32()),
        "f": pa.array(f, mask=rng.random(n) < 0.02),
        "dec": pa.array([None if i % 37 == 0 else __import__("decimal").Decimal(int(c)).scaleb(-2)
                         for i, c in enumerate(cents)], type=pa.decimal128(15, 2)),
        "small": pa.array(rng.integers(0, 4, n).astype(np.int64)),  # a 4-entry dictionary
        "one": pa.array(np.full(n, 42, np.int64)),                  # a 1-entry dictionary (bit width 0)
    })
    path = write(tmp_path, t, compression=compression, store_decimal_as_integer=True, data_page_size=32 << 10,
                 row_group_size=40_000)
    for c in t.column_names:
        check_same(kb, rt, path, c)


def test_required_column_and_v2_plain(kb, rt, tmp_path):
    n = 123_457
    rng = np.random.default_rng(9)
    schema = pa.schema([pa.field("k", pa.int64(), nullable=False), pa.field("x", pa.int32(), nullable=False)])
    t = pa.table({"k": rng.integers(-2**62, 2**62, n).astype(np.int64),
                  "x": rng.integers(0, 1000, n).astype(np.int32)}, schema=schema)
    for version in ("1.0", "2.0"):
        path = write(tmp_path, t, name=f"r{version}.parquet", compression="SNAPPY", data_page_version=version,
                     use_dictionary=["x"], data_page_size=16 << 10)
        for c in ("k", "x"):
            check_same(kb, rt, path, c)


def test_dictionary_overflows_into_plain_pages(kb, rt, tmp_path):
    """A dictionary larger than dictionary_pagesize_limit: the writer falls
    back to PLAIN pages part way, so the chunk mixes both encodings, and the
    dictionary alone cannot decide the filter."""
    n = 200_000
    t = pa.table({"k": keys_with_nulls(n, seed=5, dom=10**9)})
    path = write(tmp_path, t, compression="SNAPPY", dictionary_pagesize_limit=16 << 10, data_page_size=16 << 10)
    infos = check_same(kb, rt, path, "k")
    assert infos[0]["dictionary_entries"] > 0
    keys = np.arange(0, 10**6, dtype=np.int64)
    kf = kb.KeyFilter.build(rt, pa.record_batch([pa.array(keys)], names=["k"]), 0)
    _, _, _, infos = decode_all(kb, rt, path, "k", kf)
    assert infos[0]["dictionary_passing"] == -1


def test_all_null_and_empty_pages(kb, rt, tmp_path):
    n = 50_000
    k = np.zeros(n, np.int64)
    mask = np.ones(n, bool)
    mask[40_000:40_010] = False  # ten values at the end of the chunk; most pages are all NULL
    k[40_000:40_010] = np.arange(10)
    t = pa.table({"k": pa.array(k, mask=mask), "z": pa.array([None] * n, type=pa.int64())})
    for dict_ in (True, False):
        path = write(tmp_path, t, name=f"n{dict_}.parquet", compression="SNAPPY", use_dictionary=dict_,
                     data_page_size=4 << 10)
        check_same(kb, rt, path, "k")
        check_same(kb, rt, path, "z")


@pytest.mark.parametrize("use_dictionary", [True, False])
@pytest.mark.parametrize("form", ["bloom", "exact", "range"])
def test_key_filter_on_encoded_pages(kb, rt, oracle, tmp_path, use_dictionary, form):
    n = 250_000
    col = keys_with_nulls(n, seed=11, dom=100_000)
    t = pa.table({"k": col})
    path = write(tmp_path, t, compression="SNAPPY", use_dictionary=use_dictionary, data_page_size=32 << 10,
                 row_group_size=100_000)
    rng = np.random.default_rng(12)
    size = {"bloom": 20_000, "exact": 1_000, "range": 5_000_000}[form]
    build = rng.integers(-100_000, 100_000, size).astype(np.int64)
    kf = kb.KeyFilter.build(rt, pa.record_batch([pa.array(build)], names=["k"]), 0)
    want_form = {"bloom": 2, "exact": 1, "range": 0}[form]
    assert kf.info()["form"] == want_form
    got, valid, passing, infos = decode_all(kb, rt, path, "k", kf)
    ref = oracle.KeyFilter(build)
    assert ref.form == want_form
    a, avalid = expect(path, "k")
    keys = a.fill_null(0).to_numpy(zero_copy_only=False).astype(np.int64)
    want = ref.evaluate(keys, avalid.astype(np.uint8))
    assert np.array_equal(passing, want)
    assert sum(i["passing_rows"] for i in infos) == int(want.sum())
    if use_dictionary:
        # the dictionary decides: its passing entries are the distinct passing keys of the chunk
        for rg, info in enumerate(infos):
            lo, hi = rg * 100_000, min(n, (rg + 1) * 100_000)
            m = avalid[lo:hi] & want[lo:hi]
            assert info["dictionary_passing"] == len(np.unique(keys[lo:hi][m]))


def test_device_scan_skips_row_groups_no_key_passes(kb, rt, tmp_path):
    """Row groups of disjoint key ranges: the statistics skip what they can;
    a row group whose range overlaps the filter but whose keys all miss it is
    skipped after its key chunk is decoded; the rest decode every column."""
    from importlib import import_module
    S = import_module("krishiv-engine_b200.scan")
    groups = []
    for g in range(4):
        k = np.arange(g * 1000, g * 1000 + 1000, 2, dtype=np.int64)  # even keys
        groups.append(pa.table({"k": k, "v": k * 3}))
    path = write(tmp_path, pa.concat_tables(groups), row_group_size=500, compression="SNAPPY")
    # odd keys in 1000..1999 (no row passes, the range overlaps), even keys in 3000..3999
    build = np.concatenate([np.arange(1001, 2000, 2), np.arange(3000, 4000, 2)]).astype(np.int64)
    kf = kb.KeyFilter.build(rt, pa.record_batch([pa.array(build)], names=["k"]), 0)
    scan = S.DeviceParquetScan(rt, path, ["k", "v"], key_column="k", key_filter=kf)
    seen = []
    for rg, cols, passing in scan:
        p = np.unpackbits(passing.columns[1].cpu().numpy(), bitorder="little")[: passing.rows].astype(bool)
        k = cols["k"].columns[0].cpu().numpy()
        v = cols["v"].columns[0].cpu().numpy()
        assert np.array_equal(v, k * 3)
        seen.append((rg, int(p.sum())))
    assert seen == [(3, 500)]
    assert scan.stats["row_groups_after_statistics"] == 3  # group 0 below the filter's range
    assert scan.stats["row_groups_skipped_after_key_decode"] == 2  # groups 1 (odd keys) and 2 (Bloom/exact miss)


def test_corrupt_and_unsupported_chunks_fail_cleanly(kb, rt, tmp_path):
    n = 10_000
    t = pa.table({"k": pa.array(np.arange(n, dtype=np.int64)), "s": pa.array([str(i) for i in range(n)])})
    path = write(tmp_path, t, compression="SNAPPY", use_dictionary=False)
    from importlib import import_module
    S = import_module("krishiv-engine_b200.scan")
    md = pq.ParquetFile(path).metadata
    with open(path, "rb") as f:
        data, d = S.column_chunk(f, md, 0, 0)
    ok, _ = kb.parquet_decode_chunk(rt, data, d["physical_type"], d["codec"], d["max_def_level"], n, "l")
    assert ok.rows == n
    # truncated: the header walk ends early
    with pytest.raises(kb.KrvError):
        kb.parquet_decode_chunk(rt, data[: len(data) // 2], d["physical_type"], d["codec"], d["max_def_level"], n, "l")
    # flipped payload bytes (the Snappy stream or the values no longer decode, or decode to other values)
    bad = bytearray(data)
    for i in range(len(bad) // 3, len(bad), 97):
        bad[i] ^= 0x5A
    try:
        r, _ = kb.parquet_decode_chunk(rt, bytes(bad), d["physical_type"], d["codec"], d["max_def_level"], n, "l")
        assert r.rows == n
    except kb.KrvError as e:
        assert e.status in (kb.INVALID_ARGUMENT,)
    # other codecs and physical types
    with pytest.raises(kb.KrvError):
        kb.parquet_decode_chunk(rt, data, d["physical_type"], 6, d["max_def_level"], n, "l")  # ZSTD
    with pytest.raises(kb.KrvError):
        kb.parquet_decode_chunk(rt, data, 7, d["codec"], d["max_def_level"], n, "l")  # FIXED_LEN_BYTE_ARRAY
    with pytest.raises(kb.KrvError):
        kb.parquet_decode_chunk(rt, data, d["physical_type"], d["codec"], d["max_def_level"], n, "u")  # INT64 as UTF-8


def _varint(v):
    out = bytearray()
    while True:
        b = v & 0x7F
        v >>= 7
        out.append(b | (0x80 if v else 0))
        if not v:
            return bytes(out)


def _i32_field(delta, v):
    return bytes([(delta << 4) | 5]) + _varint(((v << 1) ^ (v >> 31)) & 0xFFFFFFFF)


def _data_page(payload, usize, n):
    """A Thrift compact PageHeader of a v1 data page (PLAIN values, RLE levels)."""
    dph = _i32_field(1, n) + _i32_field(1, 0) + _i32_field(1, 3) + _i32_field(1, 3) + b"\x00"
    return (_i32_field(1, 0) + _i32_field(1, usize) + _i32_field(1, len(payload)) + bytes([(2 << 4) | 12]) + dph
            + b"\x00" + payload)


def test_snappy_back_references_across_fragments(kb, rt):
    """A Snappy page written by hand (not by Google's compressor): a 72 KB
    literal, then the same bytes again as 64-byte back-references 72,000
    bytes behind, so that references reach across the 64 KiB points where
    the decoder would split the stream: the fragments merge, the far
    references read back, and the values are exact; a second page of short
    overlapping references (offset 8) follows."""
    rng = np.random.default_rng(8)
    half = rng.integers(-2**62, 2**62, 9000).astype(np.int64)
    raw1 = half.tobytes() * 2
    body = bytearray(_varint(len(raw1)))
    body += bytes([62 << 2]) + (len(half.tobytes()) - 1).to_bytes(3, "little") + half.tobytes()
    for _ in range(len(half.tobytes()) // 64):
        body += bytes([(63 << 2) | 3]) + (len(half.tobytes())).to_bytes(4, "little")
    v8 = np.full(30_000, 7, np.int64)  # 240 KB of one value: a literal of 8 bytes, then offset-8 copies
    raw2 = v8.tobytes()
    body2 = bytearray(_varint(len(raw2))) + bytes([7 << 2]) + raw2[:8]
    left = len(raw2) - 8
    while left:
        n = min(64, left)
        body2 += bytes([((n - 1) << 2) | 2]) + (8).to_bytes(2, "little")
        left -= n
    chunk = _data_page(bytes(body), len(raw1), 2 * half.size) + _data_page(bytes(body2), len(raw2), v8.size)
    res, info = kb.parquet_decode_chunk(rt, chunk, kb.PQ_INT64, kb.PQ_SNAPPY, 0, 2 * half.size + v8.size, "l")
    assert info["pages"] == 2 and res.rows == 2 * half.size + v8.size
    got = res.columns[0].cpu().numpy()
    assert np.array_equal(got, np.concatenate([half, half, v8]))


def strings_of(res):
    """A decoded UTF-8 / binary column as Python values (None for NULL)."""
    if res.rows == 0:
        return []
    offs = res.columns[0].cpu().numpy()
    heap = res.heaps[0].cpu().numpy().tobytes() if res.heaps[0] is not None else b""
    valid = bits(res, 0)
    return [heap[offs[i]:offs[i + 1]] if valid[i] else None for i in range(res.rows)]


@pytest.mark.parametrize("compression", ["NONE", "SNAPPY"])
@pytest.mark.parametrize("use_dictionary", [True, False])
@pytest.mark.parametrize("page_version", ["1.0", "2.0"])
def test_string_and_binary_columns(kb, rt, tmp_path, compression, use_dictionary, page_version):
    """BYTE_ARRAY chunks (UTF-8 and binary, NULLs, empty values, values of
    a few KB, many pages and row groups, a dictionary of repeated strings)
    decode to pyarrow's values byte for byte."""
    from importlib import import_module
    S = import_module("krishiv-engine_b200.scan")
    rng = np.random.default_rng(31)
    n = 60_000
    words = ["", "a", "krishiv", "ä-ö-ü", "x" * 3000] + ["w%05d" % i for i in range(2000)]
    s = [None if rng.random() < 0.03 else words[int(rng.integers(0, len(words)))] for _ in range(n)]
    b = [None if rng.random() < 0.03 else bytes(rng.integers(0, 256, int(rng.integers(0, 40)), dtype=np.uint8))
         for _ in range(n)]
    t = pa.table({"s": pa.array(s, pa.string()), "b": pa.array(b, pa.binary())})
    path = write(tmp_path, t, compression=compression, use_dictionary=use_dictionary, data_page_version=page_version,
                 row_group_size=25_000, data_page_size=16 << 10)
    pf = pq.ParquetFile(path)
    md = pf.metadata
    for ci, name in enumerate(("s", "b")):
        got = []
        with open(path, "rb") as f:
            for rg in range(md.num_row_groups):
                data, d = S.column_chunk(f, md, rg, ci)
                res, info = kb.parquet_decode_chunk(rt, data, d["physical_type"], d["codec"], d["max_def_level"],
                                                    d["num_values"], S.arrow_format(pf.schema_arrow.field(name).type),
                                                    name)
                assert res.formats[0] == ("u" if name == "s" else "z")
                got += strings_of(res)
        want = [x.encode() if isinstance(x, str) else x for x in pq.read_table(path, columns=[name]).column(0).to_pylist()]
        assert got == want


def test_string_filter_is_unsupported(kb, rt, tmp_path):
    from importlib import import_module
    S = import_module("krishiv-engine_b200.scan")
    path = write(tmp_path, pa.table({"s": pa.array(["a", "b"])}))
    md = pq.ParquetFile(path).metadata
    with open(path, "rb") as f:
        data, d = S.column_chunk(f, md, 0, 0)
    kf = kb.KeyFilter.build(rt, pa.record_batch([pa.array(np.arange(5, dtype=np.int64))], names=["k"]), 0)
    with pytest.raises(kb.KrvError) as e:
        kb.parquet_decode_chunk(rt, data, d["physical_type"], d["codec"], d["max_def_level"], 2, "u", "s", kf)
    assert e.value.status == kb.UNSUPPORTED
