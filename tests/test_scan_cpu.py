"""Parquet scan with runtime-filter row-group pruning (host side): a row
group is skipped only when its key statistics admit no row that the filter
passes (out of the filter's key range, NULLs only when NULLs do not pass, an
empty filter), so every passing row of the file is read; files without
statistics, a missing key column and NULL-passing filters are read whole."""
import importlib

import numpy as np
import pyarrow as pa
import pyarrow.parquet as pq
import pytest


def S():
    return importlib.import_module("krishiv-engine_b200.scan")


def info(form=0, lo=0, hi=-1, nulls_pass=0, has_range=1):
    return {"form": form, "lo": lo, "hi": hi, "nulls_pass": nulls_pass, "has_range": has_range}


@pytest.fixture
def sorted_file(tmp_path):
    """10 row groups of 1,000 rows, keys ascending 0..9,999; row group 7 has
    NULL keys in place of its even rows; row group 9 holds NULLs only."""
    n = 10_000
    k = np.arange(n, dtype=np.int64)
    valid = np.ones(n, bool)
    valid[7000:8000:2] = False
    valid[9000:] = False
    t = pa.table({"k": pa.array(k, mask=~valid), "v": pa.array(k * 3)})
    path = tmp_path / "sorted.parquet"
    pq.write_table(t, path, row_group_size=1000)
    return path, k, valid


def test_range_pruning(sorted_file):
    path, k, valid = sorted_file
    md = pq.ParquetFile(path).metadata
    s = S()
    assert s.prune_row_groups(md, "k", info(lo=2500, hi=4100)) == [2, 3, 4]
    assert s.prune_row_groups(md, "k", info(lo=-50, hi=-1)) == []
    assert s.prune_row_groups(md, "k", info(lo=7001, hi=7001)) == [7]
    assert s.prune_row_groups(md, "k", info(lo=9500, hi=20000)) == []  # row group 9: NULLs only
    # NULLs pass: the row groups with NULLs are read as well
    assert s.prune_row_groups(md, "k", info(lo=0, hi=10, nulls_pass=1)) == [0, 7, 9]
    # no range known (a Bloom form without one): only the NULLs-only row group is skipped
    assert s.prune_row_groups(md, "k", info(form=2, has_range=0)) == list(range(9))
    # an empty filter passes no key: only NULL rows could pass
    assert s.prune_row_groups(md, "k", info(form=3)) == []
    assert s.prune_row_groups(md, "k", info(form=3, nulls_pass=1)) == [7, 9]
    assert s.prune_row_groups(md, "k", None) == list(range(10))


def test_missing_column_and_missing_statistics(tmp_path, sorted_file):
    path, _, _ = sorted_file
    md = pq.ParquetFile(path).metadata
    s = S()
    assert s.prune_row_groups(md, "absent", info(lo=0, hi=5)) == []
    assert s.prune_row_groups(md, "absent", info(lo=0, hi=5, nulls_pass=1)) == list(range(10))
    p2 = tmp_path / "nostats.parquet"
    pq.write_table(pa.table({"k": pa.array(np.arange(3000, dtype=np.int64))}), p2, row_group_size=1000,
                   write_statistics=False)
    assert s.prune_row_groups(pq.ParquetFile(p2).metadata, "k", info(lo=-9, hi=-5)) == [0, 1, 2]


def test_scan_reads_every_passing_row(tmp_path):
    """Random keys in row groups of mixed ranges, random filter ranges: the
    rows the filter's range passes in the whole file are exactly those it
    passes in the batches the scan reads."""
    rng = np.random.default_rng(5)
    parts = [rng.integers(lo, lo + 500, 700) for lo in rng.integers(0, 20_000, 30)]
    k = np.concatenate(parts).astype(np.int64)
    v = np.arange(k.size, dtype=np.int64)
    path = tmp_path / "mixed.parquet"
    pq.write_table(pa.table({"k": k, "v": v}), path, row_group_size=700)
    s = S()
    for _ in range(40):
        lo = int(rng.integers(-100, 20_000))
        hi = lo + int(rng.integers(0, 3000))
        scan = s.ParquetScan(path, columns=["k", "v"], key_column="k", filter_info=info(lo=lo, hi=hi), batch_rows=256)
        got = set()
        for b in scan:
            kk = b.column(0).to_numpy()
            vv = b.column(1).to_numpy()
            got |= set(vv[(kk >= lo) & (kk <= hi)].tolist())
        want = set(v[(k >= lo) & (k <= hi)].tolist())
        assert got == want
        assert scan.stats["row_groups"] == 30 and scan.stats["row_groups_read"] <= 30
        assert scan.stats["rows_read"] == 700 * scan.stats["row_groups_read"]


def test_column_chunk_bytes_and_description(tmp_path):
    """The bytes the device decoder is handed for a column chunk: from its
    dictionary page (a dictionary-encoded chunk) or its first data page,
    `total_compressed_size` bytes, starting with a Thrift compact PageHeader
    whose first field is the page type (DICTIONARY_PAGE 2, DATA_PAGE 0,
    DATA_PAGE_V2 3); the description carries the physical type, codec,
    maximum definition level and value count; the Arrow formats."""
    S = importlib.import_module("krishiv-engine_b200.scan")
    n = 10_000
    t = pa.table({"k": pa.array(np.arange(n) % 7, type=pa.int64()),
                  "x": pa.array(np.linspace(0, 1, n)),
                  "s": pa.array([None if i % 5 == 0 else "v%d" % (i % 3) for i in range(n)]),
                  "r": pa.array(np.arange(n, dtype=np.int32))})
    schema = pa.schema([pa.field("k", pa.int64()), pa.field("x", pa.float64()), pa.field("s", pa.string()),
                        pa.field("r", pa.int32(), nullable=False)])
    t = t.cast(schema)
    for version, data_type in (("1.0", 0), ("2.0", 3)):
        path = str(tmp_path / f"c{version}.parquet")
        pq.write_table(t, path, use_dictionary=["k", "s"], compression="SNAPPY", data_page_version=version)
        md = pq.ParquetFile(path).metadata
        with open(path, "rb") as f:
            for ci, (phys, dict_, max_def) in enumerate(((2, True, 1), (5, False, 1), (6, True, 1), (1, False, 0))):
                data, d = S.column_chunk(f, md, 0, ci)
                cc = md.row_group(0).column(ci)
                assert len(data) == cc.total_compressed_size
                assert d == {"physical_type": phys, "codec": 1, "max_def_level": max_def, "num_values": n}
                # field 1 (delta 1, i32) of the PageHeader: the page type, zigzag-coded
                assert data[0] == 0x15 and data[1] == 2 * (2 if dict_ else data_type)
    fmt = {pa.int32(): "i", pa.int64(): "l", pa.float64(): "g", pa.date32(): "tdD", pa.string(): "u",
           pa.binary(): "z", pa.decimal128(15, 2): "d:15,2"}
    for typ, want in fmt.items():
        assert S.arrow_format(typ) == want
    with pytest.raises(ValueError):
        S.arrow_format(pa.list_(pa.int64()))
