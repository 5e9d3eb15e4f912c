"""Parquet scan with runtime-filter row-group pruning, on the host.

Reference: the Krishiv engine lowers a published runtime filter to a
predicate on the scanned column (`ScanFilter::predicate`,
crates/krishiv-io/src/runtime_filter/mod.rs:418) that the Parquet reader
uses to skip row groups whose statistics admit no passing row; a NULL key
never passes unless the filter says so (`KeyFilter::nulls_pass`,
runtime_filter/filter.rs). Here the same test runs on the row groups'
min/max/null-count statistics against a key filter's summary
(`KeyFilter.info()`: its form, its key range, whether NULLs pass), and the
surviving row groups are decoded by pyarrow on the host into Arrow batches
that the operators take as host batches (or that a caller copies to the
device). Which row groups are read never changes a result: a skipped row
group holds no row that the filter passes.

`DeviceParquetScan` reads the same row groups, but hands each column chunk's
bytes, as the file stores them, to the device decoder
(`krv_parquet_decode_chunk`): pages are decompressed and decoded in HBM, and
the key filter is evaluated on the encoded pages (once per dictionary entry
of a dictionary-encoded chunk, as the reference's dictionary stage does,
crates/krishiv-io/src/parquet/dict_probe.rs); a row group whose key chunk
passes no row is skipped once that chunk is decoded, before its other
columns are read (the reference's `any_entry_in` skips a dictionary-encoded
one of them before its data pages)."""
from __future__ import annotations

from typing import Dict, Iterator, List, Optional, Sequence

FILTER_RANGE, FILTER_EXACT, FILTER_BLOOM, FILTER_EMPTY = 0, 1, 2, 3


def row_group_may_pass(stats, info: Dict[str, int]) -> bool:
    """Whether a row group whose key column has statistics `stats`
    (pyarrow's column-chunk Statistics, or None) may hold a row that the
    filter summarised by `info` passes."""
    if stats is None:
        return True
    nulls_pass = bool(info.get("nulls_pass", 0))
    has_nulls = (not stats.has_null_count) or stats.null_count > 0
    if nulls_pass and has_nulls:
        return True
    values = stats.num_values > 0 if stats.num_values is not None else True
    if info["form"] == FILTER_EMPTY:
        return False  # no key: only a NULL could pass, and it does not
    if not values:
        return False  # NULLs only, and they do not pass
    if not info.get("has_range", 0) or not stats.has_min_max:
        return True
    lo, hi = int(info["lo"]), int(info["hi"])
    try:
        mn, mx = int(stats.min), int(stats.max)
    except (TypeError, ValueError):
        return True
    return not (mx < lo or mn > hi)


def prune_row_groups(metadata, column: str, info: Optional[Dict[str, int]]) -> List[int]:
    """The row groups of a Parquet file (pyarrow FileMetaData) to read for a
    scan of `column` under the key filter `info` (None: all of them)."""
    n = metadata.num_row_groups
    if info is None:
        return list(range(n))
    names = [metadata.schema.column(i).path for i in range(metadata.num_columns)]
    if column not in names:
        # a missing column is NULL in every row (the reference lowers it to
        # a constant): the file is read only if NULLs pass
        return list(range(n)) if info.get("nulls_pass", 0) else []
    ci = names.index(column)
    keep = []
    for rg in range(n):
        cc = metadata.row_group(rg).column(ci)
        if row_group_may_pass(cc.statistics if cc.is_stats_set else None, info):
            keep.append(rg)
    return keep


class ParquetScan:
    """Reads a Parquet file's row groups that may pass a key filter, as Arrow
    record batches of at most `batch_rows` rows. `stats` says how many row
    groups and rows were read and skipped."""

    def __init__(self, path, columns: Optional[Sequence[str]] = None, key_column: Optional[str] = None,
                 filter_info: Optional[Dict[str, int]] = None, batch_rows: int = 1 << 20):
        import pyarrow.parquet as pq
        self.file = pq.ParquetFile(path)
        self.columns = list(columns) if columns is not None else None
        md = self.file.metadata
        self.row_groups = prune_row_groups(md, key_column, filter_info) if key_column else list(range(md.num_row_groups))
        self.batch_rows = batch_rows
        kept = sum(md.row_group(rg).num_rows for rg in self.row_groups)
        self.stats = {"row_groups": md.num_row_groups, "row_groups_read": len(self.row_groups),
                      "rows": md.num_rows, "rows_read": kept}

    def __iter__(self) -> Iterator:
        for rg in self.row_groups:
            t = self.file.read_row_group(rg, columns=self.columns)
            yield from t.to_batches(max_chunksize=self.batch_rows)


# pyarrow names of the Parquet physical types and codecs the device decoder takes
_PHYSICAL = {"INT32": 1, "INT64": 2, "DOUBLE": 5, "BYTE_ARRAY": 6}
_CODEC = {"UNCOMPRESSED": 0, "SNAPPY": 1}


def arrow_format(t) -> str:
    """The Arrow C format string of a pyarrow type the device decoder writes."""
    import pyarrow as pa
    if pa.types.is_int32(t):
        return "i"
    if pa.types.is_int64(t):
        return "l"
    if pa.types.is_float64(t):
        return "g"
    if pa.types.is_string(t):
        return "u"
    if pa.types.is_binary(t):
        return "z"
    if pa.types.is_date32(t):
        return "tdD"
    if pa.types.is_decimal(t):
        width = getattr(t, "bit_width", 128)
        return f"d:{t.precision},{t.scale}" + (",64" if width == 64 else "")
    raise ValueError(f"the device decoder does not write {t}")


def column_chunk(f, metadata, rg: int, ci: int):
    """The bytes of column chunk `ci` of row group `rg` (from its dictionary
    page, if any, through its last page) and the decoder's description of it."""
    cc = metadata.row_group(rg).column(ci)
    start = cc.dictionary_page_offset if cc.has_dictionary_page and cc.dictionary_page_offset else cc.data_page_offset
    f.seek(start)
    data = f.read(cc.total_compressed_size)
    if cc.physical_type not in _PHYSICAL or cc.compression not in _CODEC:
        raise ValueError(f"column chunk of {cc.physical_type} / {cc.compression}: not taken by the device decoder")
    desc = {"physical_type": _PHYSICAL[cc.physical_type], "codec": _CODEC[cc.compression],
            "max_def_level": metadata.schema.column(ci).max_definition_level, "num_values": cc.num_values}
    return data, desc


class DeviceParquetScan:
    """The row groups of a Parquet file that may pass a key filter, decoded on
    the device: each yields (row group, {column: DeviceResult}, pass) where
    `pass` is the key filter's DeviceResult "pass" column over the key column
    (None without a filter). Row groups skipped on their statistics, or
    after their key chunk passed no row, are counted in `stats`."""

    def __init__(self, rt, path, columns: Sequence[str], key_column: Optional[str] = None, key_filter=None):
        import pyarrow.parquet as pq
        self.rt = rt
        self.path = path
        self.pf = pq.ParquetFile(path)
        md = self.pf.metadata
        self.columns = list(columns)
        self.key_column = key_column
        self.key_filter = key_filter
        info = key_filter.info() if key_filter is not None else None
        self.row_groups = prune_row_groups(md, key_column, info) if key_column else list(range(md.num_row_groups))
        names = [md.schema.column(i).path for i in range(md.num_columns)]
        self.index = {c: names.index(c) for c in set(self.columns) | ({key_column} if key_column else set())}
        self.types = {c: self.pf.schema_arrow.field(c).type for c in self.index}
        self.stats = {"row_groups": md.num_row_groups, "row_groups_after_statistics": len(self.row_groups),
                      "row_groups_skipped_after_key_decode": 0, "rows": md.num_rows}

    def _decode(self, f, rg, c, key_filter=None):
        from importlib import import_module
        kb = import_module(__name__.rsplit(".", 1)[0])
        data, d = column_chunk(f, self.pf.metadata, rg, self.index[c])
        return kb.parquet_decode_chunk(self.rt, data, d["physical_type"], d["codec"], d["max_def_level"],
                                       d["num_values"], arrow_format(self.types[c]), c, key_filter)

    def __iter__(self):
        with open(self.path, "rb") as f:
            for rg in self.row_groups:
                cols, passing = {}, None
                if self.key_column and self.key_filter is not None:
                    res, info = self._decode(f, rg, self.key_column, self.key_filter)
                    if info["passing_rows"] == 0:
                        # no row passes (with a dictionary: no entry did): the other columns are not read
                        self.stats["row_groups_skipped_after_key_decode"] += 1
                        continue
                    cols[self.key_column] = res
                    passing = res
                for c in self.columns:
                    if c not in cols:
                        cols[c] = self._decode(f, rg, c)[0]
                yield rg, cols, passing
