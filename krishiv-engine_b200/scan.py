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

Decoding Parquet pages on the device is not done here."""
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
