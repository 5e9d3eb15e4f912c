"""Helpers shared by the GPU parity tests: building pyarrow batches and
turning operator output back into comparable multisets."""
import collections

import numpy as np
import pyarrow as pa


def arr(values, valid=None, type=None):
    mask = None if valid is None else ~np.asarray(valid, dtype=bool)
    return pa.array(values, type=type, mask=mask)


def batch(**cols):
    names = list(cols)
    return pa.RecordBatch.from_arrays([cols[n] for n in names], names=names)


def concat(batches):
    batches = [b for b in batches if b is not None]
    if not batches:
        return None
    return pa.Table.from_batches(batches).combine_chunks()


def pairs_from_output(table, pid="pid", bid="bid"):
    """Multiset of (probe id or -1, build id or -1) of a join output with
    id columns on both sides."""
    if table is None or table.num_rows == 0:
        return collections.Counter()
    names = table.column_names
    p = table.column(pid).to_pylist() if pid in names else [None] * table.num_rows
    b = table.column(bid).to_pylist() if bid in names else [None] * table.num_rows
    return collections.Counter((-1 if x is None else x, -1 if y is None else y) for x, y in zip(p, b))


def rel_err(a, b):
    a, b = float(a), float(b)
    if a == b:
        return 0.0
    return abs(a - b) / max(abs(b), 1e-300)
