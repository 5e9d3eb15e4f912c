"""Python binding of libkrv_gpu.so, the B200 hash join, grouped aggregate and
runtime key filter operators (C ABI: include/krv_gpu.h).

The package directory name has a hyphen, so import it with importlib:

    kb = importlib.import_module("krishiv-engine_b200")

Data crosses as Arrow record batches: pyarrow batches through the Arrow C Data
Interface (host buffers), or device columns (torch CUDA tensors) through the
Arrow C Device Data Interface. There is no CPU fallback: if the CUDA library
is missing every call fails.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Dict, List, Optional, Sequence

HERE = os.path.dirname(os.path.abspath(__file__))
# KRV_LIB_PATH selects another build of the library (e.g. an installed copy).
LIB_PATH = os.environ.get("KRV_LIB_PATH") or os.path.join(HERE, "libkrv_gpu.so")

# ---- status codes (krv_gpu.h) --------------------------------------------------------
OK, NEED_MORE_INPUT, HAVE_MORE_OUTPUT, FINISHED = 0, 1, 2, 3
INVALID_ARGUMENT, UNSUPPORTED, NEED_MEMORY, ARITHMETIC_OVERFLOW = -1, -2, -3, -4
CUDA_ERROR, TIMEOUT, TOO_MANY_ROWS, INTERNAL = -5, -6, -7, -8

INNER, LEFT_OUTER, LEFT_SEMI, LEFT_ANTI, NULL_AWARE_ANTI, EXISTENCE = 0, 1, 2, 3, 4, 5
RIGHT_SEMI, RIGHT_ANTI, RIGHT_OUTER, FULL_OUTER = 6, 7, 8, 9
JOIN_TYPES = {"inner": INNER, "left_outer": LEFT_OUTER, "left_semi": LEFT_SEMI, "left_anti": LEFT_ANTI,
              "null_aware_anti": NULL_AWARE_ANTI, "existence": EXISTENCE, "right_semi": RIGHT_SEMI,
              "right_anti": RIGHT_ANTI, "right_outer": RIGHT_OUTER, "full_outer": FULL_OUTER}

COUNT_STAR, COUNT, SUM, MIN, MAX, AVG = 0, 1, 2, 3, 4, 5
AGG_FUNCS = {"count_star": COUNT_STAR, "count": COUNT, "sum": SUM, "min": MIN, "max": MAX, "avg": AVG}
MODE_AUTO, MODE_GLOBAL, MODE_SHARED = 0, 1, 2
AGG_INPUT_RAW, AGG_INPUT_STATE = 0, 1
AGG_OUTPUT_FINAL, AGG_OUTPUT_PARTIAL = 0, 1

FILTER_RANGE, FILTER_EXACT, FILTER_BLOOM, FILTER_EMPTY = 0, 1, 2, 3
STAR_FUSED, STAR_PLAIN = 0, 1

GEN_UNIFORM_I64, GEN_UNIFORM_I32, GEN_UNIT_F64, GEN_PERMUTATION, GEN_ZIPF = 0, 1, 2, 3, 4

MAX_KEYS = 4
MAX_GROUP_KEYS = 8
MAX_OUT = 32
MAX_AGGS = 32
SCRATCH_MAX_GROUPS = 65536  # KRV_SCRATCH_MAX_GROUPS
SERVE_BATCHED, SERVE_PLAIN = 0, 1


class KrvError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"[{status}] {msg}")
        self.status = status


# ---- Arrow C (Device) Data Interface --------------------------------------------------
class ArrowSchema(C.Structure):
    pass


ArrowSchema._fields_ = [("format", C.c_char_p), ("name", C.c_char_p), ("metadata", C.c_char_p),
                        ("flags", C.c_int64), ("n_children", C.c_int64),
                        ("children", C.POINTER(C.POINTER(ArrowSchema))),
                        ("dictionary", C.POINTER(ArrowSchema)),
                        ("release", C.CFUNCTYPE(None, C.POINTER(ArrowSchema))),
                        ("private_data", C.c_void_p)]


class ArrowArray(C.Structure):
    pass


ArrowArray._fields_ = [("length", C.c_int64), ("null_count", C.c_int64), ("offset", C.c_int64),
                       ("n_buffers", C.c_int64), ("n_children", C.c_int64),
                       ("buffers", C.POINTER(C.c_void_p)),
                       ("children", C.POINTER(C.POINTER(ArrowArray))),
                       ("dictionary", C.POINTER(ArrowArray)),
                       ("release", C.CFUNCTYPE(None, C.POINTER(ArrowArray))),
                       ("private_data", C.c_void_p)]


class ArrowDeviceArray(C.Structure):
    _fields_ = [("array", ArrowArray), ("device_id", C.c_int64), ("device_type", C.c_int32),
                ("sync_event", C.c_void_p), ("reserved", C.c_int64 * 3)]


ARROW_DEVICE_CUDA = 2

# ---- specs (krv_gpu.h) ------------------------------------------------------------------
class JoinSpec(C.Structure):
    _fields_ = [("join_type", C.c_int32), ("n_keys", C.c_int32), ("probe_keys", C.c_int32 * MAX_KEYS),
                ("build_keys", C.c_int32 * MAX_KEYS), ("null_safe", C.c_int32 * MAX_KEYS),
                ("single_match", C.c_int32), ("has_residual_filter", C.c_int32),
                ("n_probe_out", C.c_int32), ("probe_out", C.c_int32 * MAX_OUT),
                ("n_build_out", C.c_int32), ("build_out", C.c_int32 * MAX_OUT),
                ("radix_bits", C.c_int32), ("max_load", C.c_float), ("seed", C.c_uint64),
                ("runtime_filter", C.c_int32), ("pad0", C.c_int32), ("build_rows_hint", C.c_int64),
                ("max_output_rows", C.c_int64)]


CMP = {"=": 0, "!=": 1, "<": 2, "<=": 3, ">": 4, ">=": 5}
OPERAND_PROBE, OPERAND_BUILD, OPERAND_CONST_I64, OPERAND_CONST_F64 = 0, 1, 2, 3
MAX_FILTER_TERMS = 8


class FilterOperand(C.Structure):
    _fields_ = [("kind", C.c_int32), ("column", C.c_int32), ("i64", C.c_int64), ("f64", C.c_double)]


class FilterTerm(C.Structure):
    _fields_ = [("op", C.c_int32), ("pad0", C.c_int32), ("left", FilterOperand), ("right", FilterOperand)]


class JoinFilter(C.Structure):
    _fields_ = [("n_terms", C.c_int32), ("pad0", C.c_int32), ("terms", FilterTerm * MAX_FILTER_TERMS)]


def join_filter(terms) -> JoinFilter:
    """A residual join filter (krv_join_filter): `terms` is a list of
    (left, op, right), op one of = != < <= > >=, each operand ("probe", col),
    ("build", col), an int (int64 constant) or a float (float64 constant).
    Every term must be TRUE for a pair to match."""
    f = JoinFilter()
    f.n_terms = len(terms)

    def operand(o):
        if isinstance(o, tuple):
            return FilterOperand(kind=OPERAND_PROBE if o[0] == "probe" else OPERAND_BUILD, column=o[1])
        if isinstance(o, float):
            return FilterOperand(kind=OPERAND_CONST_F64, f64=o)
        return FilterOperand(kind=OPERAND_CONST_I64, i64=int(o))
    for i, (l, op, r) in enumerate(terms):
        f.terms[i] = FilterTerm(op=CMP[op], left=operand(l), right=operand(r))
    return f


class JoinCounters(C.Structure):
    _fields_ = [(n, C.c_int64) for n in ("build_rows", "build_keys", "table_slots", "probe_rows",
                                         "output_rows", "max_chain", "partitions")]


class AggExpr(C.Structure):
    _fields_ = [("function", C.c_int32), ("column", C.c_int32), ("input", C.c_int32), ("column2", C.c_int32),
                ("arg_precision", C.c_int32), ("arg_scale", C.c_int32), ("arg_bits", C.c_int32),
                ("reserved", C.c_int32)]


class AggSpec(C.Structure):
    _fields_ = [("n_group_by", C.c_int32), ("group_by", C.c_int32 * MAX_GROUP_KEYS), ("n_aggregates", C.c_int32),
                ("aggregates", AggExpr * MAX_AGGS), ("ansi", C.c_int32), ("mode", C.c_int32),
                ("expected_groups", C.c_int64), ("max_output_rows", C.c_int64), ("output", C.c_int32),
                ("reserved", C.c_int32)]


class KeyFilterOptions(C.Structure):
    _fields_ = [("max_values", C.c_int64), ("exact_max_values", C.c_int64), ("bloom", C.c_int32),
                ("pad0", C.c_int32), ("bloom_max_items", C.c_int64), ("bloom_max_bytes", C.c_int64),
                ("bloom_fpp", C.c_double), ("bloom_max_fpp", C.c_double), ("bloom_bytes", C.c_int64)]


class KeyFilterInfo(C.Structure):
    _fields_ = [("form", C.c_int32), ("nulls_pass", C.c_int32), ("has_range", C.c_int32), ("pad0", C.c_int32),
                ("lo", C.c_int64), ("hi", C.c_int64), ("keys", C.c_int64), ("distinct", C.c_int64),
                ("bloom_bytes", C.c_int64)]


class ParquetColumn(C.Structure):
    _fields_ = [("physical_type", C.c_int32), ("codec", C.c_int32), ("max_def_level", C.c_int32), ("pad0", C.c_int32),
                ("num_values", C.c_int64), ("format", C.c_char_p), ("name", C.c_char_p)]


class ParquetInfo(C.Structure):
    _fields_ = [("rows", C.c_int64), ("pages", C.c_int64), ("dictionary_entries", C.c_int64),
                ("dictionary_passing", C.c_int64), ("passing_rows", C.c_int64)]


PQ_INT32, PQ_INT64, PQ_DOUBLE, PQ_BYTE_ARRAY = 1, 2, 5, 6
PQ_UNCOMPRESSED, PQ_SNAPPY = 0, 1


class StarSpec(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("dim_key", "dim_pred", "dim_attr", "pred_a", "pred_b", "fact_fk_a",
                                         "fact_fk_b", "fact_price", "fact_discount", "group_by", "use_filters",
                                         "mode")]


class StarChain(C.Structure):
    _fields_ = [("n_fact_columns", C.c_int32), ("group_col", C.c_int32), ("price_col", C.c_int32),
                ("discount_col", C.c_int32), ("mode", C.c_int32)]


class StarCounters(C.Structure):
    _fields_ = [("fact_rows", C.c_int64), ("passed_filters", C.c_int64), ("joined_rows", C.c_int64),
                ("dim_a_keys", C.c_int64), ("dim_b_keys", C.c_int64), ("filter_a_form", C.c_int32),
                ("filter_b_form", C.c_int32), ("filter_a_bytes", C.c_int64), ("filter_b_bytes", C.c_int64),
                ("fk_a_sectors", C.c_int64)]


class GraceOptions(C.Structure):
    _fields_ = [("device_budget_bytes", C.c_int64), ("probe_filter_bits", C.c_int32), ("pad0", C.c_int32),
                ("reserved", C.c_int64 * 2)]


class ServerOptions(C.Structure):
    _fields_ = [("mode", C.c_int32), ("autotune", C.c_int32), ("ansi", C.c_int32), ("max_tick_requests", C.c_int32),
                ("tick_rows", C.c_int64), ("hbm_budget_bytes", C.c_int64)]


class ServerStats(C.Structure):
    _fields_ = [("ticks", C.c_int64), ("requests_done", C.c_int64), ("rows_probed", C.c_int64),
                ("pending", C.c_int64), ("running", C.c_int64), ("budget_in_use", C.c_int64), ("tuned", C.c_int32),
                ("threads", C.c_int32), ("item_rows", C.c_int64), ("smem_groups", C.c_int32), ("pad0", C.c_int32)]


class GenSpec(C.Structure):
    _fields_ = [("kind", C.c_int32), ("column", C.c_uint32), ("seed", C.c_uint64), ("lo", C.c_int64),
                ("hi", C.c_int64), ("x0", C.c_double), ("x1", C.c_double), ("null_fraction", C.c_double),
                ("row0", C.c_int64)]


# ---- library ------------------------------------------------------------------------------
_lib = None

# name -> (restype, argtypes)
_SIGS = {
    "krv_last_error": (C.c_char_p, []),
    "krv_last_need_bytes": (C.c_int64, []),
    "krv_version": (C.c_char_p, []),
    "krv_runtime_create": (C.c_int32, [C.c_int32, C.c_int64, C.c_void_p, C.POINTER(C.c_void_p)]),
    "krv_runtime_destroy": (None, [C.c_void_p]),
    "krv_runtime_synchronize": (C.c_int32, [C.c_void_p]),
    "krv_runtime_used_bytes": (C.c_int64, [C.c_void_p]),
    "krv_runtime_budget_bytes": (C.c_int64, [C.c_void_p]),
    "krv_runtime_stream": (C.c_void_p, [C.c_void_p]),
    "krv_runtime_launches": (C.c_int64, [C.c_void_p]),
    "krv_join_spec_init": (None, [C.POINTER(JoinSpec)]),
    "krv_join_create": (C.c_int32, [C.c_void_p, C.POINTER(JoinSpec), C.POINTER(C.c_void_p)]),
    "krv_join_build_push": (C.c_int32, [C.c_void_p, C.POINTER(ArrowArray), C.POINTER(ArrowSchema)]),
    "krv_join_build_push_device": (C.c_int32, [C.c_void_p, C.POINTER(ArrowDeviceArray), C.POINTER(ArrowSchema)]),
    "krv_join_build_finish": (C.c_int32, [C.c_void_p]),
    "krv_join_probe": (C.c_int32, [C.c_void_p, C.POINTER(ArrowArray), C.POINTER(ArrowSchema),
                                   C.POINTER(ArrowArray), C.POINTER(ArrowSchema)]),
    "krv_join_probe_device": (C.c_int32, [C.c_void_p, C.POINTER(ArrowDeviceArray), C.POINTER(ArrowSchema),
                                          C.POINTER(ArrowDeviceArray), C.POINTER(ArrowSchema)]),
    "krv_join_finish": (C.c_int32, [C.c_void_p, C.POINTER(ArrowArray), C.POINTER(ArrowSchema)]),
    "krv_join_finish_device": (C.c_int32, [C.c_void_p, C.POINTER(ArrowDeviceArray), C.POINTER(ArrowSchema)]),
    "krv_join_key_filter": (C.c_int32, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "krv_join_counters_get": (C.c_int32, [C.c_void_p, C.POINTER(JoinCounters)]),
    "krv_join_set_filter": (C.c_int32, [C.c_void_p, C.POINTER(JoinFilter)]),
    "krv_hash_rows_device": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32,
                                         C.c_uint64, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "krv_join_destroy": (None, [C.c_void_p]),
    "krv_agg_spec_init": (None, [C.POINTER(AggSpec)]),
    "krv_agg_create": (C.c_int32, [C.c_void_p, C.POINTER(AggSpec), C.POINTER(C.c_void_p)]),
    "krv_agg_push": (C.c_int32, [C.c_void_p, C.POINTER(ArrowArray), C.POINTER(ArrowSchema)]),
    "krv_agg_push_device": (C.c_int32, [C.c_void_p, C.POINTER(ArrowDeviceArray), C.POINTER(ArrowSchema)]),
    "krv_agg_finish": (C.c_int32, [C.c_void_p]),
    "krv_agg_next_output": (C.c_int32, [C.c_void_p, C.POINTER(ArrowArray), C.POINTER(ArrowSchema)]),
    "krv_agg_next_output_device": (C.c_int32, [C.c_void_p, C.POINTER(ArrowDeviceArray), C.POINTER(ArrowSchema)]),
    "krv_agg_groups": (C.c_int64, [C.c_void_p]),
    "krv_agg_destroy": (None, [C.c_void_p]),
    "krv_key_filter_options_default": (None, [C.POINTER(KeyFilterOptions)]),
    "krv_key_filter_build": (C.c_int32, [C.c_void_p, C.POINTER(KeyFilterOptions), C.POINTER(ArrowArray),
                                         C.POINTER(ArrowSchema), C.c_int32, C.POINTER(C.c_void_p)]),
    "krv_key_filter_build_device": (C.c_int32, [C.c_void_p, C.POINTER(KeyFilterOptions),
                                                C.POINTER(ArrowDeviceArray), C.POINTER(ArrowSchema), C.c_int32,
                                                C.POINTER(C.c_void_p)]),
    "krv_key_filter_evaluate": (C.c_int32, [C.c_void_p, C.POINTER(ArrowArray), C.POINTER(ArrowSchema), C.c_int32,
                                            C.POINTER(ArrowArray), C.POINTER(ArrowSchema)]),
    "krv_key_filter_evaluate_device": (C.c_int32, [C.c_void_p, C.POINTER(ArrowDeviceArray), C.POINTER(ArrowSchema),
                                                   C.c_int32, C.POINTER(ArrowDeviceArray), C.POINTER(ArrowSchema)]),
    "krv_key_filter_info_get": (C.c_int32, [C.c_void_p, C.POINTER(KeyFilterInfo)]),
    "krv_key_filter_bloom_bytes": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_int64]),
    "krv_key_filter_destroy": (None, [C.c_void_p]),
    "krv_star_spec_init": (None, [C.POINTER(StarSpec)]),
    "krv_star_create": (C.c_int32, [C.c_void_p, C.POINTER(StarSpec), C.POINTER(C.c_void_p)]),
    "krv_star_from_joins": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(StarChain),
                                        C.POINTER(C.c_void_p)]),
    "krv_star_build": (C.c_int32, [C.c_void_p, C.POINTER(ArrowArray), C.POINTER(ArrowSchema),
                                   C.POINTER(ArrowArray), C.POINTER(ArrowSchema)]),
    "krv_star_build_device": (C.c_int32, [C.c_void_p, C.POINTER(ArrowDeviceArray), C.POINTER(ArrowSchema),
                                          C.POINTER(ArrowDeviceArray), C.POINTER(ArrowSchema)]),
    "krv_star_probe": (C.c_int32, [C.c_void_p, C.POINTER(ArrowArray), C.POINTER(ArrowSchema)]),
    "krv_star_probe_device": (C.c_int32, [C.c_void_p, C.POINTER(ArrowDeviceArray), C.POINTER(ArrowSchema)]),
    "krv_star_result": (C.c_int32, [C.c_void_p, C.POINTER(ArrowArray), C.POINTER(ArrowSchema)]),
    "krv_star_reset": (C.c_int32, [C.c_void_p]),
    "krv_star_counters_get": (C.c_int32, [C.c_void_p, C.POINTER(StarCounters)]),
    "krv_star_destroy": (None, [C.c_void_p]),
    "krv_gen_fill": (C.c_int32, [C.c_void_p, C.POINTER(GenSpec), C.c_int64, C.c_void_p, C.c_void_p]),
    "krv_grace_options_init": (None, [C.POINTER(GraceOptions)]),
    "krv_join_create_partitioned": (C.c_int32, [C.c_void_p, C.POINTER(JoinSpec), C.POINTER(GraceOptions),
                                                C.POINTER(C.c_void_p)]),
    "krv_join_spilled_partitions": (C.c_int64, [C.c_void_p]),
    "krv_join_filtered_probe_rows": (C.c_int64, [C.c_void_p]),
    "krv_parquet_decode_chunk": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_int64, C.POINTER(ParquetColumn), C.c_void_p,
                                             C.POINTER(ArrowDeviceArray), C.POINTER(ArrowSchema),
                                             C.POINTER(ParquetInfo)]),
    "krv_server_options_init": (None, [C.POINTER(ServerOptions)]),
    "krv_server_create": (C.c_int32, [C.c_void_p, C.POINTER(ServerOptions), C.POINTER(C.c_void_p)]),
    "krv_server_add_table": (C.c_int32, [C.c_void_p, C.POINTER(ArrowDeviceArray), C.POINTER(ArrowSchema), C.c_int32,
                                         C.c_int32, C.POINTER(C.c_int64)]),
    "krv_server_drop_table": (C.c_int32, [C.c_void_p, C.c_int64]),
    "krv_server_submit": (C.c_int32, [C.c_void_p, C.c_int64, C.POINTER(ArrowDeviceArray), C.POINTER(ArrowSchema),
                                      C.c_int32, C.c_int32, C.POINTER(C.c_int64)]),
    "krv_server_step": (C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(C.c_int64)]),
    "krv_server_poll": (C.c_int32, [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int32),
                                    C.POINTER(ArrowDeviceArray), C.POINTER(ArrowSchema)]),
    "krv_server_stats_get": (C.c_int32, [C.c_void_p, C.POINTER(ServerStats)]),
    "krv_server_destroy": (None, [C.c_void_p]),
    "krv_agg_sum_i64_scratch": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_int64, C.c_int64, C.c_void_p, C.c_void_p,
                                            C.c_void_p, C.c_void_p, C.c_void_p]),
}


def exported_names() -> List[str]:
    return sorted(_SIGS)


def lib():
    """Loads libkrv_gpu.so (built by build.py). Fails loudly when missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run python krishiv-engine_b200/build.py")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def build(jobs: int = 8) -> str:
    """Compiles the CUDA library in-tree (nvcc, sm_100a)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("_krv_build", os.path.join(HERE, "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.build(jobs)


def check(status: int) -> int:
    """Raises KrvError for a negative status (with the library's error text)."""
    if status >= 0:
        return status
    msg = lib().krv_last_error().decode("utf-8", "replace")
    raise KrvError(status, msg)


# ---- Arrow helpers ----------------------------------------------------------------------
def _release_array(arr: ArrowArray):
    if arr.release:
        arr.release(C.byref(arr))


def _release_schema(s: ArrowSchema):
    if s.release:
        s.release(C.byref(s))


class HostBatch:
    """A pyarrow RecordBatch exported through the C Data Interface for one
    borrowed call; released when the call is done (a context manager)."""

    def __init__(self, batch):
        self.array = ArrowArray()
        self.schema = ArrowSchema()
        batch._export_to_c(C.addressof(self.array), C.addressof(self.schema))

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        _release_array(self.array)
        _release_schema(self.schema)


def import_host(arr: ArrowArray, schema: ArrowSchema):
    import pyarrow as pa
    return pa.RecordBatch._import_from_c(C.addressof(arr), C.addressof(schema))


_NOOP_ARRAY_RELEASE = C.CFUNCTYPE(None, C.POINTER(ArrowArray))(lambda p: None)

_TORCH_FORMAT = {}


def _format_of(t) -> str:
    import torch
    return {torch.int64: "l", torch.int32: "i", torch.float64: "g", torch.uint8: "C"}[t.dtype]


class DeviceBatch:
    """Device columns (torch CUDA tensors) as an ArrowDeviceArray, borrowed
    by the library for the duration of one call.

    `columns`: list of (name, tensor, valid_tensor_or_None, arrow_type_or_None).
    A validity tensor is a uint8 bitmap (bit i = row i). The Arrow type
    defaults from the tensor dtype; pass e.g. pa.decimal64(15, 2) for an
    int64 tensor of unscaled decimals."""

    def __init__(self, columns: Sequence, device: int = 0):
        import pyarrow as pa
        self._keep = []
        n = int(columns[0][1].shape[0]) if columns else 0
        fields = []
        self.children = (C.POINTER(ArrowArray) * max(1, len(columns)))()
        self._child_structs = []
        for i, col in enumerate(columns):
            name, t, valid = col[0], col[1], col[2] if len(col) > 2 else None
            atype = col[3] if len(col) > 3 and col[3] is not None else None
            if atype is None:
                atype = {"l": pa.int64(), "i": pa.int32(), "g": pa.float64(), "C": pa.uint8()}[_format_of(t)]
            fields.append(pa.field(name, atype, nullable=valid is not None))
            bufs = (C.c_void_p * 2)(valid.data_ptr() if valid is not None else None, t.data_ptr())
            a = ArrowArray(length=n, null_count=-1 if valid is not None else 0, offset=0, n_buffers=2,
                           n_children=0, buffers=bufs, children=None, dictionary=None,
                           release=_NOOP_ARRAY_RELEASE, private_data=None)
            self._keep += [t, valid, bufs, a]
            self._child_structs.append(a)
            self.children[i] = C.pointer(a)
        top_bufs = (C.c_void_p * 1)(None)
        self._keep.append(top_bufs)
        self.rows = n
        self.dev = ArrowDeviceArray()
        self.dev.array = ArrowArray(length=n, null_count=0, offset=0, n_buffers=1, n_children=len(columns),
                                    buffers=top_bufs, children=self.children, dictionary=None,
                                    release=_NOOP_ARRAY_RELEASE, private_data=None)
        self.dev.device_id = device
        self.dev.device_type = ARROW_DEVICE_CUDA
        self.dev.sync_event = None
        self.pa_schema = pa.schema(fields)
        self.schema = ArrowSchema()
        self.pa_schema._export_to_c(C.addressof(self.schema))

    def __del__(self):
        try:
            _release_schema(self.schema)
        except Exception:
            pass


class _CudaArray:
    def __init__(self, ptr: int, n: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr, False), "version": 3,
                                         "strides": None}


class DeviceResult:
    """A library-owned ArrowDeviceArray moved to Python. Columns are exposed as
    torch tensors that share its device memory; the memory is released when
    this object goes away."""

    _TYPESTR = {"l": "<i8", "i": "<i4", "g": "<f8", "C": "|u1", "tdD": "<i4"}

    def __init__(self, dev: ArrowDeviceArray, schema: ArrowSchema):
        import torch
        self.dev = dev
        self.schema = schema
        self.rows = dev.array.length
        self.names, self.formats, self.columns, self.valid = [], [], [], []
        self.heaps = []  # UTF-8 / binary columns: their bytes (columns[i] holds the int32 offsets)
        for i in range(dev.array.n_children):
            cs = schema.children[i].contents
            fmt = cs.format.decode()
            self.names.append(cs.name.decode() if cs.name else "")
            self.formats.append(fmt)
            ch = dev.array.children[i].contents
            data = ch.buffers[1]
            vptr = ch.buffers[0]
            heap = None
            if fmt in ("u", "z"):
                ts, n = "<i4", self.rows + 1
                offs = torch.as_tensor(_CudaArray(data, n, ts), device="cuda") if data else None
                nbytes = int(offs[-1].item()) if offs is not None else 0
                if nbytes and ch.buffers[2]:
                    heap = torch.as_tensor(_CudaArray(ch.buffers[2], nbytes, "|u1"), device="cuda")
            elif fmt.startswith("d:"):
                width = 8 if fmt.endswith(",64") else 16
                ts, n = "<i8", self.rows * (width // 8)
            elif fmt == "b":
                ts, n = "|u1", (self.rows + 7) // 8
            else:
                ts, n = self._TYPESTR[fmt], self.rows
            self.columns.append(torch.as_tensor(_CudaArray(data, n, ts), device="cuda") if n and data else None)
            self.heaps.append(heap)
            self.valid.append(torch.as_tensor(_CudaArray(vptr, (self.rows + 7) // 8, "|u1"), device="cuda")
                              if vptr and self.rows else None)

    def __del__(self):
        try:
            _release_array(self.dev.array)
            _release_schema(self.schema)
        except Exception:
            pass


# ---- operators ------------------------------------------------------------------------------
class Runtime:
    """A device, a CUDA stream and an HBM budget (krv_runtime_create)."""

    def __init__(self, device: int = 0, budget_bytes: int = 0, stream: Optional[int] = None):
        h = C.c_void_p()
        check(lib().krv_runtime_create(device, budget_bytes, stream, C.byref(h)))
        self.h = h
        self.device = device

    @classmethod
    def on_torch_stream(cls, device: int = 0, budget_bytes: int = 0, stream=None) -> "Runtime":
        """A runtime on a torch CUDA stream that is made current, so torch
        tensors, events and the library's kernels are ordered on one stream.
        (The legacy default stream has the handle 0, which the C ABI reads as
        "create a stream", hence a dedicated stream.)"""
        import torch
        torch.cuda.set_device(device)
        s = stream if stream is not None else torch.cuda.Stream(device=device)
        torch.cuda.set_stream(s)
        r = cls(device, budget_bytes, s.cuda_stream)
        r.torch_stream = s
        return r

    def synchronize(self):
        check(lib().krv_runtime_synchronize(self.h))

    @property
    def used_bytes(self) -> int:
        return lib().krv_runtime_used_bytes(self.h)

    @property
    def launches(self) -> int:
        return lib().krv_runtime_launches(self.h)

    @property
    def stream(self) -> int:
        return lib().krv_runtime_stream(self.h)

    def close(self):
        if getattr(self, "h", None):
            lib().krv_runtime_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def hash_rows(rt: "Runtime", db: "DeviceBatch", key_columns=(0,), null_safe=None, seed: int = 0, depth: int = 0,
              radix: int = 4):
    """The join's key hash of every row of a DeviceBatch (krv_hash_rows_device):
    (h, g, partition) as CUDA tensors (uint64 values in int64 tensors, int32
    partition ids)."""
    import torch
    n = db.rows
    dev = f"cuda:{rt.device}"
    h = torch.empty(n, dtype=torch.int64, device=dev)
    g = torch.empty(n, dtype=torch.int64, device=dev)
    p = torch.empty(n, dtype=torch.int32, device=dev)
    cols = (C.c_int32 * len(key_columns))(*key_columns)
    ns = (C.c_int32 * len(key_columns))(*(null_safe or [0] * len(key_columns)))
    check(lib().krv_hash_rows_device(rt.h, C.byref(db.dev), C.byref(db.schema), cols, ns, len(key_columns),
                                     seed & 0xFFFFFFFFFFFFFFFF, depth, radix, h.data_ptr() if n else None,
                                     g.data_ptr() if n else None, p.data_ptr() if n else None))
    return h, g, p


def join_spec(join_type="inner", probe_keys=(0,), build_keys=(0,), null_safe=None, single_match=False,
              probe_out=None, build_out=None, runtime_filter=False, max_load=0.0, max_output_rows=0,
              build_rows_hint=0, radix_bits=0) -> JoinSpec:
    s = JoinSpec()
    lib().krv_join_spec_init(C.byref(s))
    s.join_type = JOIN_TYPES[join_type] if isinstance(join_type, str) else int(join_type)
    s.n_keys = len(probe_keys)
    for i, (p, b) in enumerate(zip(probe_keys, build_keys)):
        s.probe_keys[i] = p
        s.build_keys[i] = b
        s.null_safe[i] = int(bool(null_safe[i])) if null_safe else 0
    s.single_match = int(single_match)
    if probe_out is not None:
        s.n_probe_out = len(probe_out)
        for i, c in enumerate(probe_out):
            s.probe_out[i] = c
    if build_out is not None:
        s.n_build_out = len(build_out)
        for i, c in enumerate(build_out):
            s.build_out[i] = c
    s.runtime_filter = int(runtime_filter)
    s.max_load = max_load
    s.max_output_rows = max_output_rows
    s.build_rows_hint = build_rows_hint
    s.radix_bits = radix_bits
    return s


class HashJoin:
    """The hash join operator (HashJoin, crates/krishiv-exec/src/join/mod.rs:1014).
    `partitioned=True` makes the partitioned (grace) join of
    crates/krishiv-exec/src/join/grace.rs (krv_join_create_partitioned): inner
    or left outer on one int64 key, within `device_budget` bytes (0: the
    runtime's budget), spilling partitions to page-locked host memory;
    `probe_filter_bits` (partitioned only) sets the bits per build key of the
    Bloom filter its partition passes build and test (None: the default, 10;
    0: no filter)."""

    def __init__(self, rt: Runtime, spec: JoinSpec, partitioned: bool = False, device_budget: int = 0,
                 filter=None, probe_filter_bits=None):
        self.rt = rt
        h = C.c_void_p()
        if partitioned:
            o = GraceOptions()
            lib().krv_grace_options_init(C.byref(o))
            o.device_budget_bytes = device_budget
            if probe_filter_bits is not None:
                o.probe_filter_bits = int(probe_filter_bits)
            check(lib().krv_join_create_partitioned(rt.h, C.byref(spec), C.byref(o), C.byref(h)))
        else:
            check(lib().krv_join_create(rt.h, C.byref(spec), C.byref(h)))
        self.h = h
        if filter is not None:
            # a residual filter (join_filter(...) or its list of terms)
            f = filter if isinstance(filter, JoinFilter) else join_filter(filter)
            check(lib().krv_join_set_filter(self.h, C.byref(f)))

    def build_push(self, batch):
        with HostBatch(batch) as hb:
            check(lib().krv_join_build_push(self.h, C.byref(hb.array), C.byref(hb.schema)))

    def build_push_device(self, db: DeviceBatch):
        check(lib().krv_join_build_push_device(self.h, C.byref(db.dev), C.byref(db.schema)))

    def build_finish(self):
        check(lib().krv_join_build_finish(self.h))

    def probe(self, batch) -> list:
        """All output batches (pyarrow) of one probe batch."""
        out = []
        with HostBatch(batch) as hb:
            arr, sch = ArrowArray(), ArrowSchema()
            st = check(lib().krv_join_probe(self.h, C.byref(hb.array), C.byref(hb.schema), C.byref(arr),
                                            C.byref(sch)))
            out.append(import_host(arr, sch))
        while st == HAVE_MORE_OUTPUT:
            arr, sch = ArrowArray(), ArrowSchema()
            st = check(lib().krv_join_probe(self.h, None, None, C.byref(arr), C.byref(sch)))
            out.append(import_host(arr, sch))
        return out

    def probe_device(self, db: DeviceBatch) -> DeviceResult:
        dev, sch = ArrowDeviceArray(), ArrowSchema()
        check(lib().krv_join_probe_device(self.h, C.byref(db.dev), C.byref(db.schema), C.byref(dev), C.byref(sch)))
        return DeviceResult(dev, sch)

    def probe_device_all(self, db: DeviceBatch):
        """Every output batch of one probe batch (device), one at a time."""
        dev, sch = ArrowDeviceArray(), ArrowSchema()
        st = check(lib().krv_join_probe_device(self.h, C.byref(db.dev), C.byref(db.schema), C.byref(dev),
                                               C.byref(sch)))
        yield DeviceResult(dev, sch)
        while st == HAVE_MORE_OUTPUT:
            dev, sch = ArrowDeviceArray(), ArrowSchema()
            st = check(lib().krv_join_probe_device(self.h, None, None, C.byref(dev), C.byref(sch)))
            yield DeviceResult(dev, sch)

    def finish_device(self):
        """The rows emitted after the last probe batch (device), one batch at a
        time: a partitioned join's spilled partitions."""
        st = HAVE_MORE_OUTPUT
        while st == HAVE_MORE_OUTPUT:
            dev, sch = ArrowDeviceArray(), ArrowSchema()
            st = check(lib().krv_join_finish_device(self.h, C.byref(dev), C.byref(sch)))
            yield DeviceResult(dev, sch)

    def spilled_partitions(self) -> int:
        return lib().krv_join_spilled_partitions(self.h)

    def filtered_probe_rows(self) -> int:
        """Probe rows the partitioned join's Bloom filter ruled out."""
        return lib().krv_join_filtered_probe_rows(self.h)

    def finish(self) -> list:
        out = []
        st = HAVE_MORE_OUTPUT
        while st == HAVE_MORE_OUTPUT:
            arr, sch = ArrowArray(), ArrowSchema()
            st = check(lib().krv_join_finish(self.h, C.byref(arr), C.byref(sch)))
            out.append(import_host(arr, sch))
        return out

    def key_filter(self) -> "KeyFilter":
        h = C.c_void_p()
        check(lib().krv_join_key_filter(self.h, C.byref(h)))
        return KeyFilter(self.rt, h)

    def counters(self) -> Dict[str, int]:
        c = JoinCounters()
        check(lib().krv_join_counters_get(self.h, C.byref(c)))
        return {n: getattr(c, n) for n, _ in JoinCounters._fields_}

    def close(self):
        if getattr(self, "h", None):
            lib().krv_join_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def agg_spec(group_by, aggregates: Sequence, ansi=True, mode=MODE_AUTO, expected_groups=0,
             max_output_rows=0, partial=False) -> AggSpec:
    """`group_by`: one column index or a sequence of up to MAX_GROUP_KEYS.
    `aggregates`: (function, column) over raw input, or (function, "state",
    column[, column2[, (arg_precision, arg_scale, arg_bits)]]) over the state
    columns of a partial aggregate. `partial`: emit each aggregate's state
    columns."""
    s = AggSpec()
    lib().krv_agg_spec_init(C.byref(s))
    keys = [group_by] if isinstance(group_by, int) else list(group_by)
    s.n_group_by = len(keys)
    for i, k in enumerate(keys):
        s.group_by[i] = k
    s.n_aggregates = len(aggregates)
    for i, a in enumerate(aggregates):
        f = a[0]
        s.aggregates[i].function = AGG_FUNCS[f] if isinstance(f, str) else int(f)
        if len(a) > 2 and a[1] == "state":
            s.aggregates[i].input = AGG_INPUT_STATE
            s.aggregates[i].column = a[2]
            s.aggregates[i].column2 = a[3] if len(a) > 3 and a[3] is not None else -1
            if len(a) > 4:
                s.aggregates[i].arg_precision, s.aggregates[i].arg_scale, s.aggregates[i].arg_bits = a[4]
        else:
            s.aggregates[i].column = a[1]
    s.output = AGG_OUTPUT_PARTIAL if partial else AGG_OUTPUT_FINAL
    s.ansi = int(ansi)
    s.mode = mode
    s.expected_groups = expected_groups
    s.max_output_rows = max_output_rows
    return s


def merging(aggregates: Sequence, first: int, arg_types: Sequence) -> list:
    """The second-phase aggregates over the state columns that a partial
    aggregate (agg_spec(..., partial=True)) writes for `aggregates`, those
    columns starting at column `first` (after the group keys), in the
    reference's order (AggregateExpr::merging, aggregate/mod.rs:561-569, over
    AggregateExpr::state_fields, :747-800): COUNT one column, SUM one (two
    for a decimal argument: sum, nonempty), AVG two (sum, count), MIN/MAX
    one. `arg_types` gives each aggregate's raw argument type (pyarrow;
    None for COUNT(*)): decimals decide SUM's state and AVG's result type."""
    import pyarrow as pa
    out, at = [], first
    for a, t in zip(aggregates, arg_types):
        f = a[0]
        dec = t is not None and pa.types.is_decimal(t)
        if f in ("count", "count_star", "min", "max"):
            out.append((f, "state", at))
            at += 1
        elif f == "sum":
            out.append((f, "state", at, at + 1) if dec else (f, "state", at))
            at += 2 if dec else 1
        elif f == "avg":
            raw = (t.precision, t.scale, t.bit_width) if dec else None
            out.append((f, "state", at, at + 1, raw) if raw else (f, "state", at, at + 1))
            at += 2
        else:
            raise ValueError("unknown aggregate function %r" % (f,))
    return out


class HashAggregate:
    """The grouped hash aggregate (HashAggregate, crates/krishiv-exec/src/aggregate/sink.rs:181)."""

    def __init__(self, rt: Runtime, spec: AggSpec):
        self.rt = rt
        h = C.c_void_p()
        check(lib().krv_agg_create(rt.h, C.byref(spec), C.byref(h)))
        self.h = h

    def push(self, batch):
        with HostBatch(batch) as hb:
            check(lib().krv_agg_push(self.h, C.byref(hb.array), C.byref(hb.schema)))

    def push_device(self, db: DeviceBatch):
        check(lib().krv_agg_push_device(self.h, C.byref(db.dev), C.byref(db.schema)))

    def finish(self):
        check(lib().krv_agg_finish(self.h))

    def result(self) -> list:
        out = []
        st = HAVE_MORE_OUTPUT
        while st == HAVE_MORE_OUTPUT:
            arr, sch = ArrowArray(), ArrowSchema()
            st = check(lib().krv_agg_next_output(self.h, C.byref(arr), C.byref(sch)))
            out.append(import_host(arr, sch))
        return out

    def result_device(self) -> DeviceResult:
        dev, sch = ArrowDeviceArray(), ArrowSchema()
        check(lib().krv_agg_next_output_device(self.h, C.byref(dev), C.byref(sch)))
        return DeviceResult(dev, sch)

    @property
    def groups(self) -> int:
        return lib().krv_agg_groups(self.h)

    def close(self):
        if getattr(self, "h", None):
            lib().krv_agg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def key_filter_options(**kw) -> KeyFilterOptions:
    o = KeyFilterOptions()
    lib().krv_key_filter_options_default(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


class KeyFilter:
    """A runtime key filter (KeyFilter, crates/krishiv-io/src/runtime_filter/filter.rs:627)."""

    def __init__(self, rt: Runtime, h):
        self.rt = rt
        self.h = h

    @classmethod
    def build(cls, rt: Runtime, batch, column: int, options: Optional[KeyFilterOptions] = None):
        h = C.c_void_p()
        with HostBatch(batch) as hb:
            check(lib().krv_key_filter_build(rt.h, C.byref(options) if options else None, C.byref(hb.array),
                                             C.byref(hb.schema), column, C.byref(h)))
        return cls(rt, h)

    @classmethod
    def build_device(cls, rt: Runtime, db: DeviceBatch, column: int, options: Optional[KeyFilterOptions] = None):
        h = C.c_void_p()
        check(lib().krv_key_filter_build_device(rt.h, C.byref(options) if options else None, C.byref(db.dev),
                                                C.byref(db.schema), column, C.byref(h)))
        return cls(rt, h)

    def evaluate(self, batch, column: int):
        with HostBatch(batch) as hb:
            arr, sch = ArrowArray(), ArrowSchema()
            check(lib().krv_key_filter_evaluate(self.h, C.byref(hb.array), C.byref(hb.schema), column,
                                                C.byref(arr), C.byref(sch)))
            return import_host(arr, sch).column(0)

    def evaluate_device(self, db: DeviceBatch, column: int) -> DeviceResult:
        dev, sch = ArrowDeviceArray(), ArrowSchema()
        check(lib().krv_key_filter_evaluate_device(self.h, C.byref(db.dev), C.byref(db.schema), column,
                                                   C.byref(dev), C.byref(sch)))
        return DeviceResult(dev, sch)

    def info(self) -> Dict[str, int]:
        i = KeyFilterInfo()
        check(lib().krv_key_filter_info_get(self.h, C.byref(i)))
        return {n: getattr(i, n) for n, _ in KeyFilterInfo._fields_ if n != "pad0"}

    def bloom_bytes(self) -> bytes:
        n = self.info()["bloom_bytes"]
        buf = C.create_string_buffer(n)
        check(lib().krv_key_filter_bloom_bytes(self.h, buf, n))
        return buf.raw

    def close(self):
        if getattr(self, "h", None):
            lib().krv_key_filter_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def parquet_decode_chunk(rt: Runtime, chunk, physical_type: int, codec: int, max_def_level: int, num_values: int,
                         fmt: str, name: str = "", key_filter: Optional[KeyFilter] = None):
    """One Parquet column chunk (its bytes as the file stores them: bytes, or
    a uint8 numpy array) decoded on the device (krv_parquet_decode_chunk):
    a DeviceResult of the column and, with `key_filter`, the filter's
    boolean "pass" column, and the decode's counts."""
    import numpy as np
    buf = np.frombuffer(chunk, dtype=np.uint8) if isinstance(chunk, (bytes, bytearray, memoryview)) else chunk
    buf = np.ascontiguousarray(buf, dtype=np.uint8)
    col = ParquetColumn(physical_type=physical_type, codec=codec, max_def_level=max_def_level, num_values=num_values,
                        format=fmt.encode(), name=name.encode())
    dev, sch, info = ArrowDeviceArray(), ArrowSchema(), ParquetInfo()
    check(lib().krv_parquet_decode_chunk(rt.h, buf.ctypes.data_as(C.c_void_p), buf.size, C.byref(col),
                                         key_filter.h if key_filter is not None else None, C.byref(dev),
                                         C.byref(sch), C.byref(info)))
    return DeviceResult(dev, sch), {n: getattr(info, n) for n, _ in ParquetInfo._fields_}


def star_spec(pred_a: int, pred_b: int, group_by: int = 0, use_filters: bool = True, mode: int = STAR_FUSED):
    s = StarSpec()
    lib().krv_star_spec_init(C.byref(s))
    s.pred_a, s.pred_b, s.group_by, s.use_filters, s.mode = pred_a, pred_b, group_by, int(use_filters), mode
    return s


class StarPipeline:
    """Star join with runtime filters and a grouped sum (krv_star_*)."""

    def __init__(self, rt: Runtime, spec: StarSpec = None, _handle=None):
        self.rt = rt
        if _handle is not None:
            self.h = _handle
            return
        h = C.c_void_p()
        check(lib().krv_star_create(rt.h, C.byref(spec), C.byref(h)))
        self.h = h

    @classmethod
    def from_joins(cls, rt: Runtime, join_a: "HashJoin", join_b: "HashJoin", n_fact_columns: int, group_col: int,
                   price_col: int, discount_col: int, mode: int = STAR_FUSED) -> "StarPipeline":
        """The fused plan of the operator chain fact -> join_a -> join_b ->
        SUM(price * (1 - discount)) GROUP BY group_col (columns of join_b's
        output), from the joins' finished build sides (krv_star_from_joins).
        Raises KrvError(KRV_UNSUPPORTED) when the chain is not of that shape."""
        chain = StarChain(n_fact_columns, group_col, price_col, discount_col, mode)
        h = C.c_void_p()
        check(lib().krv_star_from_joins(rt.h, join_a.h, join_b.h, C.byref(chain), C.byref(h)))
        return cls(rt, _handle=h)

    def build(self, dim_a, dim_b):
        with HostBatch(dim_a) as a, HostBatch(dim_b) as b:
            check(lib().krv_star_build(self.h, C.byref(a.array), C.byref(a.schema), C.byref(b.array),
                                       C.byref(b.schema)))

    def build_device(self, a: DeviceBatch, b: DeviceBatch):
        check(lib().krv_star_build_device(self.h, C.byref(a.dev), C.byref(a.schema), C.byref(b.dev),
                                          C.byref(b.schema)))

    def probe(self, fact):
        with HostBatch(fact) as f:
            check(lib().krv_star_probe(self.h, C.byref(f.array), C.byref(f.schema)))

    def probe_device(self, f: DeviceBatch):
        check(lib().krv_star_probe_device(self.h, C.byref(f.dev), C.byref(f.schema)))

    def result(self):
        arr, sch = ArrowArray(), ArrowSchema()
        check(lib().krv_star_result(self.h, C.byref(arr), C.byref(sch)))
        return import_host(arr, sch)

    def reset(self):
        check(lib().krv_star_reset(self.h))

    def counters(self) -> Dict[str, int]:
        c = StarCounters()
        check(lib().krv_star_counters_get(self.h, C.byref(c)))
        return {n: getattr(c, n) for n, _ in StarCounters._fields_}

    def close(self):
        if getattr(self, "h", None):
            lib().krv_star_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def gen_fill(rt: Runtime, out, kind: int, seed: int, column: int, lo: int = 0, hi: int = 0, x0: float = 0.0,
             x1: float = 0.0, null_fraction: float = 0.0, row0: int = 0, valid=None):
    """Fills the CUDA tensor `out` (and bitmap `valid`) with a counter-based
    synthetic column (krv_gen_fill)."""
    s = GenSpec(kind=kind, column=column, seed=seed, lo=lo, hi=hi, x0=x0, x1=x1, null_fraction=null_fraction,
                row0=row0)
    check(lib().krv_gen_fill(rt.h, C.byref(s), int(out.shape[0]), out.data_ptr(),
                             valid.data_ptr() if valid is not None else None))


def agg_sum_i64_scratch(keys, values, out_keys, out_sums, out_counts, out_info, stream=None):
    """GROUP BY `keys` SUM(`values`), COUNT(*) without allocating device memory
    (krv_agg_sum_i64_scratch). All arguments are int64 CUDA tensors of the
    current device; the three outputs hold max_groups = len(out_keys) values
    (at most SCRATCH_MAX_GROUPS) and out_info two: the group count (-1 when the
    keys had more distinct values than max_groups) and a wrap flag. `stream`
    is a raw cudaStream_t handle (None: the default stream). Asynchronous."""
    import torch
    named = {"keys": keys, "values": values, "out_keys": out_keys, "out_sums": out_sums,
             "out_counts": out_counts, "out_info": out_info}
    for name, t in named.items():
        if t.dtype != torch.int64:
            raise ValueError(f"{name} must be int64, not {t.dtype}")
        if not t.is_cuda:
            raise ValueError(f"{name} must be a CUDA tensor")
        if t.dim() != 1 or not t.is_contiguous():
            raise ValueError(f"{name} must be a contiguous 1-D tensor")
    devices = {t.device for t in named.values()}
    if len(devices) != 1:
        raise ValueError("all tensors must be on one device")
    n = int(keys.shape[0])
    if int(values.shape[0]) != n:
        raise ValueError("keys and values differ in length")
    g = int(out_keys.shape[0])
    if int(out_sums.shape[0]) < g or int(out_counts.shape[0]) < g:
        raise ValueError("out_sums and out_counts must hold at least len(out_keys) values")
    if int(out_info.shape[0]) < 2:
        raise ValueError("out_info must hold two values")
    check(lib().krv_agg_sum_i64_scratch(keys.data_ptr() if n else None, values.data_ptr() if n else None, n, g,
                                        out_keys.data_ptr() if g else None, out_sums.data_ptr() if g else None,
                                        out_counts.data_ptr() if g else None, out_info.data_ptr(), stream))


def server_options(**kw) -> ServerOptions:
    o = ServerOptions()
    lib().krv_server_options_init(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


class Server:
    """Join + grouped aggregate requests against resident build tables
    (krv_server_*): SELECT t.g, SUM(p.x), COUNT(*) FROM p JOIN t USING (k)
    GROUP BY t.g. Requests are DeviceBatch probes; the server keeps them (and
    so their tensors) until they are polled."""

    def __init__(self, rt: Runtime, opts: ServerOptions = None):
        self.rt = rt
        h = C.c_void_p()
        check(lib().krv_server_create(rt.h, C.byref(opts) if opts is not None else None, C.byref(h)))
        self.h = h
        self._inflight = {}

    def add_table(self, db: DeviceBatch, key_column: int = 0, group_column: int = 1) -> int:
        tid = C.c_int64()
        check(lib().krv_server_add_table(self.h, C.byref(db.dev), C.byref(db.schema), key_column, group_column,
                                         C.byref(tid)))
        return tid.value

    def drop_table(self, table_id: int):
        check(lib().krv_server_drop_table(self.h, table_id))

    def submit(self, table_id: int, db: DeviceBatch, key_column: int = 0, value_column: int = 1) -> int:
        rid = C.c_int64()
        check(lib().krv_server_submit(self.h, table_id, C.byref(db.dev), C.byref(db.schema), key_column, value_column,
                                      C.byref(rid)))
        self._inflight[rid.value] = db
        return rid.value

    def step(self, wait: bool = False) -> int:
        n = C.c_int64()
        check(lib().krv_server_step(self.h, 1 if wait else 0, C.byref(n)))
        return n.value

    def poll(self):
        """(request id, status, DeviceResult or None) of the next finished
        request, or None when none has finished."""
        rid, st = C.c_int64(), C.c_int32()
        dev, sch = ArrowDeviceArray(), ArrowSchema()
        s = check(lib().krv_server_poll(self.h, C.byref(rid), C.byref(st), C.byref(dev), C.byref(sch)))
        if s == FINISHED:
            return None
        self._inflight.pop(rid.value, None)
        return rid.value, st.value, (DeviceResult(dev, sch) if st.value == OK else None)

    def stats(self) -> Dict[str, int]:
        c = ServerStats()
        check(lib().krv_server_stats_get(self.h, C.byref(c)))
        return {n: getattr(c, n) for n, _ in ServerStats._fields_ if n != "pad0"}

    def close(self):
        if getattr(self, "h", None):
            lib().krv_server_destroy(self.h)
            self.h = None
        self._inflight = {}

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
