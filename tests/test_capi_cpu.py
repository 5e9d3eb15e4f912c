"""The C-ABI library without a GPU: it loads, exports every function that
include/krv_gpu.h declares, the Python binding covers each, and calls that
need a device fail with a status (never a crash) when none is present."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    text = open(os.path.join(ROOT, "include", "krv_gpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(krv_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_boundary():
    names = declared()
    for must in ("krv_join_create", "krv_join_build_push", "krv_join_build_finish", "krv_join_probe",
                 "krv_join_finish", "krv_agg_create", "krv_agg_push", "krv_agg_finish", "krv_agg_next_output",
                 "krv_key_filter_build", "krv_key_filter_evaluate", "krv_star_probe", "krv_last_error"):
        assert must in names


def test_library_exports_every_declared_symbol(kb):
    lib = C.CDLL(kb.LIB_PATH)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_every_symbol(kb):
    assert sorted(kb.exported_names()) == declared()
    kb.lib()  # every signature binds


def test_spec_initializers(kb):
    s = kb.join_spec("left_outer", probe_keys=(0, 1), build_keys=(2, 3), null_safe=[0, 1])
    assert s.join_type == kb.LEFT_OUTER and s.n_keys == 2 and s.build_keys[1] == 3 and s.null_safe[1] == 1
    assert s.n_probe_out == -1 and s.n_build_out == -1
    a = kb.agg_spec(0, [("sum", 1), ("count_star", 0)])
    assert a.n_aggregates == 2 and a.aggregates[0].function == kb.SUM
    o = kb.key_filter_options()
    assert (o.max_values, o.exact_max_values, o.bloom_max_items, o.bloom_max_bytes) == (50, 4096, 4000000, 8 << 20)
    assert (o.bloom_fpp, o.bloom_max_fpp) == (0.01, 0.05)


def test_no_device_is_an_error_status(kb):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    with pytest.raises(kb.KrvError) as e:
        kb.Runtime(0)
    assert e.value.status in (kb.CUDA_ERROR, kb.INVALID_ARGUMENT)
    assert kb.lib().krv_last_error()


def test_version(kb):
    assert b"sm_100a" in kb.lib().krv_version()


# Each C struct of include/krv_gpu.h and its ctypes mirror in the binding.
STRUCTS = {"krv_join_spec": "JoinSpec", "krv_join_counters": "JoinCounters", "krv_grace_options": "GraceOptions",
           "krv_agg_expr": "AggExpr", "krv_agg_spec": "AggSpec", "krv_key_filter_options": "KeyFilterOptions",
           "krv_key_filter_info": "KeyFilterInfo", "krv_star_spec": "StarSpec", "krv_star_counters": "StarCounters",
           "krv_gen_spec": "GenSpec", "krv_server_options": "ServerOptions", "krv_server_stats": "ServerStats",
           "krv_parquet_column": "ParquetColumn", "krv_parquet_info": "ParquetInfo"}


def test_header_is_c_and_structs_match_the_binding(kb, tmp_path):
    """The header compiles as C11, and every struct's size and every field's
    offset seen by a C compiler equal the Python binding's ctypes layout."""
    import shutil
    import subprocess
    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "krv_gpu.h"', "int main(void) {"]
    for cname, pyname in STRUCTS.items():
        cls = getattr(kb, pyname)
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for f in cls._fields_:
            lines.append(f'printf("{cname}.{f[0]} %zu\\n", offsetof({cname}, {f[0]}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True, capture_output=True)
    got = dict(line.split() for line in subprocess.run([str(exe)], check=True, capture_output=True,
                                                           text=True).stdout.splitlines())
    for cname, pyname in STRUCTS.items():
        cls = getattr(kb, pyname)
        assert int(got[cname]) == C.sizeof(cls), cname
        for f in cls._fields_:
            assert int(got[f"{cname}.{f[0]}"]) == getattr(cls, f[0]).offset, (cname, f[0])


def test_state_aggregate_specs(kb):
    s = kb.agg_spec([0, 1], [("sum", "state", 2, 3), ("avg", "state", 4, 5, (15, 2, 128)), ("count_star", "state", 6),
                             ("min", 7)], partial=True)
    assert s.n_group_by == 2 and s.output == kb.AGG_OUTPUT_PARTIAL
    a = s.aggregates
    assert (a[0].input, a[0].column, a[0].column2) == (kb.AGG_INPUT_STATE, 2, 3)
    assert (a[1].arg_precision, a[1].arg_scale, a[1].arg_bits) == (15, 2, 128)
    assert (a[2].input, a[2].column, a[2].column2) == (kb.AGG_INPUT_STATE, 6, -1)
    assert (a[3].input, a[3].column, a[3].column2) == (kb.AGG_INPUT_RAW, 7, -1)


def test_a_c_program_links_and_calls_the_library(kb, tmp_path):
    """A plain C caller (no Python, no PyTorch) links libkrv_gpu.so through the
    header, reads the version and gets a status, not a crash, from a call
    that needs a device (here: none, or the box's first GPU)."""
    import shutil
    import subprocess
    import torch
    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    src = tmp_path / "caller.c"
    src.write_text(r'''
#include <stdio.h>
#include "krv_gpu.h"
int main(void) {
    krv_runtime *rt = NULL;
    krv_status st = krv_runtime_create(0, 0, NULL, &rt);
    printf("%s\n%d\n", krv_version(), (int)st);
    if (st == KRV_OK) krv_runtime_destroy(rt);
    else printf("%s\n", krv_last_error());
    return 0;
}
''')
    exe = tmp_path / "caller"
    libdir = os.path.dirname(kb.LIB_PATH)
    subprocess.run(["gcc", "-std=c11", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                    "-L", libdir, "-lkrv_gpu", "-Wl,-rpath," + libdir], check=True, capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines()
    assert "sm_100a" in out[0]
    if torch.cuda.is_available():
        assert int(out[1]) == kb.OK
    else:
        assert int(out[1]) in (kb.CUDA_ERROR, kb.INVALID_ARGUMENT) and out[2]


def test_merging_specs(kb):
    """merging() lays out the second phase over the partial states as the
    reference's AggregateExpr::merging does: TPC-H Q1's aggregates after two
    group keys, and integer / float / decimal mixes."""
    import pyarrow as pa
    d15 = pa.decimal128(15, 2)
    q1 = [("sum", 2), ("sum", 3), ("sum", 4), ("sum", 5), ("avg", 2), ("avg", 3), ("avg", 6), ("count_star", 0)]
    types = [d15, d15, pa.decimal128(32, 4), pa.decimal128(38, 6), d15, d15, d15, None]
    assert kb.merging(q1, 2, types) == [
        ("sum", "state", 2, 3), ("sum", "state", 4, 5), ("sum", "state", 6, 7), ("sum", "state", 8, 9),
        ("avg", "state", 10, 11, (15, 2, 128)), ("avg", "state", 12, 13, (15, 2, 128)),
        ("avg", "state", 14, 15, (15, 2, 128)), ("count_star", "state", 16)]
    mix = [("sum", 1), ("min", 1), ("avg", 2), ("count", 3), ("max", 3)]
    assert kb.merging(mix, 1, [pa.int64(), pa.int64(), pa.float64(), pa.int32(), pa.int32()]) == [
        ("sum", "state", 1), ("min", "state", 2), ("avg", "state", 3, 4), ("count", "state", 5), ("max", "state", 6)]
    s = kb.agg_spec([0, 1], kb.merging(q1, 2, types))
    assert s.aggregates[4].arg_bits == 128 and s.aggregates[0].column2 == 3


def test_option_defaults(kb):
    """The partitioned join's options: the device budget from the runtime
    and a Bloom filter of 10 bits per build key in the partition pass."""
    import ctypes as C
    o = kb.GraceOptions()
    o.probe_filter_bits = -1
    kb.lib().krv_grace_options_init(C.byref(o))
    assert o.device_budget_bytes == 0 and o.probe_filter_bits == 10
    assert (kb.PQ_INT32, kb.PQ_INT64, kb.PQ_DOUBLE, kb.PQ_BYTE_ARRAY) == (1, 2, 5, 6)  # parquet.thrift Type
