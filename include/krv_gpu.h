/*
 * krv_gpu.h -- C ABI of the B200 (sm_100a) hash join, grouped hash aggregate
 * and runtime key filter (split-block Bloom) operators.
 *
 * The operators are drop-ins for the Krishiv engine's physical operators on
 * this path. Each entry point names the reference interface it replaces
 * (file:line in the Krishiv engine repository). Data crosses as Arrow
 * RecordBatches through the Arrow C Data Interface (host buffers) or the
 * Arrow C Device Data Interface (CUDA device buffers), see krv_arrow.h.
 *
 * Conventions
 *  - Every call returns a krv_status. Negative values are errors; the text
 *    of the last error on the calling thread is krv_last_error().
 *  - Inputs are borrowed: the caller owns an input ArrowArray until the call
 *    returns and the library never calls its release callback. Outputs are
 *    moved to the caller, who releases them (the C Data Interface's release
 *    callback frees the library-owned buffers).
 *  - A handle is thread-compatible: one thread at a time. Every handle runs
 *    on its runtime's CUDA stream. A built join table is read-only after
 *    krv_join_build_finish.
 *  - Device memory is charged to the runtime's HBM budget; a call that would
 *    exceed it returns KRV_NEED_MEMORY and krv_last_need_bytes() tells how
 *    many bytes it asked for (the reference's SinkStatus::NeedMemory /
 *    OperatorOutput::NeedMemory, crates/krishiv-exec/src/operator.rs:188-477).
 *  - Kernels never trap. They report errors through a device status word.
 */
#ifndef KRV_GPU_H
#define KRV_GPU_H

#include <stddef.h>
#include <stdint.h>

#include "krv_arrow.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Every declaration below is an exported symbol of libkrv_gpu.so (the
 * library builds with hidden visibility by default). */
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

typedef int32_t krv_status;

/* Operator protocol (OperatorOutput / SinkStatus, operator.rs:188-311, 346-477) */
#define KRV_OK 0
#define KRV_NEED_MORE_INPUT 1   /* output (if any) written; feed the next batch */
#define KRV_HAVE_MORE_OUTPUT 2  /* output written; call again with no input */
#define KRV_FINISHED 3          /* no more output */
/* Errors (KrishivError classes the path raises) */
#define KRV_INVALID_ARGUMENT (-1)
#define KRV_UNSUPPORTED (-2)          /* KRISHIV_UNSUPPORTED_FEATURE, join/mod.rs:745-752 */
#define KRV_NEED_MEMORY (-3)          /* over the HBM budget */
#define KRV_ARITHMETIC_OVERFLOW (-4)  /* ARITHMETIC_OVERFLOW, aggregate/mod.rs:1177 (ANSI) */
#define KRV_CUDA_ERROR (-5)
#define KRV_TIMEOUT (-6)              /* a device wait gave up (bounded spin) */
#define KRV_TOO_MANY_ROWS (-7)        /* SCALAR_SUBQUERY_TOO_MANY_ROWS (single-match join) */
#define KRV_INTERNAL (-8)

/* Text of the last failing call on this thread ("" if none). */
const char *krv_last_error(void);
/* Bytes the last KRV_NEED_MEMORY on this thread asked for. */
int64_t krv_last_need_bytes(void);
/* Library version string. */
const char *krv_version(void);

/* ---- runtime: device, stream and HBM budget ------------------------------ */
typedef struct krv_runtime krv_runtime;
/* `cuda_stream` (a cudaStream_t) or NULL for a stream the runtime creates.
 * `hbm_budget_bytes` <= 0: no budget beyond the device's free memory.
 * Replaces the per-query memory pool (crates/krishiv-memory/src/lib.rs:1-30)
 * for device memory. */
krv_status krv_runtime_create(int32_t device, int64_t hbm_budget_bytes, void *cuda_stream,
                              krv_runtime **out);
void krv_runtime_destroy(krv_runtime *rt);
krv_status krv_runtime_synchronize(krv_runtime *rt);
int64_t krv_runtime_used_bytes(const krv_runtime *rt);
int64_t krv_runtime_budget_bytes(const krv_runtime *rt);
void *krv_runtime_stream(const krv_runtime *rt);
/* Kernels this library launched on the runtime since it was created. */
int64_t krv_runtime_launches(const krv_runtime *rt);

/* ---- hash join ------------------------------------------------------------ */
/* JoinType, crates/krishiv-exec/src/join/mod.rs:216-293 */
#define KRV_JOIN_INNER 0
#define KRV_JOIN_LEFT_OUTER 1
#define KRV_JOIN_LEFT_SEMI 2
#define KRV_JOIN_LEFT_ANTI 3
#define KRV_JOIN_NULL_AWARE_ANTI 4
#define KRV_JOIN_EXISTENCE 5
#define KRV_JOIN_RIGHT_SEMI 6
#define KRV_JOIN_RIGHT_ANTI 7
#define KRV_JOIN_RIGHT_OUTER 8
#define KRV_JOIN_FULL_OUTER 9

#define KRV_MAX_KEYS 4
#define KRV_MAX_OUT_COLUMNS 32

/* JoinSpec, join/mod.rs:327-350, plus the join's config keys
 * (krishiv.exec.join.radixBits, crates/krishiv-common/src/config/
 * registry_join.rs:11-160) and the runtime filter options. Key columns are
 * int32/int64/date32/decimal/float64, or (unpartitioned joins) UTF-8 ("u")
 * and binary ("z") columns, whose key tuples are then coded as one int64;
 * string columns (keys included) may be projected into the output, and such
 * a join publishes no runtime filter. */
typedef struct {
    int32_t join_type;                     /* KRV_JOIN_* */
    int32_t n_keys;                        /* 1..KRV_MAX_KEYS */
    int32_t probe_keys[KRV_MAX_KEYS];      /* probe (left) key columns */
    int32_t build_keys[KRV_MAX_KEYS];      /* build (right) key columns */
    int32_t null_safe[KRV_MAX_KEYS];       /* `<=>` instead of `=` */
    int32_t single_match;                  /* LeftOuter only: > 1 match fails */
    int32_t has_residual_filter;           /* 1: krv_join_set_filter gives the filter before the build */
    /* Output projection: probe columns then build columns. -1 = every column. */
    int32_t n_probe_out;
    int32_t probe_out[KRV_MAX_OUT_COLUMNS];
    int32_t n_build_out;
    int32_t build_out[KRV_MAX_OUT_COLUMNS];
    /* Tuning; 0 selects the autotuned value. */
    int32_t radix_bits;        /* level-0 partitions of a partitioned build */
    float max_load;            /* hash-table load factor */
    uint64_t seed;             /* table hash seed g = fin(h ^ seed) (0: fixed default) */
    int32_t runtime_filter;    /* build a key filter at build_finish (one key only) */
    int32_t pad0;
    int64_t build_rows_hint;   /* presize the build arena */
    int64_t max_output_rows;   /* output batch bound; 0 = one batch per input */
} krv_join_spec;
void krv_join_spec_init(krv_join_spec *spec);

/* ---- residual join filters ----------------------------------------------
 * JoinSpec::filter (join/mod.rs:327-350), applied to every candidate pair of
 * equal keys before it counts (join/probe.rs:393-489, the filter at
 * :425-436): a pair matches only where the filter is TRUE (NULL is not a
 * match), and the outer, semi, anti and existence results and the build-side
 * marks of right/full joins follow the filtered matches; single_match counts
 * filtered matches. The filter is a conjunction of comparisons between
 * probe columns, build columns and constants (columns of the input batches,
 * by index). Operands are int32/int64/date32 columns, decimal64 columns
 * (compared as unscaled values: both sides of a comparison of two decimal
 * columns must have one scale; a constant is unscaled at the column's
 * scale), or float64 columns; a comparison with a float64 operand compares
 * as float64 with Spark's order (NaN equal to NaN and above every other
 * value, -0.0 equal to 0.0). A NULL operand makes its comparison, and so the
 * filter, not TRUE. Not for null-aware anti joins (as the reference, which
 * rejects that combination), partitioned joins, or joins on string keys. */
#define KRV_MAX_FILTER_TERMS 8
#define KRV_CMP_EQ 0
#define KRV_CMP_NE 1
#define KRV_CMP_LT 2
#define KRV_CMP_LE 3
#define KRV_CMP_GT 4
#define KRV_CMP_GE 5
#define KRV_OPERAND_PROBE 0      /* column `column` of the probe batch */
#define KRV_OPERAND_BUILD 1      /* column `column` of the build batch */
#define KRV_OPERAND_CONST_I64 2  /* the constant i64 */
#define KRV_OPERAND_CONST_F64 3  /* the constant f64 */
typedef struct {
    int32_t kind;    /* KRV_OPERAND_* */
    int32_t column;
    int64_t i64;
    double f64;
} krv_filter_operand;
typedef struct {
    int32_t op;      /* KRV_CMP_*: left op right */
    int32_t pad0;
    krv_filter_operand left, right;
} krv_filter_term;
typedef struct {
    int32_t n_terms; /* 1..KRV_MAX_FILTER_TERMS, all of which must be TRUE */
    int32_t pad0;
    krv_filter_term terms[KRV_MAX_FILTER_TERMS];
} krv_join_filter;

/* Counters (join/mod.rs:353-607) */
typedef struct {
    int64_t build_rows;
    int64_t build_keys;        /* distinct keys indexed */
    int64_t table_slots;
    int64_t probe_rows;
    int64_t output_rows;
    int64_t max_chain;         /* longest duplicate chain */
    int64_t partitions;        /* level-0 partitions of a partitioned build */
} krv_join_counters;

typedef struct krv_join krv_join;
typedef struct krv_key_filter krv_key_filter;

/* HashJoin::try_new (join/mod.rs:1014) */
krv_status krv_join_create(krv_runtime *rt, const krv_join_spec *spec, krv_join **out);
/* Sets the join's residual filter (see krv_join_filter); before the first
 * build push. Column operands are checked against the batches' schemas at
 * the first probe. */
krv_status krv_join_set_filter(krv_join *j, const krv_join_filter *filter);
/* BuildSink::sink (join/build.rs:1225-1335) */
krv_status krv_join_build_push(krv_join *j, const struct ArrowArray *batch,
                               const struct ArrowSchema *schema);
krv_status krv_join_build_push_device(krv_join *j, const struct ArrowDeviceArray *batch,
                                      const struct ArrowSchema *schema);
/* BuildSink::finalize (join/build.rs:1366-1695) */
krv_status krv_join_build_finish(krv_join *j);
/* ProbeOp::execute (join/probe.rs:1103): joins `in` (NULL to drain pending
 * output) into `out`. KRV_NEED_MORE_INPUT when this input is done,
 * KRV_HAVE_MORE_OUTPUT when more output waits. */
krv_status krv_join_probe(krv_join *j, const struct ArrowArray *in,
                          const struct ArrowSchema *in_schema, struct ArrowArray *out,
                          struct ArrowSchema *out_schema);
krv_status krv_join_probe_device(krv_join *j, const struct ArrowDeviceArray *in,
                                 const struct ArrowSchema *in_schema,
                                 struct ArrowDeviceArray *out, struct ArrowSchema *out_schema);
/* ProbeOp::finish / end_input (join/probe.rs:1149-1228) and emit_build
 * (:610-): rows emitted once every probe row is known (right semi/anti,
 * right/full outer build rows). KRV_HAVE_MORE_OUTPUT or KRV_FINISHED. */
krv_status krv_join_finish(krv_join *j, struct ArrowArray *out, struct ArrowSchema *out_schema);
krv_status krv_join_finish_device(krv_join *j, struct ArrowDeviceArray *out,
                                  struct ArrowSchema *out_schema);
/* The runtime filter published at build_finish (BuildSink::publish,
 * join/build.rs:482). A new reference: destroy it with krv_key_filter_destroy. */
krv_status krv_join_key_filter(krv_join *j, krv_key_filter **out);
krv_status krv_join_counters_get(const krv_join *j, krv_join_counters *out);
void krv_join_destroy(krv_join *j);

/* The key hash the join tables and partitions use, for every row of a device
 * batch: the seedless row hash h of the key columns (RowLayout::encode +
 * fold/mix, rows/layout.rs:487-555, 1131-1144: a NULL key mixes NULL_HASH when
 * null_safe[k] is set and is skipped otherwise), g = fin(h ^ seed)
 * (rows/layout.rs:1080), and the partition id at `depth` (Hashing::partition,
 * join/keys.rs:118-128, and the grace levels of hash.rs:139-148: depth 0 takes
 * the top `radix` bits of h, radix clamped to 3..6; depth d >= 1 takes bits
 * [48-3d, 51-3d) of g, d clamped to 6). out_h, out_g (uint64) and out_part
 * (int32) are device arrays of the batch's length on the runtime's device;
 * any of them may be NULL. Asynchronous on the runtime's stream. */
krv_status krv_hash_rows_device(krv_runtime *rt, const struct ArrowDeviceArray *batch,
                                const struct ArrowSchema *schema, const int32_t *key_columns,
                                const int32_t *null_safe, int32_t n_keys, uint64_t seed, int32_t depth,
                                int32_t radix, uint64_t *out_h, uint64_t *out_g, int32_t *out_part);

/* ---- partitioned (grace) hash join -----------------------------------------
 * The engine's grace join (join/grace.rs:828-1481): both sides are radix
 * partitioned by the key hash (level 0: top radix_bits of h, 3..6; a partition
 * still too large is split 8 ways by bits [48-3d, 51-3d) of g); partitions are
 * joined in HBM while their tables fit half of the device budget and spill to
 * page-locked host memory otherwise. Inner and left outer joins on one int64
 * key (NULL keys allowed); other columns 4 or 8 bytes wide, without NULLs.
 * Same calls as krv_join_*: krv_join_probe returns the rows it can join now
 * (KRV_HAVE_MORE_OUTPUT while more wait), and after the last probe batch
 * krv_join_finish returns the spilled partitions' rows, one batch per call,
 * KRV_HAVE_MORE_OUTPUT until the last (KRV_FINISHED). spec->build_rows_hint,
 * when set, decides the partitions and which of them spill up front. */
typedef struct {
    int64_t device_budget_bytes;  /* device bytes for the join (0: the runtime's budget, else half the free memory) */
    /* Bits per build key of the blocked Bloom filter that the build side's
     * partition pass fills (one 32-byte block per key, keyed by the row hash
     * h) and the probe side's partition pass tests: a probe row it rules out
     * matches nothing, so it is padded at once (left outer) or dropped
     * (inner) and is never partitioned or spilled. Sized from
     * spec->build_rows_hint, else 1/32 of the budget up to 64 MiB; at most
     * 1/16 of the budget. 0: no filter. krv_grace_options_init sets 10. */
    int32_t probe_filter_bits;
    int32_t pad0;
    int64_t reserved[2];
} krv_grace_options;
void krv_grace_options_init(krv_grace_options *o);
krv_status krv_join_create_partitioned(krv_runtime *rt, const krv_join_spec *spec, const krv_grace_options *opt,
                                       krv_join **out);
/* Partitions of a partitioned join that spilled to host memory. */
int64_t krv_join_spilled_partitions(const krv_join *j);
/* Probe rows of a partitioned join that its Bloom filter ruled out in the
 * partition pass (0 for an unpartitioned join or without the filter). */
int64_t krv_join_filtered_probe_rows(const krv_join *j);

/* ---- grouped hash aggregate ---------------------------------------------- */
/* AggregateFunction (aggregate/mod.rs:134), the core five. MIN/MAX of a
 * decimal128 column of precision 19 to 38 keep all 128 bits (the reference's
 * MinMax over Values::Int(i128), aggregate/accumulator.rs:238-248); MIN/MAX
 * of UTF-8 and binary columns compare bytes (MinMax over Values::Bytes);
 * COUNT takes any column. An aggregate with 128-bit or string MIN/MAX runs
 * its global-table kernels only. */
#define KRV_AGG_COUNT_STAR 0
#define KRV_AGG_COUNT 1
#define KRV_AGG_SUM 2
#define KRV_AGG_MIN 3
#define KRV_AGG_MAX 4
#define KRV_AGG_AVG 5

#define KRV_AGG_MODE_AUTO 0
#define KRV_AGG_MODE_GLOBAL 1   /* one global hash table */
#define KRV_AGG_MODE_SHARED 2   /* shared-memory pre-aggregation + global table */

#define KRV_MAX_AGGREGATES 32
#define KRV_MAX_GROUP_KEYS 8

/* AggInput (aggregate/mod.rs:413-419) and AggregateOutput (:421-427) */
#define KRV_AGG_INPUT_RAW 0
#define KRV_AGG_INPUT_STATE 1
#define KRV_AGG_OUTPUT_FINAL 0
#define KRV_AGG_OUTPUT_PARTIAL 1

/* AggregateExpr (aggregate/mod.rs:431-454). With KRV_AGG_INPUT_STATE the
 * arguments are the state columns a KRV_AGG_OUTPUT_PARTIAL aggregate wrote
 * for the same function (AggregateExpr::merging, :561-569): `column` is the
 * first, `column2` the second where the state has two (SUM of a decimal:
 * sum, nonempty; AVG: sum, count), and arg_precision / arg_scale /
 * arg_bits describe the raw decimal argument (AVG of a decimal, whose result
 * type follows the raw type; 0: derived from the state's sum type). */
typedef struct {
    int32_t function;  /* KRV_AGG_* */
    int32_t column;    /* input column (ignored by raw COUNT(*)) */
    int32_t input;     /* KRV_AGG_INPUT_* */
    int32_t column2;   /* second state column, or -1 */
    int32_t arg_precision, arg_scale;
    int32_t arg_bits;  /* the raw decimal argument's width, 64 or 128 (0: the state sum's) */
    int32_t reserved;
} krv_agg_expr;

/* AggregateSpec, aggregate/mod.rs:1083-1108 (final output). Group keys: one
 * int32/int64/date32/decimal(18) column runs on the single-key tables
 * directly; up to KRV_MAX_GROUP_KEYS columns of those types, decimal(38),
 * float64, UTF-8 strings ("u") and binary ("z") are first given dense codes
 * (NULL is a key value; float keys compare normalised). String and binary
 * columns are taken as group keys only. */
typedef struct {
    int32_t n_group_by;             /* 1..KRV_MAX_GROUP_KEYS */
    int32_t group_by[KRV_MAX_GROUP_KEYS];
    int32_t n_aggregates;
    krv_agg_expr aggregates[KRV_MAX_AGGREGATES];
    int32_t ansi;                   /* spark.sql.ansi.enabled: overflow raises */
    int32_t mode;                   /* KRV_AGG_MODE_* */
    int64_t expected_groups;        /* planner estimate (0: unknown) */
    int64_t max_output_rows;        /* output batch bound; 0 = one batch */
    int32_t output;                 /* KRV_AGG_OUTPUT_*: final values, or each aggregate's
                                       state columns (AggregateExpr::state_fields, :747-800):
                                       COUNT: count; SUM: sum (+ nonempty for decimals);
                                       AVG: sum, count; MIN/MAX: value */
    int32_t reserved;
} krv_agg_spec;
void krv_agg_spec_init(krv_agg_spec *spec);

typedef struct krv_agg krv_agg;
/* HashAggregate::new (aggregate/sink.rs:222) */
krv_status krv_agg_create(krv_runtime *rt, const krv_agg_spec *spec, krv_agg **out);
/* HashAggregate::sink (aggregate/sink.rs:1459) */
krv_status krv_agg_push(krv_agg *a, const struct ArrowArray *batch,
                        const struct ArrowSchema *schema);
krv_status krv_agg_push_device(krv_agg *a, const struct ArrowDeviceArray *batch,
                               const struct ArrowSchema *schema);
/* HashAggregate::finalize (aggregate/sink.rs:1585) */
krv_status krv_agg_finish(krv_agg *a);
/* impl Source for HashAggregate (aggregate/sink.rs:1854): the next result
 * batch (group key, then one column per aggregate). KRV_HAVE_MORE_OUTPUT
 * while more batches wait, KRV_FINISHED with the last one. */
krv_status krv_agg_next_output(krv_agg *a, struct ArrowArray *out,
                               struct ArrowSchema *out_schema);
krv_status krv_agg_next_output_device(krv_agg *a, struct ArrowDeviceArray *out,
                                      struct ArrowSchema *out_schema);
/* Groups currently in the table. */
int64_t krv_agg_groups(const krv_agg *a);
void krv_agg_destroy(krv_agg *a);

/* ---- runtime key filter (split-block Bloom) ------------------------------- */
/* KeyFilterOptions, crates/krishiv-io/src/runtime_filter/filter.rs:29-73 */
typedef struct {
    int64_t max_values;        /* 50 */
    int64_t exact_max_values;  /* 4096 (member.rs:38) */
    int32_t bloom;             /* 1 */
    int32_t pad0;
    int64_t bloom_max_items;   /* 4,000,000 */
    int64_t bloom_max_bytes;   /* 8 MiB */
    double bloom_fpp;          /* 0.01 */
    double bloom_max_fpp;      /* 0.05 */
    int64_t bloom_bytes;       /* planned size, 0 = sized for the keys */
} krv_key_filter_options;
/* KeyFilterOptions::default (filter.rs:89-104) */
void krv_key_filter_options_default(krv_key_filter_options *o);

#define KRV_FILTER_RANGE 0   /* min/max only (or a dense range: exact) */
#define KRV_FILTER_EXACT 1   /* exact set of <= exact_max_values keys */
#define KRV_FILTER_BLOOM 2   /* range + split-block Bloom filter */
#define KRV_FILTER_EMPTY 3   /* no key: nothing passes */

typedef struct {
    int32_t form;
    int32_t nulls_pass;
    int32_t has_range;
    int32_t pad0;
    int64_t lo, hi;
    int64_t keys;         /* non-NULL keys added, duplicates counted */
    int64_t distinct;     /* distinct keys (exact) */
    int64_t bloom_bytes;
} krv_key_filter_info;

/* KeyFilterBuilder::add + finish (filter.rs:157-593) over column `column` of
 * `batch` (int64 keys; NULL keys are not kept, as for an `=` join key). */
krv_status krv_key_filter_build(krv_runtime *rt, const krv_key_filter_options *opt,
                                const struct ArrowArray *batch, const struct ArrowSchema *schema,
                                int32_t column, krv_key_filter **out);
krv_status krv_key_filter_build_device(krv_runtime *rt, const krv_key_filter_options *opt,
                                       const struct ArrowDeviceArray *batch,
                                       const struct ArrowSchema *schema, int32_t column,
                                       krv_key_filter **out);
/* KeyFilter::evaluate (filter.rs:768-798): a boolean column, TRUE where the
 * row of `column` may match. */
krv_status krv_key_filter_evaluate(krv_key_filter *f, const struct ArrowArray *batch,
                                   const struct ArrowSchema *schema, int32_t column,
                                   struct ArrowArray *out, struct ArrowSchema *out_schema);
krv_status krv_key_filter_evaluate_device(krv_key_filter *f, const struct ArrowDeviceArray *batch,
                                          const struct ArrowSchema *schema, int32_t column,
                                          struct ArrowDeviceArray *out,
                                          struct ArrowSchema *out_schema);
krv_status krv_key_filter_info_get(const krv_key_filter *f, krv_key_filter_info *out);
/* The Bloom bits in the Parquet SBBF layout (RuntimeBloom::to_bytes). */
krv_status krv_key_filter_bloom_bytes(const krv_key_filter *f, void *host_out, int64_t nbytes);
void krv_key_filter_destroy(krv_key_filter *f);

/* ---- Parquet column chunks decoded on the device -----------------------------
 * The engine's Parquet reader (crates/krishiv-io/src/parquet/decode.rs) decodes
 * row groups on the host and evaluates pushed predicates once per dictionary
 * entry of a dictionary-encoded chunk (parquet/dict_probe.rs:1-27, `passes`,
 * `any_entry_in`). krv_parquet_decode_chunk takes one column chunk's bytes as
 * the file stores them (host memory, from the chunk's dictionary page, or
 * first data page, through its last page: ColumnMetaData.dictionary_page_offset
 * or data_page_offset, total_compressed_size), walks the page headers on the
 * host, and decompresses and decodes every page on the device into one Arrow
 * column of `num_values` rows. With a key filter, the batch gets a second,
 * boolean column "pass": TRUE where the row may match (KeyFilter::evaluate,
 * filter.rs:776-798), evaluated on the encoded pages: once per dictionary
 * entry for dictionary-encoded pages, per value for PLAIN ones; a NULL row
 * passes only if the filter lets NULLs pass. info->dictionary_passing = 0
 * says that no row of the chunk can pass but a NULL (the row group can be
 * skipped, as any_entry_in decides). Flat columns (max definition level 0 or
 * 1, no repetition); physical INT32 (as "i", "tdD", "l", "d:p,s,64" or
 * "d:p,s"), INT64 (as "l", "d:p,s,64" or "d:p,s"), DOUBLE (as "g") and
 * BYTE_ARRAY (as "u" or "z": int32 offsets and bytes);
 * PLAIN, PLAIN_DICTIONARY and RLE_DICTIONARY values; UNCOMPRESSED and SNAPPY
 * chunks; data pages v1 and v2. Others: KRV_UNSUPPORTED. Bytes that do not
 * decode: KRV_INVALID_ARGUMENT. The filter applies to integer columns. */
#define KRV_PQ_INT32 1         /* parquet.thrift Type */
#define KRV_PQ_INT64 2
#define KRV_PQ_DOUBLE 5
#define KRV_PQ_BYTE_ARRAY 6
#define KRV_PQ_UNCOMPRESSED 0  /* parquet.thrift CompressionCodec */
#define KRV_PQ_SNAPPY 1
typedef struct {
    int32_t physical_type;  /* KRV_PQ_INT32, KRV_PQ_INT64, KRV_PQ_DOUBLE or KRV_PQ_BYTE_ARRAY */
    int32_t codec;          /* KRV_PQ_UNCOMPRESSED or KRV_PQ_SNAPPY */
    int32_t max_def_level;  /* 0: required, 1: optional */
    int32_t pad0;
    int64_t num_values;     /* ColumnMetaData.num_values: the chunk's rows */
    const char *format;     /* Arrow format of the decoded column */
    const char *name;       /* its name (may be NULL) */
} krv_parquet_column;
typedef struct {
    int64_t rows;
    int64_t pages;               /* data pages */
    int64_t dictionary_entries;  /* 0 without a dictionary page */
    int64_t dictionary_passing;  /* entries the filter passes (-1: no filter, no dictionary, or
                                    some data page not dictionary encoded) */
    int64_t passing_rows;        /* rows the filter passes (-1: no filter) */
} krv_parquet_info;
krv_status krv_parquet_decode_chunk(krv_runtime *rt, const void *chunk, int64_t chunk_bytes,
                                    const krv_parquet_column *column, const krv_key_filter *filter,
                                    struct ArrowDeviceArray *out, struct ArrowSchema *out_schema,
                                    krv_parquet_info *info);

/* ---- star join pipeline (runtime filter + two joins + grouped sum) --------
 * The fused plan shape
 *   SELECT d.attr, SUM(f.price * (1 - f.discount))
 *   FROM fact f JOIN dim_a a ON f.fk_a = a.key JOIN dim_b b ON f.fk_b = b.key
 *   WHERE a.pred = :pa AND b.pred = :pb GROUP BY <a or b>.attr
 * built from the operators above: HashJoinNode (join/mod.rs:1188-1211) twice,
 * the runtime filters they publish applied to the fact scan's row stage
 * (crates/krishiv-exec/src/operators/runtime_filter.rs:1-45) and a
 * HashAggregate. KRV_STAR_FUSED runs the fact side as one persistent kernel;
 * KRV_STAR_PLAIN runs one operator per launch through the operator API. */
#define KRV_STAR_FUSED 0
#define KRV_STAR_PLAIN 1
typedef struct {
    int32_t dim_key, dim_pred, dim_attr;             /* columns of both dimension batches */
    int32_t pred_a, pred_b;                          /* the equality constants */
    int32_t fact_fk_a, fact_fk_b, fact_price, fact_discount;
    int32_t group_by;                                /* 0: dim_a.attr, 1: dim_b.attr */
    int32_t use_filters;                             /* apply the runtime filters */
    int32_t mode;                                    /* KRV_STAR_* */
} krv_star_spec;
void krv_star_spec_init(krv_star_spec *spec);
typedef struct krv_star krv_star;
typedef struct {
    int64_t fact_rows;
    int64_t passed_filters;    /* fact rows that passed both runtime filters */
    int64_t joined_rows;       /* fact rows that joined both dimensions */
    int64_t dim_a_keys, dim_b_keys;
    int32_t filter_a_form, filter_b_form;
    int64_t filter_a_bytes, filter_b_bytes;
    int64_t fk_a_sectors;      /* 32-byte sectors of fk_a the fused kernel read */
} krv_star_counters;
krv_status krv_star_create(krv_runtime *rt, const krv_star_spec *spec, krv_star **out);
krv_status krv_star_build(krv_star *s, const struct ArrowArray *dim_a,
                          const struct ArrowSchema *schema_a, const struct ArrowArray *dim_b,
                          const struct ArrowSchema *schema_b);
krv_status krv_star_build_device(krv_star *s, const struct ArrowDeviceArray *dim_a,
                                 const struct ArrowSchema *schema_a,
                                 const struct ArrowDeviceArray *dim_b,
                                 const struct ArrowSchema *schema_b);
/* Adds one fact batch to the running aggregate. In the fused mode a
 * page-locked host batch is not copied whole: fk_b (read whole) crosses the
 * host link in bulk copies overlapping the kernels, fk_a, price and discount
 * are read in place row by row; the call returns when none of the batch's
 * buffers is read any more. */
krv_status krv_star_probe(krv_star *s, const struct ArrowArray *fact,
                          const struct ArrowSchema *schema);
krv_status krv_star_probe_device(krv_star *s, const struct ArrowDeviceArray *fact,
                                 const struct ArrowSchema *schema);
/* The result so far: (attr int32, sum float64), one row per group with rows. */
krv_status krv_star_result(krv_star *s, struct ArrowArray *out, struct ArrowSchema *out_schema);
krv_status krv_star_reset(krv_star *s);
krv_status krv_star_counters_get(const krv_star *s, krv_star_counters *out);
void krv_star_destroy(krv_star *s);

/* The fused plan recognised in an operator chain: fact batch -> join_a ->
 * join_b -> grouped SUM(price * (1 - discount)), as HashJoinNode twice and a
 * HashAggregate would run it (join/mod.rs:1188-1211; runtime filters applied
 * to the fact scan, operators/runtime_filter.rs:1-45). join_a is probed by
 * the fact batch; join_b by join_a's output (probe columns, then build
 * columns, as the join specs project them). Both joins are inner, on one
 * int64 key, unpartitioned, without residual filter, with their build sides
 * finished: those rows, after whatever predicate the caller applied before
 * building, are the dimensions. The chain names, in join_b's output, the
 * int32 build column grouped by and the fact's price (int64) and discount
 * (float64) columns; the runtime filters apply when both joins publish one.
 * The dimensions' rows are copied at the call: the joins may go afterwards.
 * KRV_UNSUPPORTED when the chain is not of this shape (the caller runs the
 * operators one by one). Then krv_star_probe(_device), _result, _destroy. */
typedef struct {
    int32_t n_fact_columns;          /* columns of the fact batch */
    int32_t group_col;               /* column of join_b's output: a build column of either join */
    int32_t price_col, discount_col; /* columns of join_b's output: fact columns */
    int32_t mode;                    /* KRV_STAR_FUSED or KRV_STAR_PLAIN */
} krv_star_chain;
krv_status krv_star_from_joins(krv_runtime *rt, const krv_join *join_a, const krv_join *join_b,
                               const krv_star_chain *chain, krv_star **out);

/* ---- synthetic data on the device (benchmarks) ----------------------------
 * Counter-based SplitMix64 generators: value(seed, column, row) is the same
 * function on every device and in the CPU test oracle. */
#define KRV_GEN_UNIFORM_I64 0   /* int64 uniform in [lo, hi] */
#define KRV_GEN_UNIFORM_I32 1   /* int32 uniform in [lo, hi] */
#define KRV_GEN_UNIT_F64 2      /* float64 lo + (hi - lo) * u, u uniform in [0, 1) */
#define KRV_GEN_PERMUTATION 3   /* int64 permutation of [0, n) (lo + perm) */
#define KRV_GEN_ZIPF 4          /* int64: a Zipf(s = x0) rank over [0, hi) through a permutation */
typedef struct {
    int32_t kind;
    uint32_t column;       /* stream id of this column */
    uint64_t seed;
    int64_t lo, hi;        /* integer bounds / scale */
    double x0, x1;         /* float bounds / Zipf exponent */
    double null_fraction;  /* share of NULL rows (validity stream column + 0x10000) */
    int64_t row0;          /* first row number (generate rows [row0, row0 + n)) */
} krv_gen_spec;
/* Fills `n` values at device pointer `out` (and the validity bitmap at
 * `out_valid`, bit offset 0, when null_fraction > 0 and out_valid != NULL). */
krv_status krv_gen_fill(krv_runtime *rt, const krv_gen_spec *spec, int64_t n, void *out,
                        void *out_valid);

/* ---- request server: batched and served join + aggregate -----------------
 * SELECT t.g, SUM(p.x), COUNT(*) FROM p JOIN t ON p.k = t.k GROUP BY t.g for a
 * stream of probe requests p against build tables t kept resident on the
 * device. The reference runs each such query as a pipeline of its operators
 * (HashJoinNode, join/mod.rs:1188-1211; HashAggregate, aggregate/sink.rs:181);
 * the server is the batching/serving loop around them. Requests are admitted
 * while the state of the running ones (48 bytes per group of their table)
 * fits hbm_budget_bytes, the NeedMemory rule of operator.rs:314-330.
 *  - KRV_SERVE_BATCHED: ticks of at most tick_rows probe rows from every
 *    running request, one probe + aggregate launch per tick fed from a device
 *    work queue, captured as a CUDA graph; large requests span ticks.
 *  - KRV_SERVE_PLAIN: one request at a time through the join and aggregate
 *    operators, one launch per operator step.
 * Tables are (int64 key, int64 group) without NULL groups; requests are
 * (int64 key, int64 value) device batches, NULL keys never match, values
 * without NULLs. The caller keeps a request's buffers alive and unchanged until
 * it is polled. Results are device batches (group int64, SUM int64, COUNT
 * int64), one row per group with a match, in no particular order. */
#define KRV_SERVE_BATCHED 0
#define KRV_SERVE_PLAIN 1
typedef struct {
    int32_t mode;               /* KRV_SERVE_* */
    int32_t autotune;           /* try the candidate kernel shapes on the first ticks */
    int32_t ansi;               /* a SUM that leaves int64 fails its request */
    int32_t max_tick_requests;  /* requests running at once (1..512; 0: 512) */
    int64_t tick_rows;          /* probe rows per tick (0: 64 Mi) */
    int64_t hbm_budget_bytes;   /* device bytes for running requests (0: no limit) */
} krv_server_options;
void krv_server_options_init(krv_server_options *o);
typedef struct {
    int64_t ticks;
    int64_t requests_done;
    int64_t rows_probed;
    int64_t pending;        /* submitted, not admitted */
    int64_t running;        /* admitted, rows left */
    int64_t budget_in_use;  /* bytes of admitted requests' state */
    int32_t tuned;          /* the autotuner has chosen */
    int32_t threads;        /* chosen shape: threads per CTA */
    int64_t item_rows;      /* rows per work item */
    int32_t smem_groups;    /* shared-memory aggregation up to this many groups */
    int32_t pad0;
} krv_server_stats;
typedef struct krv_server krv_server;
krv_status krv_server_create(krv_runtime *rt, const krv_server_options *o, krv_server **out);
/* Builds a resident table from columns key_column and group_column. */
krv_status krv_server_add_table(krv_server *s, const struct ArrowDeviceArray *batch,
                                const struct ArrowSchema *schema, int32_t key_column,
                                int32_t group_column, int64_t *table_id);
krv_status krv_server_drop_table(krv_server *s, int64_t table_id);
krv_status krv_server_submit(krv_server *s, int64_t table_id, const struct ArrowDeviceArray *probe,
                             const struct ArrowSchema *schema, int32_t key_column,
                             int32_t value_column, int64_t *request_id);
/* Retires finished work and starts the next (a tick, or one plain request);
 * with wait != 0 also waits for the oldest tick. *outstanding = requests not
 * yet finished. */
krv_status krv_server_step(krv_server *s, int32_t wait, int64_t *outstanding);
/* KRV_OK with the next finished request (its status in *request_status; the
 * result in out when that is KRV_OK, else out is left released), or
 * KRV_FINISHED when no request has finished. */
krv_status krv_server_poll(krv_server *s, int64_t *request_id, krv_status *request_status,
                           struct ArrowDeviceArray *out, struct ArrowSchema *out_schema);
krv_status krv_server_stats_get(const krv_server *s, krv_server_stats *out);
void krv_server_destroy(krv_server *s);

/* ---- grouped SUM/COUNT with no allocation ----------------------------------
 * No counterpart in the reference. For a caller that may not allocate device
 * memory where it calls (all of HBM is in its own accounted pool, or a
 * cudaMalloc / cudaFree would stall its device): GROUP BY keys with SUM(values)
 * and COUNT(*), both int64 columns without NULLs, the results of
 * krv_agg_create/push/finish for that spec with ansi = 0. The hash table is a
 * fixed device array of this library (4 MiB per device); the call allocates
 * nothing and only launches kernels on `stream` (NULL: the default stream) of
 * the current device. All pointers are device memory of that device.
 *  - max_groups may be at most KRV_SCRATCH_MAX_GROUPS (larger: an
 *    KRV_INVALID_ARGUMENT error before any device work); out_keys, out_sums
 *    and out_counts hold max_groups values each;
 *  - out_info[0] = the number of groups written (in no particular order), or
 *    -1 when the input had more distinct keys than max_groups (the outputs are
 *    then void; so are they when a key found no free slot in 8192 probes, which
 *    takes more distinct keys than the table holds); out_info[1] = 1 when some
 *    sum left int64 and wrapped;
 *  - nothing has to start at zero: each call clears its table first;
 *  - the first call on a device looks up the table's address there: make it
 *    before any stream capture;
 *  - the table is shared by all calls on a device: calls that overlap in time
 *    (other streams or host threads) race. Calls in order on one stream do not. */
#define KRV_SCRATCH_MAX_GROUPS 65536
krv_status krv_agg_sum_i64_scratch(const int64_t *keys, const int64_t *values, int64_t n,
                                   int64_t max_groups, int64_t *out_keys, int64_t *out_sums,
                                   int64_t *out_counts, int64_t *out_info, void *stream);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif
#endif
