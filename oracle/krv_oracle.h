/*
 * krv_oracle.h -- CPU oracle for the hash-join / grouped-aggregate /
 * runtime-Bloom path.
 *
 * TEST INFRASTRUCTURE ONLY. This is a plain-C restatement of the Krishiv
 * engine's CPU algorithms for the path, used by the tests, by the smoke
 * check and by the CPU-baseline leg of the benchmark as the CHECKER. The
 * product library (libkrv_gpu.so) never links, loads or calls it.
 *
 * Every function cites the reference file:line it restates (paths are
 * relative to the Krishiv engine repository).
 */
#ifndef KRV_ORACLE_H
#define KRV_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- key columns --------------------------------------------------------
 * One key column: `width` bytes per value (4, 8 or 16, little endian),
 * `is_float` for float64 keys (normalized -0.0 -> 0.0, one NaN), `valid`
 * one byte per row (1 = valid) or NULL for "no NULLs". */
typedef struct {
    const void *data;
    const uint8_t *valid;
    int32_t width;
    int32_t is_float;
} orc_col;

/* crates/krishiv-exec/src/rows/layout.rs:1131-1139 (fold) */
uint64_t orc_fold(uint64_t a, uint64_t b);
/* rows/layout.rs:487-555, 790-798, 871-904: the seedless stored hash `h` of
 * each row. `null_bit[c]` != 0 gives column c a validity bit (join layout:
 * only null-safe keys, rows/layout.rs:330-334), so a NULL mixes NULL_HASH. */
void orc_row_hash(const orc_col *cols, int ncols, const int32_t *null_bit,
                  int64_t n, uint64_t *out);
/* rows/layout.rs:1080-1082 */
uint64_t orc_finalize(uint64_t h, uint64_t seed);
/* crates/krishiv-exec/src/join/keys.rs:118-128 */
int32_t orc_partition(uint64_t h, int32_t depth, int32_t radix, uint64_t seed);
/* crates/krishiv-exec/src/join/build.rs:470-475 */
uint64_t orc_null_spread(uint64_t seq);

/* crates/krishiv-kernels/src/hash/routing.rs:112-142 -- XXH64 (seed 0) of
 * the `nbytes` (1, 2, 4, 8, 16) little-endian bytes of (hi:lo). */
uint64_t orc_xxh64_fixed(uint64_t lo, uint64_t hi, int32_t nbytes);
/* crates/krishiv-io/src/runtime_filter/hash.rs:56-65 for every row. */
void orc_int_hashes(const int64_t *v, int64_t n, int32_t width, uint64_t *out);

/* ---- split-block Bloom filter (crates/krishiv-io/src/runtime_filter/bloom.rs) */
/* bloom.rs:96-110 */
int64_t orc_bloom_bytes_for(uint64_t items, double fpp);
/* bloom.rs:136-148 (words: bytes/4 u32, zeroed by the caller) */
void orc_bloom_insert(uint32_t *words, int64_t nbytes, const uint64_t *hashes, int64_t n);
/* bloom.rs:184-196 (one byte per answer) */
void orc_bloom_check(const uint32_t *words, int64_t nbytes, const uint64_t *hashes,
                     int64_t n, uint8_t *out);
/* bloom.rs:275- */
double orc_bloom_expected_fpp(int64_t nbytes, uint64_t items);

/* ---- key filter (crates/krishiv-io/src/runtime_filter/filter.rs) -------- */
enum { ORC_FORM_RANGE = 0, ORC_FORM_EXACT = 1, ORC_FORM_BLOOM = 2, ORC_FORM_EMPTY = 3 };
typedef struct {
    int32_t form;         /* ORC_FORM_* of the member test */
    int32_t nulls_pass;   /* a NULL key was stored (null-safe key) */
    int32_t has_range;
    int32_t pad;
    int64_t lo, hi;       /* the key range */
    int64_t keys;         /* non-NULL keys added (with duplicates) */
    int64_t distinct;     /* distinct non-NULL keys */
    int64_t bloom_bytes;  /* Bloom size when form == BLOOM */
} orc_key_filter;
/* filter.rs:231-330 (add), 533-593 (finish_with), 595-621 (dense, bloom)
 * with the default options filter.rs:89-104. int64 keys (width 8).
 * `bloom_words` (>= 8 MiB / 4 words) receives the Bloom bits. */
void orc_key_filter_build(const int64_t *keys, const uint8_t *valid, int64_t n,
                          orc_key_filter *out, uint32_t *bloom_words,
                          int64_t **exact_set, int64_t *exact_n);
/* filter.rs:776-798 + member.rs:423-560: 1 = the row may match. */
void orc_key_filter_eval(const orc_key_filter *f, const uint32_t *bloom_words,
                         const int64_t *exact_set, int64_t exact_n,
                         const int64_t *keys, const uint8_t *valid, int64_t n,
                         uint8_t *out);

/* ---- hash join (crates/krishiv-exec/src/join/) ---------------------------- */
enum {
    ORC_INNER = 0, ORC_LEFT_OUTER = 1, ORC_LEFT_SEMI = 2, ORC_LEFT_ANTI = 3,
    ORC_NULL_AWARE_ANTI = 4, ORC_EXISTENCE = 5, ORC_RIGHT_SEMI = 6,
    ORC_RIGHT_ANTI = 7, ORC_RIGHT_OUTER = 8, ORC_FULL_OUTER = 9
};
/* The join of probe ⋈ build as index pairs: out_probe[i] / out_build[i] are
 * row numbers, -1 for the NULL-padded side; an existence join writes the
 * `exists` flag (0/1) to out_build. Returns the row count (or -1 on error,
 * -2 for SCALAR_SUBQUERY_TOO_MANY_ROWS under single_match). Arrays are
 * malloc'ed; free with orc_free. Restates join/mod.rs:21-52, 216-293,
 * rows/index.rs:211-283, 375-448, join/probe.rs:266-606. */
int64_t orc_hash_join(int32_t join_type, const orc_col *build_keys, int64_t nb,
                      const orc_col *probe_keys, int64_t np, int32_t nkeys,
                      const int32_t *null_safe, int32_t single_match, uint64_t seed,
                      int32_t radix, int64_t **out_probe, int64_t **out_build);
/* JoinSpec::filter (join/mod.rs:327-350) applied to candidate pairs
 * (join/probe.rs:393-489, :425-436): a conjunction of comparisons whose
 * operands are a probe column, a build column (ORC_SIDE_*: `col`) or a
 * constant (i64, or f64 when is_float); comparisons with a float operand
 * compare as double in Spark's order (NaN equal to NaN and largest, -0.0
 * equal to 0.0); a NULL operand is not TRUE. */
enum { ORC_SIDE_PROBE = 0, ORC_SIDE_BUILD = 1, ORC_SIDE_CONST = 2 };
typedef struct {
    int32_t side;
    int32_t is_float;
    orc_col col;
    int64_t i64;
    double f64;
} orc_operand;
typedef struct {
    int32_t op; /* 0 =, 1 !=, 2 <, 3 <=, 4 >, 5 >= */
    int32_t pad;
    orc_operand l, r;
} orc_term;
typedef struct {
    int32_t n;
    int32_t pad;
    orc_term t[8];
} orc_filter;
/* orc_hash_join with a residual filter (NULL: none). */
int64_t orc_hash_join_filtered(int32_t join_type, const orc_col *build_keys, int64_t nb,
                               const orc_col *probe_keys, int64_t np, int32_t nkeys,
                               const int32_t *null_safe, int32_t single_match, uint64_t seed,
                               int32_t radix, const orc_filter *filter, int64_t **out_probe,
                               int64_t **out_build);
void orc_free(void *p);

/* ---- grouped aggregate (crates/krishiv-exec/src/aggregate/) ---------------- */
enum { ORC_T_I32 = 0, ORC_T_I64 = 1, ORC_T_F64 = 2, ORC_T_DEC64 = 3, ORC_T_DEC128 = 4 };
enum { ORC_COUNT_STAR = 0, ORC_COUNT = 1, ORC_SUM = 2, ORC_MIN = 3, ORC_MAX = 4, ORC_AVG = 5 };
typedef struct {
    const void *data;       /* values (width by type; DEC128 = 16 bytes) */
    const uint8_t *valid;   /* 1 byte per row, NULL = no NULLs */
    int32_t type;           /* ORC_T_* */
    int32_t precision, scale;
    int32_t pad;
} orc_value_col;
typedef struct {
    int32_t func;           /* ORC_COUNT_STAR .. ORC_AVG */
    int32_t col;            /* value column index (ignored for COUNT(*)) */
} orc_agg_expr;
/* One result column per expression, one row per group. Result types follow
 * aggregate/mod.rs:588-740: COUNT -> int64 (i64 slot); SUM int -> int64;
 * SUM/AVG float, AVG int -> float64 (f64 slot); SUM dec(p,s) ->
 * dec(min(38,p+10),s), AVG dec(p,s) -> dec(min(38,p+4),min(38,s+4)) (i128
 * slot as lo/hi); MIN/MAX -> the input type (i64 slot holds ints and
 * decimals, f64 slot floats). `valid` 0 = NULL result. For float SUM/AVG,
 * `f64` holds the compensated (Neumaier) sum-based value and `f64_seq` the
 * reference's sequential `+=` value. */
typedef struct {
    int64_t *i64;
    double *f64;
    double *f64_seq;
    uint64_t *lo;
    int64_t *hi;
    uint8_t *valid;
} orc_agg_out;
/* Group keys: one int64 or int32 column (`key_width` 8/4) with optional
 * validity; NULL keys form one group. Returns the number of groups and
 * writes the key of each group to *out_keys (malloc'ed, with *out_key_valid),
 * fills `outs[e]` (arrays malloc'ed here). Error codes: -3 ANSI overflow
 * (ARITHMETIC_OVERFLOW). Restates aggregate/rowtable.rs (find-or-insert by
 * `g`), accumulator.rs:387-590, accumulator/fold.rs, helpers.rs:498-610. */
int64_t orc_hash_aggregate(const void *key, const uint8_t *key_valid, int32_t key_width,
                           int64_t n, const orc_value_col *cols, int32_t ncols,
                           const orc_agg_expr *exprs, int32_t nexprs, int32_t ansi,
                           int64_t **out_keys, uint8_t **out_key_valid, orc_agg_out *outs);
/* helpers.rs:595-610 (avg_fast) with the avg_decimal (helpers.rs:539-590)
 * digit loop as the fallback. Returns 1 and the value, or 0 when it does not
 * fit decimal(p, s). */
int32_t orc_avg_decimal(int64_t sum_lo, int64_t sum_hi, int32_t sum_scale, int64_t count,
                        int32_t p, int32_t s, uint64_t *out_lo, int64_t *out_hi);

/* ---- synthetic data (counter-based, identical to the device generators) --- */
uint64_t orc_rand(uint64_t seed, uint32_t column, uint64_t row);
/* uniform integer in [lo, hi] */
int64_t orc_rand_range(uint64_t seed, uint32_t column, uint64_t row, int64_t lo, int64_t hi);
/* uniform double in [0, 1) */
double orc_rand_unit(uint64_t seed, uint32_t column, uint64_t row);
/* a seeded permutation of [0, n): a 4-round Feistel network over the
 * smallest even-bit power of two >= n, with cycle walking */
uint64_t orc_permute(uint64_t seed, uint64_t n, uint64_t i);
/* Zipf(s) cumulative table over ranks 1..n: cdf[k-1] = sum_{j<=k} j^-s / H */
void orc_zipf_cdf(double s, int64_t n, double *cdf);
/* the Zipf rank (0-based) of row `row`: first k with cdf[k] > u */
int64_t orc_zipf_rank(const double *cdf, int64_t n, double u);
/* n values of generator `kind` (0 uniform int64 [lo, hi], 1 uniform int32,
 * 2 float64 x0 + (x1 - x0) * u, 3 permutation lo + perm_seed(n = hi),
 * 4 Zipf(x0) over hi values through a permutation); valid[i] = 0 is a NULL
 * (share null_fraction). */
void orc_gen_column(uint64_t seed, uint32_t column, int32_t kind, int64_t lo, int64_t hi, double x0,
                    double x1, int64_t row0, int64_t n, double null_fraction, void *out,
                    uint8_t *valid);

#ifdef __cplusplus
}
#endif
#endif
