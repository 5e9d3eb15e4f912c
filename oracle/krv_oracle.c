/*
 * krv_oracle.c -- CPU oracle (TEST INFRASTRUCTURE ONLY) for the hash join,
 * grouped aggregate and runtime Bloom filter path of the Krishiv engine.
 *
 * A plain-C restatement of the reference's CPU algorithms, used only by the
 * tests, the smoke check and the benchmark's CPU-baseline leg as the checker.
 * The product library never links or calls it. Citations are file:line in the
 * Krishiv engine repository.
 *
 * Parity of this restatement is pinned against the reference's own
 * known-answer tests (see tests/test_oracle_golden.py):
 *   - crates/krishiv-exec/src/join/keys.rs:348 (seedless h of a known row),
 *   - crates/krishiv-io/src/runtime_filter/hash.rs:144-151 (XXH64 equals the
 *     public XXH64 of the little-endian bytes; checked against python-xxhash),
 *   - crates/krishiv-exec/src/join/keys.rs:345-370 (partition layout),
 *   - crates/krishiv-exec/tests/hash_join/main.rs:128-181 (nested-loop join
 *     oracle over every join type, NULLs, duplicates, empty inputs).
 *
 * Build: oracle/Makefile (gcc -O3 -ffp-contract=off, so float arithmetic is
 * plain IEEE double with no contraction).
 */
#include "krv_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;
typedef __int128 i128;

/* crates/krishiv-exec/src/rows/layout.rs:43-50 */
#define NULL_HASH 0xA5A55A5AC3C33C3CULL
#define MIX 0x243F6A8885A308D3ULL
#define FINISH 0xB7E151628AED2A6BULL
#define FIN 0x6A09E667F3BCC909ULL

/* rows/layout.rs:1131-1139: the folded multiply */
uint64_t orc_fold(uint64_t a, uint64_t b) {
    u128 p = (u128)a * (u128)b;
    return (uint64_t)p ^ (uint64_t)(p >> 64);
}

/* rows/layout.rs:1142-1144 */
static uint64_t mix(uint64_t h, uint64_t v) { return orc_fold(h ^ v, MIX); }

/* rows/layout.rs:1147-1149: every NaN is one NaN, -0.0 is 0.0 */
static uint64_t normalize64_bits(uint64_t bits) {
    double v;
    memcpy(&v, &bits, 8);
    if (isnan(v)) v = NAN;
    else v = v + 0.0;
    uint64_t out;
    memcpy(&out, &v, 8);
    return out;
}

static int col_valid(const orc_col *c, int64_t i) { return !c->valid || c->valid[i]; }

/* The words a fixed-width value mixes in (rows/layout.rs:871-904): each
 * 8-byte chunk of the little-endian value, zero-extended. */
static int value_words(const orc_col *c, int64_t i, uint64_t w[2]) {
    const uint8_t *p = (const uint8_t *)c->data + (size_t)i * (size_t)c->width;
    w[0] = w[1] = 0;
    if (c->width == 4) {
        uint32_t x;
        memcpy(&x, p, 4);
        w[0] = x;
        return 1;
    }
    if (c->width == 8) {
        memcpy(&w[0], p, 8);
        if (c->is_float) w[0] = normalize64_bits(w[0]);
        return 1;
    }
    memcpy(&w[0], p, 8);
    memcpy(&w[1], p + 8, 8);
    return 2;
}

/* rows/layout.rs:487-555: h starts at fold(SEEDLESS, MIX) = fold(0, MIX);
 * per key column in key order, a NULL with a validity bit mixes NULL_HASH
 * (write_nulls :790-798) and a valid value mixes its words (put_fixed
 * :871-904); then h = fold(h, FINISH). */
void orc_row_hash(const orc_col *cols, int ncols, const int32_t *null_bit, int64_t n,
                  uint64_t *out) {
    for (int64_t i = 0; i < n; i++) {
        uint64_t h = orc_fold(0, MIX);
        for (int c = 0; c < ncols; c++) {
            if (!col_valid(&cols[c], i)) {
                if (null_bit && null_bit[c]) h = mix(h, NULL_HASH);
                continue;
            }
            uint64_t w[2];
            int k = value_words(&cols[c], i, w);
            for (int j = 0; j < k; j++) h = mix(h, w[j]);
        }
        out[i] = orc_fold(h, FINISH);
    }
}

/* rows/layout.rs:1080-1082 */
uint64_t orc_finalize(uint64_t h, uint64_t seed) { return orc_fold(h ^ seed, FIN); }

/* join/keys.rs:118-128 (row layout): level 0 = top `radix` bits of h;
 * level d = bits [48-3d, 51-3d) of g. radix clamps to 3..6 (:92-95). */
int32_t orc_partition(uint64_t h, int32_t depth, int32_t radix, uint64_t seed) {
    if (radix < 3) radix = 3;
    if (radix > 6) radix = 6;
    if (depth == 0) return (int32_t)(h >> (64 - radix));
    int32_t d = depth < 6 ? depth : 6;
    uint32_t shift = 48u - 3u * (uint32_t)d;
    return (int32_t)((orc_finalize(h, seed) >> shift) & 7u);
}

/* join/build.rs:470-475 (SplitMix64 finalizer) */
uint64_t orc_null_spread(uint64_t seq) {
    uint64_t z = seq + 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

/* ---- XXH64 (crates/krishiv-kernels/src/hash/routing.rs:86-142) ---------- */
#define P1 0x9E3779B185EBCA87ULL
#define P2 0xC2B2AE3D27D4EB4FULL
#define P3 0x165667B19E3779F9ULL
#define P4 0x85EBCA77C2B2AE63ULL
#define P5 0x27D4EB2F165667C5ULL
static uint64_t rotl(uint64_t x, int r) { return (x << r) | (x >> (64 - r)); }
static uint64_t avalanche(uint64_t h) {
    h ^= h >> 33;
    h *= P2;
    h ^= h >> 29;
    h *= P3;
    return h ^ (h >> 32);
}
static uint64_t lane8(uint64_t h, uint64_t k) {
    uint64_t k1 = rotl(k * P2, 31) * P1;
    return rotl(h ^ k1, 27) * P1 + P4;
}
uint64_t orc_xxh64_fixed(uint64_t lo, uint64_t hi, int32_t nbytes) {
    u128 rest = ((u128)hi << 64) | lo;
    uint64_t h = P5 + (uint64_t)nbytes;
    int left = nbytes;
    while (left >= 8) {
        h = lane8(h, (uint64_t)rest);
        rest >>= 64;
        left -= 8;
    }
    if (left >= 4) {
        uint64_t k = (uint32_t)rest;
        h = rotl(h ^ (k * P1), 23) * P2 + P3;
        rest >>= 32;
        left -= 4;
    }
    while (left > 0) {
        uint64_t b = (uint8_t)rest;
        h = rotl(h ^ (b * P5), 11) * P1;
        rest >>= 8;
        left -= 1;
    }
    return avalanche(h);
}

/* crates/krishiv-io/src/runtime_filter/hash.rs:56-65 */
void orc_int_hashes(const int64_t *v, int64_t n, int32_t width, uint64_t *out) {
    for (int64_t i = 0; i < n; i++) {
        uint64_t bits = (uint64_t)v[i];
        switch (width) {
        case 1: out[i] = orc_xxh64_fixed(bits & 0xFF, 0, 1); break;
        case 2: out[i] = orc_xxh64_fixed(bits & 0xFFFF, 0, 2); break;
        case 4: out[i] = orc_xxh64_fixed(bits & 0xFFFFFFFFULL, 0, 4); break;
        default: out[i] = orc_xxh64_fixed(bits, 0, 8); break;
        }
    }
}

/* ---- SBBF (crates/krishiv-io/src/runtime_filter/bloom.rs) ---------------- */
static const uint32_t SALT[8] = {0x47b6137bu, 0x44974d91u, 0x8824ad5bu, 0xa2b7289du,
                                 0x705495c7u, 0x2df1424bu, 0x9efc4947u, 0x5c6bfb31u};
#define BLOCK_BYTES 32

/* bloom.rs:96-110 */
int64_t orc_bloom_bytes_for(uint64_t items, double fpp) {
    if (fpp < 1e-9) fpp = 1e-9;
    if (fpp > 0.5) fpp = 0.5;
    double bits = -8.0 * (double)items / log(1.0 - pow(fpp, 1.0 / 8.0));
    int64_t bytes = (int64_t)ceil(bits / 8.0);
    int64_t blocks = (bytes + BLOCK_BYTES - 1) / BLOCK_BYTES;
    if (blocks < 1) blocks = 1;
    return blocks * BLOCK_BYTES;
}

/* bloom.rs:129-132 */
static uint64_t bloom_block(uint64_t hash, uint64_t nblocks) {
    return (uint64_t)(((u128)(hash >> 32) * nblocks) >> 32);
}

/* bloom.rs:136-148 with mask :83-89 */
void orc_bloom_insert(uint32_t *words, int64_t nbytes, const uint64_t *hashes, int64_t n) {
    uint64_t nblocks = (uint64_t)nbytes / BLOCK_BYTES;
    for (int64_t i = 0; i < n; i++) {
        uint64_t b = bloom_block(hashes[i], nblocks);
        uint32_t key = (uint32_t)hashes[i];
        for (int w = 0; w < 8; w++) words[b * 8 + w] |= 1u << ((key * SALT[w]) >> 27);
    }
}

/* bloom.rs:184-196 */
void orc_bloom_check(const uint32_t *words, int64_t nbytes, const uint64_t *hashes, int64_t n,
                     uint8_t *out) {
    uint64_t nblocks = (uint64_t)nbytes / BLOCK_BYTES;
    for (int64_t i = 0; i < n; i++) {
        uint64_t b = bloom_block(hashes[i], nblocks);
        uint32_t key = (uint32_t)hashes[i];
        uint32_t miss = 0;
        for (int w = 0; w < 8; w++) {
            uint32_t bit = 1u << ((key * SALT[w]) >> 27);
            miss |= bit & ~words[b * 8 + w];
        }
        out[i] = miss == 0;
    }
}

/* bloom.rs:275-320: Poisson-weighted false-positive estimate */
double orc_bloom_expected_fpp(int64_t nbytes, uint64_t items) {
    double blocks = (double)(nbytes / BLOCK_BYTES);
    double lambda = (double)items / blocks;
    if (lambda == 0.0) return 0.0;
    if (lambda > 1024.0) return pow(1.0 - pow(31.0 / 32.0, lambda), 8);
    double spread = 10.0 * sqrt(lambda) + 20.0;
    double lo = floor(fmax(lambda - spread, 0.0)), hi = lambda + spread;
    double ln_p = -lambda;
    double k = 1.0;
    while (k <= lo) {
        ln_p += log(lambda) - log(k);
        k += 1.0;
    }
    double total = 0.0;
    k = lo;
    while (k <= hi) {
        double word = 1.0 - pow(31.0 / 32.0, k);
        total += exp(ln_p) * pow(word, 8);
        k += 1.0;
        ln_p += log(lambda) - log(k);
    }
    return total;
}

/* ---- key filter (crates/krishiv-io/src/runtime_filter/filter.rs) -------- */
/* Options: filter.rs:89-104 */
#define OPT_MAX_VALUES 50
#define OPT_EXACT_MAX 4096 /* member.rs:38 EXACT_SET_MAX */
#define OPT_BLOOM_MAX_ITEMS 4000000ULL
#define OPT_BLOOM_MAX_BYTES (8LL << 20)
#define OPT_BLOOM_FPP 0.01
#define OPT_BLOOM_MAX_FPP 0.05

static int cmp_i64(const void *a, const void *b) {
    int64_t x = *(const int64_t *)a, y = *(const int64_t *)b;
    return x < y ? -1 : x > y;
}

void orc_key_filter_build(const int64_t *keys, const uint8_t *valid, int64_t n,
                          orc_key_filter *out, uint32_t *bloom_words, int64_t **exact_set,
                          int64_t *exact_n) {
    memset(out, 0, sizeof(*out));
    *exact_set = NULL;
    *exact_n = 0;
    /* add (filter.rs:231-300): the kept rows are the valid ones; NULL `=`
     * keys are never kept by a join build, so nulls_pass stays false. */
    int64_t rows = 0, lo = INT64_MAX, hi = INT64_MIN;
    int64_t *kept = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
    for (int64_t i = 0; i < n; i++) {
        if (valid && !valid[i]) continue;
        kept[rows++] = keys[i];
        if (keys[i] < lo) lo = keys[i];
        if (keys[i] > hi) hi = keys[i];
    }
    out->keys = rows;
    if (rows == 0) {
        out->form = ORC_FORM_EMPTY;
        free(kept);
        return;
    }
    out->has_range = 1;
    out->lo = lo;
    out->hi = hi;
    /* distinct keys */
    int64_t *sorted = (int64_t *)malloc(sizeof(int64_t) * (size_t)rows);
    memcpy(sorted, kept, sizeof(int64_t) * (size_t)rows);
    qsort(sorted, (size_t)rows, sizeof(int64_t), cmp_i64);
    int64_t d = 0;
    for (int64_t i = 0; i < rows; i++)
        if (i == 0 || sorted[i] != sorted[i - 1]) sorted[d++] = sorted[i];
    out->distinct = d;
    /* finish_with (filter.rs:533-593) */
    int64_t distinct_max = OPT_MAX_VALUES > OPT_EXACT_MAX ? OPT_MAX_VALUES : OPT_EXACT_MAX;
    if (d <= distinct_max && (i128)hi - (i128)lo + 1 == (i128)d) {
        out->form = ORC_FORM_RANGE; /* dense(): the range is exact (:595-604) */
    } else if (d <= OPT_EXACT_MAX) {
        out->form = ORC_FORM_EXACT;
        *exact_set = sorted;
        *exact_n = d;
        sorted = NULL;
    } else if ((uint64_t)rows <= OPT_BLOOM_MAX_ITEMS) {
        /* bloom() (filter.rs:606-621): sized for every kept row */
        int64_t bytes = orc_bloom_bytes_for((uint64_t)rows, OPT_BLOOM_FPP);
        if (bytes > OPT_BLOOM_MAX_BYTES) bytes = OPT_BLOOM_MAX_BYTES;
        /* with_bytes rounds up to whole blocks (bloom.rs:115-121) */
        bytes = ((bytes + BLOCK_BYTES - 1) / BLOCK_BYTES) * BLOCK_BYTES;
        if (orc_bloom_expected_fpp(bytes, (uint64_t)rows) <= OPT_BLOOM_MAX_FPP) {
            uint64_t *h = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)rows);
            orc_int_hashes(kept, rows, 8, h);
            memset(bloom_words, 0, (size_t)bytes);
            orc_bloom_insert(bloom_words, bytes, h, rows);
            free(h);
            out->form = ORC_FORM_BLOOM;
            out->bloom_bytes = bytes;
        } else {
            out->form = ORC_FORM_RANGE;
        }
    } else {
        out->form = ORC_FORM_RANGE;
    }
    free(sorted);
    free(kept);
}

void orc_key_filter_eval(const orc_key_filter *f, const uint32_t *bloom_words,
                         const int64_t *exact_set, int64_t exact_n, const int64_t *keys,
                         const uint8_t *valid, int64_t n, uint8_t *out) {
    for (int64_t i = 0; i < n; i++) {
        int v = !valid || valid[i];
        int pass;
        if (f->form == ORC_FORM_EMPTY) {
            /* filter.rs:780-785: an empty producer passes only NULLs it let pass */
            pass = !v && f->nulls_pass;
            out[i] = (uint8_t)pass;
            continue;
        }
        pass = v && (!f->has_range || (keys[i] >= f->lo && keys[i] <= f->hi));
        if (pass && f->form == ORC_FORM_EXACT)
            pass = bsearch(&keys[i], exact_set, (size_t)exact_n, sizeof(int64_t), cmp_i64) != NULL;
        if (pass && f->form == ORC_FORM_BLOOM) {
            uint64_t h = orc_xxh64_fixed((uint64_t)keys[i], 0, 8);
            uint8_t hit;
            orc_bloom_check(bloom_words, f->bloom_bytes, &h, 1, &hit);
            pass = hit;
        }
        if (!v && f->nulls_pass) pass = 1;
        out[i] = (uint8_t)pass;
    }
}

/* ---- hash join ----------------------------------------------------------- */
#define NO_MATCH 0xFFFFFFFFu
#define SALT_MASK (0xFFFFULL << 48)

/* rows/layout.rs:615 (eq) for fixed-width keys: values compare as their
 * encoded words; NULL equals NULL only under a validity bit (null-safe). */
static int keys_eq(const orc_col *a, int64_t i, const orc_col *b, int64_t j, int nkeys) {
    for (int c = 0; c < nkeys; c++) {
        int va = col_valid(&a[c], i), vb = col_valid(&b[c], j);
        if (va != vb) return 0;
        if (!va) continue;
        uint64_t wa[2], wb[2];
        value_words(&a[c], i, wa);
        value_words(&b[c], j, wb);
        if (wa[0] != wb[0] || wa[1] != wb[1]) return 0;
    }
    return 1;
}

/* A row can match only when every `=` key is valid (join/keys.rs:17-19). */
static int row_matchable(const orc_col *k, int64_t i, int nkeys, const int32_t *null_safe) {
    for (int c = 0; c < nkeys; c++)
        if (!null_safe[c] && !col_valid(&k[c], i)) return 0;
    return 1;
}

/* rows/index.rs:137-142 */
static uint64_t salted_slots(uint64_t n) {
    uint64_t want = n + (n + 3) / 4, s = 1;
    while (s < want) s <<= 1;
    return s;
}

typedef struct {
    int64_t *rows;   /* arena row -> input build row */
    int64_t n;
    uint64_t *slots; /* salted directory (rows/index.rs:1-32) */
    uint64_t mask;
    uint32_t *next;  /* newest-first chains of equal keys */
    uint64_t *h;
} orc_part;

typedef struct {
    int64_t *p, *b;
    int64_t n, cap;
} pairs_t;
static void push_pair(pairs_t *o, int64_t p, int64_t b) {
    if (o->n == o->cap) {
        o->cap = o->cap ? o->cap * 2 : 1024;
        o->p = (int64_t *)realloc(o->p, sizeof(int64_t) * (size_t)o->cap);
        o->b = (int64_t *)realloc(o->b, sizeof(int64_t) * (size_t)o->cap);
    }
    o->p[o->n] = p;
    o->b[o->n] = b;
    o->n++;
}

/* One operand of a filter comparison for the pair (probe row p, build row
 * b): 0 when NULL. */
static int filter_operand(const orc_operand *o, int64_t p, int64_t b, int64_t *iv, double *fv) {
    if (o->side == ORC_SIDE_CONST) {
        *iv = o->i64;
        *fv = o->is_float ? o->f64 : (double)o->i64;
        return 1;
    }
    int64_t r = o->side == ORC_SIDE_PROBE ? p : b;
    if (o->col.valid && !o->col.valid[r]) return 0;
    if (o->col.width == 4) {
        int32_t v;
        memcpy(&v, (const uint8_t *)o->col.data + 4 * r, 4);
        *iv = v;
        *fv = (double)v;
    } else if (o->col.is_float) {
        memcpy(fv, (const uint8_t *)o->col.data + 8 * r, 8);
        *iv = 0;
    } else {
        memcpy(iv, (const uint8_t *)o->col.data + 8 * r, 8);
        *fv = (double)*iv;
    }
    return 1;
}
/* Spark's double order (aggregate/accumulator/helpers.rs:498): NaN equals
 * NaN and is above everything, -0.0 equals 0.0: -1, 0, 1. */
static int spark_cmp(double a, double b) {
    int an = a != a, bn = b != b;
    if (an || bn) return an == bn ? 0 : an ? 1 : -1;
    return a < b ? -1 : a > b ? 1 : 0;
}
static int cmp_holds(int op, int c) {
    switch (op) {
    case 0: return c == 0;
    case 1: return c != 0;
    case 2: return c < 0;
    case 3: return c <= 0;
    case 4: return c > 0;
    default: return c >= 0;
    }
}
static int filter_true(const orc_filter *f, int64_t p, int64_t b) {
    for (int t = 0; t < f->n; t++) {
        const orc_term *T = &f->t[t];
        int64_t li, ri;
        double lf, rf;
        if (!filter_operand(&T->l, p, b, &li, &lf) || !filter_operand(&T->r, p, b, &ri, &rf)) return 0;
        int as_float = (T->l.side == ORC_SIDE_CONST ? T->l.is_float : T->l.col.is_float) ||
                       (T->r.side == ORC_SIDE_CONST ? T->r.is_float : T->r.col.is_float);
        int c = as_float ? spark_cmp(lf, rf) : (li < ri ? -1 : li > ri ? 1 : 0);
        if (!cmp_holds(T->op, c)) return 0;
    }
    return 1;
}

int64_t orc_hash_join(int32_t jt, const orc_col *bk, int64_t nb, const orc_col *pk, int64_t np,
                      int32_t nkeys, const int32_t *null_safe, int32_t single_match,
                      uint64_t seed, int32_t radix, int64_t **out_probe, int64_t **out_build) {
    return orc_hash_join_filtered(jt, bk, nb, pk, np, nkeys, null_safe, single_match, seed, radix, NULL,
                                  out_probe, out_build);
}

int64_t orc_hash_join_filtered(int32_t jt, const orc_col *bk, int64_t nb, const orc_col *pk, int64_t np,
                               int32_t nkeys, const int32_t *null_safe, int32_t single_match,
                               uint64_t seed, int32_t radix, const orc_filter *filter, int64_t **out_probe,
                               int64_t **out_build) {
    if (radix < 3) radix = 3;
    if (radix > 6) radix = 6;
    int nparts = 1 << radix;
    int32_t null_bit[16];
    for (int c = 0; c < nkeys; c++) null_bit[c] = null_safe[c];
    uint64_t *bh = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(nb > 0 ? nb : 1));
    uint64_t *ph = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(np > 0 ? np : 1));
    orc_row_hash(bk, nkeys, null_bit, nb, bh);
    orc_row_hash(pk, nkeys, null_bit, np, ph);
    int keep_null_build = jt == ORC_RIGHT_ANTI || jt == ORC_RIGHT_OUTER || jt == ORC_FULL_OUTER;
    int builds_preserved = jt == ORC_RIGHT_SEMI || keep_null_build;
    /* BuildSink::sink (join/build.rs:1225-1335): rows into level-0
     * partitions by the top radix bits of h; a kept NULL-key row takes the
     * null_spread hash (build.rs:470-475) and is never indexed. */
    orc_part *parts = (orc_part *)calloc((size_t)nparts, sizeof(orc_part));
    int64_t *part_of = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nb > 0 ? nb : 1));
    uint8_t *indexed = (uint8_t *)malloc((size_t)(nb > 0 ? nb : 1));
    int any_null_build = 0;
    uint64_t null_seq = 0;
    for (int64_t i = 0; i < nb; i++) {
        int ok = row_matchable(bk, i, nkeys, null_safe);
        indexed[i] = (uint8_t)ok;
        if (!ok) any_null_build = 1;
        if (!ok && !keep_null_build) {
            part_of[i] = -1;
            continue;
        }
        uint64_t h = ok ? bh[i] : orc_null_spread(null_seq++);
        bh[i] = h;
        int p = orc_partition(h, 0, radix, seed);
        part_of[i] = p;
        parts[p].n++;
    }
    for (int p = 0; p < nparts; p++) {
        parts[p].rows = (int64_t *)malloc(sizeof(int64_t) * (size_t)(parts[p].n + 1));
        parts[p].next = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(parts[p].n + 1));
        parts[p].n = 0;
    }
    int64_t *arena_id = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nb > 0 ? nb : 1));
    for (int64_t i = 0; i < nb; i++) {
        if (part_of[i] < 0) continue;
        orc_part *P = &parts[part_of[i]];
        arena_id[i] = P->n;
        P->rows[P->n++] = i;
    }
    /* JoinIndex::build_expecting (rows/index.rs:211-283), salted form */
    for (int p = 0; p < nparts; p++) {
        orc_part *P = &parts[p];
        uint64_t len = salted_slots(P->n > 0 ? (uint64_t)P->n : 1);
        P->slots = (uint64_t *)calloc((size_t)len, sizeof(uint64_t));
        P->mask = len - 1;
        for (int64_t id = 0; id < P->n; id++) {
            P->next[id] = NO_MATCH;
            int64_t r = P->rows[id];
            if (!indexed[r]) continue;
            uint64_t g = orc_finalize(bh[r], seed);
            uint64_t salt = g & SALT_MASK;
            uint64_t slot = salt | ((uint64_t)id + 1);
            uint64_t i = g & P->mask;
            for (;;) {
                uint64_t s = P->slots[i];
                if (s == 0) {
                    P->slots[i] = slot;
                    break;
                }
                if ((s & SALT_MASK) == salt) {
                    uint32_t o = (uint32_t)(s & 0xFFFFFFFFULL) - 1;
                    if (keys_eq(bk, r, bk, P->rows[o], nkeys)) {
                        P->next[id] = o;
                        P->slots[i] = slot;
                        break;
                    }
                }
                i = (i + 1) & P->mask;
            }
        }
    }
    uint8_t *bmark = (uint8_t *)calloc((size_t)(nb > 0 ? nb : 1), 1);
    pairs_t out = {0};
    /* Cursor::new/next/pairs (join/probe.rs:126-502) and tails (:532-606) */
    for (int64_t i = 0; i < np; i++) {
        int matched = 0;
        if (row_matchable(pk, i, nkeys, null_safe) && nb > 0) {
            int p = orc_partition(ph[i], 0, radix, seed);
            orc_part *P = &parts[p];
            uint64_t g = orc_finalize(ph[i], seed);
            uint64_t salt = g & SALT_MASK;
            uint64_t s_i = g & P->mask;
            uint32_t head = NO_MATCH;
            /* JoinIndex::lookup (rows/index.rs:375-448) */
            for (;;) {
                uint64_t s = P->slots[s_i];
                if (s == 0) break;
                if ((s & SALT_MASK) == salt) {
                    uint32_t o = (uint32_t)(s & 0xFFFFFFFFULL) - 1;
                    if (keys_eq(pk, i, bk, P->rows[o], nkeys)) {
                        head = o;
                        break;
                    }
                }
                s_i = (s_i + 1) & P->mask;
            }
            for (uint32_t o = head; o != NO_MATCH; o = P->next[o]) {
                int64_t r = P->rows[o];
                /* a pair counts only where the filter is TRUE (join/probe.rs:425-436) */
                if (filter && !filter_true(filter, i, r)) continue;
                matched++;
                if (builds_preserved) bmark[r] = 1;
                if (jt == ORC_INNER || jt == ORC_LEFT_OUTER || jt == ORC_RIGHT_OUTER ||
                    jt == ORC_FULL_OUTER)
                    push_pair(&out, i, r);
            }
        }
        if (single_match && jt == ORC_LEFT_OUTER && matched > 1) {
            free(out.p);
            free(out.b);
            out.n = -2;
            goto done;
        }
        switch (jt) {
        case ORC_LEFT_OUTER:
        case ORC_FULL_OUTER:
            if (!matched) push_pair(&out, i, -1);
            break;
        case ORC_LEFT_SEMI:
            if (matched) push_pair(&out, i, -1);
            break;
        case ORC_LEFT_ANTI:
            if (!matched) push_pair(&out, i, -1);
            break;
        case ORC_NULL_AWARE_ANTI: {
            /* join/mod.rs:30-34 */
            int keep = nb == 0 || (!any_null_build && row_matchable(pk, i, nkeys, null_safe) &&
                                   !matched);
            if (keep) push_pair(&out, i, -1);
            break;
        }
        case ORC_EXISTENCE:
            push_pair(&out, i, matched ? 1 : 0);
            break;
        default:
            break;
        }
    }
    /* emit_build (join/probe.rs:610-): build rows by their marks */
    if (builds_preserved) {
        for (int64_t r = 0; r < nb; r++) {
            if (part_of[r] < 0) continue;
            if (jt == ORC_RIGHT_SEMI && bmark[r]) push_pair(&out, -1, r);
            if ((jt == ORC_RIGHT_ANTI || jt == ORC_RIGHT_OUTER || jt == ORC_FULL_OUTER) &&
                !bmark[r])
                push_pair(&out, -1, r);
        }
    }
done:
    *out_probe = out.p;
    *out_build = out.b;
    for (int p = 0; p < nparts; p++) {
        free(parts[p].rows);
        free(parts[p].next);
        free(parts[p].slots);
    }
    free(parts);
    free(part_of);
    free(indexed);
    free(arena_id);
    free(bmark);
    free(bh);
    free(ph);
    return out.n;
}

void orc_free(void *p) { free(p); }

/* ---- grouped aggregate ---------------------------------------------------- */
static i128 pow10_i128(int p) {
    i128 v = 1;
    for (int i = 0; i < p && i < 38; i++) v *= 10;
    return v;
}

/* helpers.rs:498 float_lt: NaN is the largest and equals itself */
static int float_lt(double a, double b) { return !isnan(a) && (isnan(b) || a < b); }

/* helpers.rs:539-590 (avg_decimal, digit loop) */
static int avg_decimal_slow(i128 sum, int ss, int64_t count, int p, int s, i128 *out) {
    int negative = (sum < 0) != (count < 0);
    u128 a = sum < 0 ? (u128)(-sum) : (u128)sum;
    u128 b = (u128)(count < 0 ? -(i128)count : (i128)count);
    u128 in = a / b, rem = a % b;
    int nfrac = 39 - ss;
    uint8_t frac[40];
    for (int i = 0; i < nfrac; i++) {
        rem *= 10;
        frac[i] = (uint8_t)(rem / b);
        rem %= b;
    }
    rem *= 10;
    uint8_t rd = (uint8_t)(rem / b);
    if (rd >= 5) {
        /* round_up: carry through the fraction digits */
        int i = nfrac - 1, carry = 1;
        while (i >= 0 && carry) {
            if (frac[i] == 9) frac[i] = 0;
            else {
                frac[i]++;
                carry = 0;
            }
            i--;
        }
        if (carry) in += 1;
    }
    int keep = s - ss;
    if (keep < 0) keep = 0;
    int up = keep < nfrac && frac[keep] >= 5;
    u128 v = in;
    const u128 lim = ((u128)1) << 126;
    for (int i = 0; i < keep; i++) {
        if (v > lim / 10) return 0;
        v = v * 10 + frac[i];
    }
    v += (u128)up;
    if (v >= (u128)pow10_i128(p)) return 0;
    *out = negative ? -(i128)v : (i128)v;
    return 1;
}

/* helpers.rs:595-610 (avg_fast), falling back to the digit loop */
static int avg_decimal(i128 sum, int ss, int64_t count, int p, int s, i128 *out) {
    if (count == 0) return 0;
    if (s <= 19 && s >= ss) {
        u128 mag = sum < 0 ? (u128)(-sum) : (u128)sum;
        u128 mul = (u128)pow10_i128(s - ss);
        if (mul == 0 || mag <= (~(u128)0) / mul) {
            u128 n = mag * mul;
            u128 d = (u128)(count < 0 ? -(i128)count : (i128)count);
            u128 q = n / d, r = n % d;
            q += (u128)(r >= d - r);
            if (q >= (u128)pow10_i128(p)) return 0;
            *out = ((sum < 0) != (count < 0)) ? -(i128)q : (i128)q;
            return 1;
        }
    }
    return avg_decimal_slow(sum, ss, count, p, s, out);
}

int32_t orc_avg_decimal(int64_t sum_lo, int64_t sum_hi, int32_t sum_scale, int64_t count,
                        int32_t p, int32_t s, uint64_t *out_lo, int64_t *out_hi) {
    i128 sum = (i128)(((u128)(uint64_t)sum_hi << 64) | (uint64_t)sum_lo);
    i128 v;
    if (!avg_decimal(sum, sum_scale, count, p, s, &v)) return 0;
    *out_lo = (uint64_t)v;
    *out_hi = (int64_t)(v >> 64);
    return 1;
}

typedef struct {
    i128 isum;       /* SUM int / SUM dec / AVG dec */
    double fseq;     /* sequential += (accumulator/fold.rs:401-426) */
    double fs, fc;   /* Neumaier compensated sum */
    int64_t count;
    i128 imin, imax;  /* MinMax holds Values::Int(i128) (aggregate/accumulator.rs:238-248) */
    double fmin, fmax;
    uint8_t seen, overflow;
} acc_t;

static int64_t value_i64(const orc_value_col *c, int64_t i) {
    if (c->type == ORC_T_I32) return ((const int32_t *)c->data)[i];
    return ((const int64_t *)c->data)[i];
}
static i128 value_i128(const orc_value_col *c, int64_t i) {
    if (c->type == ORC_T_DEC128) {
        const uint64_t *w = (const uint64_t *)c->data + 2 * i;
        return (i128)(((u128)w[1] << 64) | w[0]);
    }
    return (i128)value_i64(c, i);
}

int64_t orc_hash_aggregate(const void *key, const uint8_t *key_valid, int32_t key_width,
                           int64_t n, const orc_value_col *cols, int32_t ncols,
                           const orc_agg_expr *exprs, int32_t nexprs, int32_t ansi,
                           int64_t **out_keys, uint8_t **out_key_valid, orc_agg_out *outs) {
    (void)ncols;
    /* RowTable find-or-insert (aggregate/rowtable/probe.rs:149-214): an
     * open-addressing table over g = fin(h ^ seed) of the row layout's h,
     * groups numbered in first-seen order; a NULL key is one group. */
    orc_col kc = {key, key_valid, key_width, 0};
    int32_t nb = 1;
    uint64_t *h = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(n > 0 ? n : 1));
    orc_row_hash(&kc, 1, &nb, n, h);
    uint64_t cap = 1024;
    while (cap < (uint64_t)n * 2) cap <<= 1;
    int64_t *slot = (int64_t *)malloc(sizeof(int64_t) * (size_t)cap);
    for (uint64_t i = 0; i < cap; i++) slot[i] = -1;
    int64_t *gid = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
    int64_t *first = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
    int64_t ng = 0;
    for (int64_t i = 0; i < n; i++) {
        uint64_t g = orc_finalize(h[i], 0x5EEDULL);
        uint64_t s = g & (cap - 1);
        for (;;) {
            if (slot[s] < 0) {
                slot[s] = ng;
                first[ng] = i;
                gid[i] = ng++;
                break;
            }
            if (keys_eq(&kc, i, &kc, first[slot[s]], 1)) {
                gid[i] = slot[s];
                break;
            }
            s = (s + 1) & (cap - 1);
        }
    }
    *out_keys = (int64_t *)malloc(sizeof(int64_t) * (size_t)(ng > 0 ? ng : 1));
    *out_key_valid = (uint8_t *)malloc((size_t)(ng > 0 ? ng : 1));
    for (int64_t gi = 0; gi < ng; gi++) {
        int64_t r = first[gi];
        int v = !key_valid || key_valid[r];
        (*out_key_valid)[gi] = (uint8_t)v;
        (*out_keys)[gi] = !v ? 0
                          : key_width == 4 ? (int64_t)((const int32_t *)key)[r]
                                           : ((const int64_t *)key)[r];
    }
    int64_t status = ng;
    acc_t *acc = (acc_t *)malloc(sizeof(acc_t) * (size_t)(ng > 0 ? ng : 1));
    for (int e = 0; e < nexprs && status >= 0; e++) {
        const orc_agg_expr *x = &exprs[e];
        const orc_value_col *c = x->func == ORC_COUNT_STAR ? NULL : &cols[x->col];
        memset(acc, 0, sizeof(acc_t) * (size_t)(ng > 0 ? ng : 1));
        int is_float = c && c->type == ORC_T_F64;
        int is_dec = c && (c->type == ORC_T_DEC64 || c->type == ORC_T_DEC128);
        int rp = 0, rs = 0;
        if (is_dec && x->func == ORC_SUM) {
            rp = c->precision + 10 < 38 ? c->precision + 10 : 38;
            rs = c->scale;
        }
        if (is_dec && x->func == ORC_AVG) {
            rp = c->precision + 4 < 38 ? c->precision + 4 : 38;
            rs = c->scale + 4 < 38 ? c->scale + 4 : 38;
        }
        /* Accumulator::update / fold (accumulator/fold.rs) */
        for (int64_t i = 0; i < n; i++) {
            acc_t *a = &acc[gid[i]];
            if (x->func == ORC_COUNT_STAR) {
                a->count++;
                continue;
            }
            if (c->valid && !c->valid[i]) continue;
            a->count++;
            if (is_float) {
                double v = ((const double *)c->data)[i];
                if (!a->seen) {
                    a->fmin = a->fmax = v;
                } else {
                    if (float_lt(v, a->fmin)) a->fmin = v;
                    if (float_lt(a->fmax, v)) a->fmax = v;
                }
                a->fseq += v;
                double t = a->fs + v;
                if (fabs(a->fs) >= fabs(v)) a->fc += (a->fs - t) + v;
                else a->fc += (v - t) + a->fs;
                a->fs = t;
            } else {
                i128 v = value_i128(c, i);
                if (!a->seen) {
                    a->imin = a->imax = v;
                } else {
                    if (v < a->imin) a->imin = v;
                    if (v > a->imax) a->imax = v;
                }
                if (!is_dec && x->func == ORC_SUM) {
                    /* SumInt: ANSI raises on overflow, else wraps */
                    int64_t cur = (int64_t)a->isum, r;
                    if (__builtin_add_overflow(cur, (int64_t)v, &r)) {
                        if (ansi) status = -3;
                        r = (int64_t)((uint64_t)cur + (uint64_t)(int64_t)v);
                    }
                    a->isum = r;
                } else {
                    a->isum += v;
                    if (is_dec && x->func == ORC_SUM) {
                        i128 lim = pow10_i128(rp);
                        if (a->isum >= lim || a->isum <= -lim) a->overflow = 1; /* sticky */
                    }
                }
                /* AVG int reads its values as doubles (result type double) */
                a->fseq += (double)(int64_t)v;
            }
            a->seen = 1;
        }
        orc_agg_out *o = &outs[e];
        size_t m = (size_t)(ng > 0 ? ng : 1);
        o->i64 = (int64_t *)calloc(m, 8);
        o->f64 = (double *)calloc(m, 8);
        o->f64_seq = (double *)calloc(m, 8);
        o->lo = (uint64_t *)calloc(m, 8);
        o->hi = (int64_t *)calloc(m, 8);
        o->valid = (uint8_t *)calloc(m, 1);
        for (int64_t gi = 0; gi < ng; gi++) {
            acc_t *a = &acc[gi];
            switch (x->func) {
            case ORC_COUNT_STAR:
            case ORC_COUNT:
                o->i64[gi] = a->count;
                o->valid[gi] = 1;
                break;
            case ORC_SUM:
                if (!a->seen) break;
                if (is_float) {
                    o->f64[gi] = a->fs + a->fc;
                    o->f64_seq[gi] = a->fseq;
                    o->valid[gi] = 1;
                } else if (is_dec) {
                    if (a->overflow) {
                        if (ansi) status = -3;
                        break;
                    }
                    o->lo[gi] = (uint64_t)a->isum;
                    o->hi[gi] = (int64_t)(a->isum >> 64);
                    o->valid[gi] = 1;
                } else {
                    o->i64[gi] = (int64_t)a->isum;
                    o->valid[gi] = 1;
                }
                break;
            case ORC_MIN:
            case ORC_MAX:
                if (!a->seen) break;
                if (is_float) {
                    o->f64[gi] = x->func == ORC_MIN ? a->fmin : a->fmax;
                } else {
                    const i128 m = x->func == ORC_MIN ? a->imin : a->imax;
                    o->i64[gi] = (int64_t)m;
                    o->lo[gi] = (uint64_t)m;
                    o->hi[gi] = (int64_t)(m >> 64);
                }
                o->valid[gi] = 1;
                break;
            case ORC_AVG:
                if (!a->seen) break;
                if (is_float) {
                    o->f64[gi] = (a->fs + a->fc) / (double)a->count;
                    o->f64_seq[gi] = a->fseq / (double)a->count;
                    o->valid[gi] = 1;
                } else if (is_dec) {
                    i128 v;
                    if (avg_decimal(a->isum, c->scale, a->count, rp, rs, &v)) {
                        o->lo[gi] = (uint64_t)v;
                        o->hi[gi] = (int64_t)(v >> 64);
                        o->valid[gi] = 1;
                    } else if (ansi) {
                        status = -3;
                    }
                } else {
                    o->f64[gi] = a->fseq / (double)a->count;
                    o->f64_seq[gi] = o->f64[gi];
                    o->valid[gi] = 1;
                }
                break;
            default:
                break;
            }
        }
    }
    free(acc);
    free(h);
    free(slot);
    free(gid);
    free(first);
    return status;
}

/* ---- synthetic data --------------------------------------------------------
 * Counter-based SplitMix64: the value of (seed, column, row) is the
 * SplitMix64 output at step row+1 of a stream whose start is the finalizer
 * of (seed, column). The device generators compute the same function. */
static uint64_t fmix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
uint64_t orc_rand(uint64_t seed, uint32_t column, uint64_t row) {
    uint64_t base = fmix64(seed ^ fmix64((uint64_t)column + 0x632BE59BD9B4E019ULL));
    return fmix64(base + (row + 1) * 0x9E3779B97F4A7C15ULL);
}
int64_t orc_rand_range(uint64_t seed, uint32_t column, uint64_t row, int64_t lo, int64_t hi) {
    uint64_t span = (uint64_t)(hi - lo) + 1;
    uint64_t x = orc_rand(seed, column, row);
    return lo + (int64_t)(uint64_t)(((u128)x * span) >> 64);
}
double orc_rand_unit(uint64_t seed, uint32_t column, uint64_t row) {
    return (double)(orc_rand(seed, column, row) >> 11) * 0x1.0p-53;
}
uint64_t orc_permute(uint64_t seed, uint64_t n, uint64_t i) {
    int bits = 2;
    while ((1ULL << bits) < n) bits += 2;
    int half = bits / 2;
    uint64_t hmask = (1ULL << half) - 1;
    uint64_t x = i;
    do {
        uint64_t l = x >> half, r = x & hmask;
        for (uint32_t round = 0; round < 4; round++) {
            uint64_t f = orc_rand(seed, 0x70000000u + round, r) & hmask;
            uint64_t nl = r;
            r = l ^ f;
            l = nl;
        }
        x = (l << half) | r;
    } while (x >= n);
    return x;
}
void orc_zipf_cdf(double s, int64_t n, double *cdf) {
    double acc = 0.0;
    for (int64_t k = 1; k <= n; k++) {
        acc += pow((double)k, -s);
        cdf[k - 1] = acc;
    }
    for (int64_t k = 0; k < n; k++) cdf[k] /= acc;
    cdf[n - 1] = 1.0;
}
int64_t orc_zipf_rank(const double *cdf, int64_t n, double u) {
    int64_t lo = 0, hi = n - 1;
    while (lo < hi) {
        int64_t mid = lo + (hi - lo) / 2;
        if (cdf[mid] > u) hi = mid;
        else lo = mid + 1;
    }
    return lo;
}
