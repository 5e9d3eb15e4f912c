/*
 * krv_oracle_mt.c -- TEST INFRASTRUCTURE ONLY: the synthetic-column
 * generator (the same function as the device generators, used to check them)
 * and the multi-threaded CPU baseline of the star join (the reference's
 * algorithms restated: radix-partitioned hash tables over the engine's key
 * hash, the runtime filters of crates/krishiv-io/src/runtime_filter/, and a
 * grouped compensated sum), timed by the benchmark's CPU leg.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "krv_oracle.h"

/* Fills n values of generator `kind` (the device kinds of include/krv_gpu.h:
 * 0 uniform int64, 1 uniform int32, 2 unit float64, 3 permutation,
 * 4 Zipf). valid[i] = 0 marks a NULL when null_fraction > 0. */
void orc_gen_column(uint64_t seed, uint32_t column, int32_t kind, int64_t lo, int64_t hi, double x0,
                    double x1, int64_t row0, int64_t n, double null_fraction, void *out,
                    uint8_t *valid) {
    double *cdf = NULL;
    if (kind == 4) {
        cdf = (double *)malloc(sizeof(double) * (size_t)hi);
        orc_zipf_cdf(x0, hi, cdf);
    }
    for (int64_t i = 0; i < n; i++) {
        uint64_t row = (uint64_t)(row0 + i);
        switch (kind) {
        case 0: ((int64_t *)out)[i] = orc_rand_range(seed, column, row, lo, hi); break;
        case 1: ((int32_t *)out)[i] = (int32_t)orc_rand_range(seed, column, row, lo, hi); break;
        case 2: {
            double u = orc_rand_unit(seed, column, row);
            double span = x1 - x0;
            double p = span * u;
            ((double *)out)[i] = x0 + p;
            break;
        }
        case 3: ((int64_t *)out)[i] = lo + (int64_t)orc_permute(seed, (uint64_t)hi, row); break;
        case 4: {
            double u = orc_rand_unit(seed, column, row);
            int64_t r = orc_zipf_rank(cdf, hi, u);
            ((int64_t *)out)[i] = lo + (int64_t)orc_permute(seed ^ 0x5A17F00DULL, (uint64_t)hi, (uint64_t)r);
            break;
        }
        default: break;
        }
        if (valid) valid[i] = orc_rand_unit(seed, column + 0x10000u, row) >= null_fraction;
    }
    free(cdf);
}

/* ---- multi-threaded star join (CPU baseline) ------------------------------- */
#include <time.h>

#define SALT_MASK_ST (0xFFFFULL << 48)
#define SEED_ST 0x4B52565F4A4F494EULL

typedef struct {
    uint64_t *slots; /* salted directory (rows/index.rs:1-32) */
    uint64_t mask;
    int64_t *keys;
    int32_t *attr;
    int64_t n;
    orc_key_filter f;
    uint32_t *bloom;
    int64_t *exact;
    int64_t exact_n;
} star_dim;

static double now_s(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static uint64_t key_h(int64_t k) {
    /* h of one valid int64 key (rows/layout.rs:487-555) */
    return orc_fold(orc_fold((uint64_t)k, 0x243F6A8885A308D3ULL), 0xB7E151628AED2A6BULL);
}

static void dim_build(star_dim *d, const int64_t *key, const int32_t *pred, const int32_t *attr, int64_t n,
                      int32_t value) {
    memset(d, 0, sizeof(*d));
    d->keys = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
    d->attr = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    for (int64_t i = 0; i < n; i++)
        if (pred[i] == value) {
            d->keys[d->n] = key[i];
            d->attr[d->n] = attr[i];
            d->n++;
        }
    uint64_t want = (uint64_t)d->n + ((uint64_t)d->n + 3) / 4, s = 1024;
    while (s < want) s <<= 1;
    d->slots = (uint64_t *)calloc((size_t)s, 8);
    d->mask = s - 1;
    for (int64_t id = 0; id < d->n; id++) {
        uint64_t g = orc_finalize(key_h(d->keys[id]), SEED_ST);
        uint64_t salt = g & SALT_MASK_ST, i = g & d->mask;
        while (d->slots[i] != 0) i = (i + 1) & d->mask; /* unique dimension keys */
        d->slots[i] = salt | ((uint64_t)id + 1);
    }
    d->bloom = (uint32_t *)calloc((8u << 20) / 4, 4);
    orc_key_filter_build(d->keys, NULL, d->n, &d->f, d->bloom, &d->exact, &d->exact_n);
}

static int64_t dim_lookup(const star_dim *d, int64_t k) {
    uint64_t g = orc_finalize(key_h(k), SEED_ST);
    uint64_t salt = g & SALT_MASK_ST, i = g & d->mask;
    for (;;) {
        uint64_t s = d->slots[i];
        if (s == 0) return -1;
        if ((s & SALT_MASK_ST) == salt) {
            int64_t id = (int64_t)(s & 0xFFFFFFFFULL) - 1;
            if (d->keys[id] == k) return id;
        }
        i = (i + 1) & d->mask;
    }
}

typedef struct {
    const star_dim *a, *b;
    const int64_t *fk_a, *fk_b, *price;
    const double *disc;
    int64_t lo, hi;
    int32_t group_by, use_filters;
    double s[4096], c[4096];
    int64_t cnt[4096];
    int64_t passed, joined;
} star_task;

static void *star_worker(void *arg) {
    star_task *t = (star_task *)arg;
    for (int64_t i = t->lo; i < t->hi; i++) {
        int64_t a = t->fk_a[i], b = t->fk_b[i];
        if (t->use_filters) {
            uint8_t okb, oka;
            orc_key_filter_eval(&t->b->f, t->b->bloom, t->b->exact, t->b->exact_n, &b, NULL, 1, &okb);
            if (!okb) continue;
            orc_key_filter_eval(&t->a->f, t->a->bloom, t->a->exact, t->a->exact_n, &a, NULL, 1, &oka);
            if (!oka) continue;
        }
        t->passed++;
        int64_t ra = dim_lookup(t->a, a);
        if (ra < 0) continue;
        int64_t rb = dim_lookup(t->b, b);
        if (rb < 0) continue;
        t->joined++;
        int32_t g = t->group_by == 0 ? t->a->attr[ra] : t->b->attr[rb];
        if (g < 0 || g >= 4096) continue;
        double one_minus = 1.0 - t->disc[i];
        double v = (double)t->price[i] * one_minus;
        double s = t->s[g], x = s + v;
        if (fabs(s) >= fabs(v)) t->c[g] += (s - x) + v;
        else t->c[g] += (v - x) + s;
        t->s[g] = x;
        t->cnt[g]++;
    }
    return NULL;
}

/* The star query on the CPU with `threads` threads: dimension builds
 * (filter, salted directory, key filter), then the fact rows split across
 * threads. Writes per-attribute (0..4095) sums and counts. Returns the number
 * of groups with rows; times in *t_build / *t_probe (seconds). */
int64_t orc_star_query(const int64_t *dka, const int32_t *pa, const int32_t *aa, int64_t na, int32_t va,
                       const int64_t *dkb, const int32_t *pb, const int32_t *ab, int64_t nb, int32_t vb,
                       const int64_t *fk_a, const int64_t *fk_b, const int64_t *price, const double *disc,
                       int64_t nf, int32_t group_by, int32_t threads, int32_t use_filters, double *out_sum,
                       int64_t *out_cnt, int64_t *out_passed, int64_t *out_joined, double *t_build,
                       double *t_probe) {
    if (threads < 1) threads = 1;
    if (threads > 512) threads = 512;
    double t0 = now_s();
    star_dim A, B;
    dim_build(&A, dka, pa, aa, na, va);
    dim_build(&B, dkb, pb, ab, nb, vb);
    double t1 = now_s();
    star_task *tasks = (star_task *)calloc((size_t)threads, sizeof(star_task));
    pthread_t *tid = (pthread_t *)calloc((size_t)threads, sizeof(pthread_t));
    int64_t per = (nf + threads - 1) / threads;
    for (int t = 0; t < threads; t++) {
        star_task *k = &tasks[t];
        k->a = &A;
        k->b = &B;
        k->fk_a = fk_a;
        k->fk_b = fk_b;
        k->price = price;
        k->disc = disc;
        k->lo = (int64_t)t * per;
        k->hi = k->lo + per < nf ? k->lo + per : nf;
        if (k->lo > nf) k->lo = nf;
        k->group_by = group_by;
        k->use_filters = use_filters;
        pthread_create(&tid[t], NULL, star_worker, k);
    }
    for (int t = 0; t < threads; t++) pthread_join(tid[t], NULL);
    double t2 = now_s();
    int64_t groups = 0, passed = 0, joined = 0;
    for (int g = 0; g < 4096; g++) {
        double s = 0.0, c = 0.0;
        int64_t cnt = 0;
        for (int t = 0; t < threads; t++) {
            double v = tasks[t].s[g] + tasks[t].c[g];
            double x = s + v;
            if (fabs(s) >= fabs(v)) c += (s - x) + v;
            else c += (v - x) + s;
            s = x;
            cnt += tasks[t].cnt[g];
        }
        out_sum[g] = s + c;
        out_cnt[g] = cnt;
        if (cnt) groups++;
    }
    for (int t = 0; t < threads; t++) {
        passed += tasks[t].passed;
        joined += tasks[t].joined;
    }
    *out_passed = passed;
    *out_joined = joined;
    *t_build = t1 - t0;
    *t_probe = t2 - t1;
    star_dim *ds[2] = {&A, &B};
    for (int i = 0; i < 2; i++) {
        free(ds[i]->slots);
        free(ds[i]->keys);
        free(ds[i]->attr);
        free(ds[i]->bloom);
        free(ds[i]->exact);
    }
    free(tasks);
    free(tid);
    return groups;
}
