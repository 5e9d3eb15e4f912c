// aggregate.cu -- the grouped hash aggregate: COUNT(*), COUNT, SUM, MIN, MAX,
// AVG over int32/int64/decimal/float64 columns, grouped by one int32 or int64
// key, with Spark's result types, exact integer and decimal arithmetic and
// ANSI overflow errors.
//
// Reference: crates/krishiv-exec/src/aggregate/ (HashAggregate, sink.rs:181;
// result types, mod.rs:588-740; accumulators, accumulator.rs:212-590 and
// accumulator/fold.rs; decimal AVG, accumulator/helpers.rs:539-610).
//
// Device layout. A global table maps each key to a dense group id: `keys`
// (int64, empty = 0x8080...80) and `gids` (u32) of S = 2^k slots, probed
// linearly from the key's hash; group g's accumulators are one record of
// `rec` bytes at states + g * rec (rows, then per value column its non-NULL
// count, sum, min and max as needed). Group 0 is the NULL key and group 1 the
// key equal to the empty marker. In the shared-memory mode every CTA keeps a
// small table of (key, group id, record) for the keys it sees first (under
// Zipf keys, the heavy ones) and merges it into the global records at the end.
//
// Large batches take the partitioned path instead (count, split and
// partition kernels below): hot keys folded into per-CTA shared-memory
// records, every other row sorted into hash partitions and each partition's
// keys reduced in registers and merged once per chunk.
//
// Accumulation is exact and order-independent: counts and integer sums are
// integer adds (64-bit atomics in global memory, 32-bit limbs with carries in
// shared memory), decimal and int64 sums are 128-bit, float64 sums are
// double-double (TwoSum-compensated), MIN/MAX of floats use an
// order-preserving integer map with NaN largest.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <tuple>

#include "krv_device.cuh"
#include "ops.h"

namespace krv {

namespace {

constexpr long long kEmptyKey = (long long)0x8080808080808080ULL;
constexpr uint32_t kPending = 0xFFFFFFFFu;
constexpr uint32_t kOverflowGid = 0xFFFFFFFEu;
constexpr uint32_t kNullGid = 0, kMarkerGid = 1, kFirstGid = 2;
constexpr int kMaxValueCols = 16;

// F_WIDE: MIN/MAX of a decimal128 column of precision 19 to 38, kept in 16
// bytes (lo, hi) and updated by 128-bit compare-and-swap; such a plan runs
// the global-table kernels only.
// F_STR: MIN/MAX of a UTF-8 or binary column, whose values arrive as codes
// of a value dictionary; a record keeps the best code (-1: none yet),
// replaced by compare-and-swap after a byte-wise compare of the strings.
// Such a plan, too, runs the global-table kernels only.
enum : int32_t { F_SUM = 1, F_MIN = 2, F_MAX = 4, F_WIDE = 8, F_STR = 16 };

struct AggColDev {
    const void *data;
    const uint8_t *valid;
    int64_t voff;
    int32_t type;  // Type
    int32_t flags;
    int32_t off_count, off_sum, off_min, off_max;
    // F_STR: the value dictionary's strings (start, length per code; bytes)
    const long long *s_off;
    const int32_t *s_len;
    const uint8_t *s_heap;
};
struct AggPlanDev {
    AggColDev c[kMaxValueCols];
    int32_t ncols;
    int32_t rec;  // record bytes, a multiple of 16
    int32_t off_rows;
    int32_t pad;
};
struct KeyIn {
    const void *data;
    const uint8_t *valid;
    int64_t voff;
    int32_t width;  // 4 or 8
    int32_t pad;
};
struct TableDev {
    long long *keys;
    uint32_t *gids;
    uint64_t mask;
    uint8_t *states;
    long long *gkeys;
    unsigned long long *ngroups;
    unsigned long long limit;
    uint32_t *status;
};

__device__ __forceinline__ long long key_at(const KeyIn &k, int64_t i) {
    return k.width == 4 ? (long long)static_cast<const int32_t *>(k.data)[i]
                        : static_cast<const long long *>(k.data)[i];
}

// 128-bit compare-and-swap (atom.cas.b128) on the 16-byte aligned pair
// p[0] (low word), p[1] (high word): lo/hi in, the old value out.
__device__ __forceinline__ void cas128(unsigned long long *p, unsigned long long &lo, unsigned long long &hi,
                                       unsigned long long nlo, unsigned long long nhi) {
    asm volatile(
        "{\n\t.reg .b128 cmp, swp, old;\n\t"
        "mov.b128 cmp, {%0, %1};\n\t"
        "mov.b128 swp, {%3, %4};\n\t"
        "atom.cas.b128 old, [%2], cmp, swp;\n\t"
        "mov.b128 {%0, %1}, old;\n\t}"
        : "+l"(lo), "+l"(hi)
        : "l"(p), "l"(nlo), "l"(nhi)
        : "memory");
}
__device__ __forceinline__ bool i128_less(long long ahi, unsigned long long alo, long long bhi, unsigned long long blo) {
    return ahi < bhi || (ahi == bhi && alo < blo);
}
// MIN (or MAX) of the signed 128-bit value (vlo, vhi) into p: read the pair
// atomically (a compare-and-swap that changes nothing), then swap while the
// value is still better. Every failed swap saw a better value stored, so the
// loop ends; the bound is a guard only.
__device__ __forceinline__ void atomic_minmax_i128(unsigned long long *p, unsigned long long vlo, long long vhi,
                                                   bool is_max) {
    unsigned long long clo = 0, chi = 0;
    cas128(p, clo, chi, 0ull, 0ull);
    for (int it = 0; it < (1 << 20); it++) {
        const bool better = is_max ? i128_less((long long)chi, clo, vhi, vlo) : i128_less(vhi, vlo, (long long)chi, clo);
        if (!better) return;
        unsigned long long olo = clo, ohi = chi;
        cas128(p, olo, ohi, vlo, (unsigned long long)vhi);
        if (olo == clo && ohi == chi) return;
        clo = olo;
        chi = ohi;
    }
}
__device__ __forceinline__ void plain_minmax_i128(unsigned long long *p, unsigned long long vlo, long long vhi,
                                                  bool is_max) {
    const bool better = is_max ? i128_less((long long)p[1], p[0], vhi, vlo) : i128_less(vhi, vlo, (long long)p[1], p[0]);
    if (better) {
        p[0] = vlo;
        p[1] = (unsigned long long)vhi;
    }
}

// Byte-wise order of two dictionary strings (Spark orders strings and binary
// by their unsigned bytes, a prefix first).
__device__ __forceinline__ int str_cmp(const AggColDev &C, long long a, long long b) {
    const uint8_t *pa = C.s_heap + C.s_off[a], *pb = C.s_heap + C.s_off[b];
    const int la = C.s_len[a], lb = C.s_len[b];
    const int m = la < lb ? la : lb;
    for (int i = 0; i < m; i++)
        if (pa[i] != pb[i]) return pa[i] < pb[i] ? -1 : 1;
    return la < lb ? -1 : la > lb ? 1 : 0;
}
// MIN (or MAX) of string code `v` into the record's code slot: swap while
// the stored code's string is worse. Each failed swap saw a better stored
// value, so the loop ends; the bound is a guard only.
__device__ __forceinline__ void atomic_minmax_str(const AggColDev &C, uint8_t *slot, long long v, bool is_max) {
    unsigned long long *p = reinterpret_cast<unsigned long long *>(slot);
    long long cur = *reinterpret_cast<volatile long long *>(p);
    for (int it = 0; it < (1 << 20); it++) {
        if (cur == v) return;
        if (cur >= 0) {
            const int c = str_cmp(C, v, cur);
            if (is_max ? c <= 0 : c >= 0) return;
        }
        const long long old = (long long)atomicCAS(p, (unsigned long long)cur, (unsigned long long)v);
        if (old == cur) return;
        cur = old;
    }
}
__device__ __forceinline__ void plain_minmax_str(const AggColDev &C, uint8_t *slot, long long v, bool is_max) {
    long long *p = reinterpret_cast<long long *>(slot);
    if (*p < 0 || (is_max ? str_cmp(C, v, *p) > 0 : str_cmp(C, v, *p) < 0)) *p = v;
}

__device__ __forceinline__ void init_record(const AggPlanDev &P, uint8_t *r) {
    for (int b = 0; b < P.rec; b += 8) *reinterpret_cast<unsigned long long *>(r + b) = 0ull;
    for (int c = 0; c < P.ncols; c++) {
        const AggColDev &C = P.c[c];
        if (C.flags & F_STR) {
            if (C.flags & F_MIN) *reinterpret_cast<long long *>(r + C.off_min) = -1;
            if (C.flags & F_MAX) *reinterpret_cast<long long *>(r + C.off_max) = -1;
            continue;
        }
        if (C.flags & F_WIDE) {
            unsigned long long *mn = reinterpret_cast<unsigned long long *>(r + C.off_min);
            unsigned long long *mx = reinterpret_cast<unsigned long long *>(r + C.off_max);
            if (C.flags & F_MIN) mn[0] = ~0ull, mn[1] = (unsigned long long)LLONG_MAX;
            if (C.flags & F_MAX) mx[0] = 0ull, mx[1] = (unsigned long long)LLONG_MIN;
            continue;
        }
        if (C.flags & F_MIN) {
            if (C.type == (int)Type::I32 || C.type == (int)Type::Date32) *reinterpret_cast<int *>(r + C.off_min) = INT_MAX;
            else if (C.type == (int)Type::F64) *reinterpret_cast<unsigned long long *>(r + C.off_min) = ~0ull;
            else *reinterpret_cast<long long *>(r + C.off_min) = LLONG_MAX;
        }
        if (C.flags & F_MAX) {
            if (C.type == (int)Type::I32 || C.type == (int)Type::Date32) *reinterpret_cast<int *>(r + C.off_max) = INT_MIN;
            else if (C.type == (int)Type::F64) *reinterpret_cast<unsigned long long *>(r + C.off_max) = 0ull;
            else *reinterpret_cast<long long *>(r + C.off_max) = LLONG_MIN;
        }
    }
}

// Accumulator::update for one row (accumulator/fold.rs): NULL inputs are
// skipped; the row counts toward COUNT(*) regardless.
__device__ __forceinline__ void update_record(const AggPlanDev &P, uint8_t *r, int64_t i) {
    atomicAdd(reinterpret_cast<unsigned long long *>(r + P.off_rows), 1ull);
    for (int c = 0; c < P.ncols; c++) {
        const AggColDev &C = P.c[c];
        if (!bit_get(C.valid, C.voff, i)) continue;
        atomicAdd(reinterpret_cast<unsigned long long *>(r + C.off_count), 1ull);
        if (C.flags & F_STR) {
            const long long code = static_cast<const long long *>(C.data)[i];
            if (C.flags & F_MIN) atomic_minmax_str(C, r + C.off_min, code, false);
            if (C.flags & F_MAX) atomic_minmax_str(C, r + C.off_max, code, true);
            continue;
        }
        if (C.type == (int)Type::I32 || C.type == (int)Type::Date32) {
            const int v = static_cast<const int *>(C.data)[i];
            if (C.flags & F_SUM) atomicAdd(reinterpret_cast<unsigned long long *>(r + C.off_sum), (unsigned long long)(long long)v);
            if (C.flags & F_MIN) atomicMin(reinterpret_cast<int *>(r + C.off_min), v);
            if (C.flags & F_MAX) atomicMax(reinterpret_cast<int *>(r + C.off_max), v);
        } else if (C.type == (int)Type::F64) {
            const double v = static_cast<const double *>(C.data)[i];
            if (C.flags & F_SUM)
                atomic_add_dd(reinterpret_cast<double *>(r + C.off_sum), reinterpret_cast<double *>(r + C.off_sum + 8), v);
            if (C.flags & (F_MIN | F_MAX)) {
                const unsigned long long key = f64_order_key(v);
                if (C.flags & F_MIN) atomicMin(reinterpret_cast<unsigned long long *>(r + C.off_min), key);
                if (C.flags & F_MAX) atomicMax(reinterpret_cast<unsigned long long *>(r + C.off_max), key);
            }
        } else if (C.type == (int)Type::Dec128) {
            const long long *p = static_cast<const long long *>(C.data) + 2 * i;
            if (C.flags & F_SUM)
                atomic_add_i128(reinterpret_cast<unsigned long long *>(r + C.off_sum),
                                reinterpret_cast<long long *>(r + C.off_sum + 8), p[0], p[1]);
            if (C.flags & F_WIDE) {
                if (C.flags & F_MIN)
                    atomic_minmax_i128(reinterpret_cast<unsigned long long *>(r + C.off_min), p[0], p[1], false);
                if (C.flags & F_MAX)
                    atomic_minmax_i128(reinterpret_cast<unsigned long long *>(r + C.off_max), p[0], p[1], true);
            } else {
                // precision <= 18: the value is its low word
                if (C.flags & F_MIN) atomicMin(reinterpret_cast<long long *>(r + C.off_min), p[0]);
                if (C.flags & F_MAX) atomicMax(reinterpret_cast<long long *>(r + C.off_max), p[0]);
            }
        } else {  // I64, Dec64
            const long long v = static_cast<const long long *>(C.data)[i];
            if (C.flags & F_SUM)
                atomic_add_i128_from_i64(reinterpret_cast<unsigned long long *>(r + C.off_sum),
                                         reinterpret_cast<long long *>(r + C.off_sum + 8), v);
            if (C.flags & F_MIN) atomicMin(reinterpret_cast<long long *>(r + C.off_min), v);
            if (C.flags & F_MAX) atomicMax(reinterpret_cast<long long *>(r + C.off_max), v);
        }
    }
}

// update_record for a record only one thread touches at a time: plain
// arithmetic, the float64 sum compensated (TwoSum into hi, the error into lo).
__device__ __forceinline__ void update_record_plain(const AggPlanDev &P, uint8_t *r, int64_t i) {
    *reinterpret_cast<unsigned long long *>(r + P.off_rows) += 1ull;
    for (int c = 0; c < P.ncols; c++) {
        const AggColDev &C = P.c[c];
        if (!bit_get(C.valid, C.voff, i)) continue;
        *reinterpret_cast<unsigned long long *>(r + C.off_count) += 1ull;
        if (C.flags & F_STR) {
            const long long code = static_cast<const long long *>(C.data)[i];
            if (C.flags & F_MIN) plain_minmax_str(C, r + C.off_min, code, false);
            if (C.flags & F_MAX) plain_minmax_str(C, r + C.off_max, code, true);
            continue;
        }
        if (C.type == (int)Type::I32 || C.type == (int)Type::Date32) {
            const int v = static_cast<const int *>(C.data)[i];
            if (C.flags & F_SUM) *reinterpret_cast<long long *>(r + C.off_sum) += (long long)v;
            if (C.flags & F_MIN) {
                int *m = reinterpret_cast<int *>(r + C.off_min);
                *m = v < *m ? v : *m;
            }
            if (C.flags & F_MAX) {
                int *m = reinterpret_cast<int *>(r + C.off_max);
                *m = v > *m ? v : *m;
            }
        } else if (C.type == (int)Type::F64) {
            const double v = static_cast<const double *>(C.data)[i];
            if (C.flags & F_SUM) {
                double *hi = reinterpret_cast<double *>(r + C.off_sum), *lo = hi + 1;
                double sum, err;
                two_sum(*hi, v, sum, err);
                *hi = sum;
                *lo = __dadd_rn(*lo, err);
            }
            if (C.flags & (F_MIN | F_MAX)) {
                const unsigned long long key = f64_order_key(v);
                if (C.flags & F_MIN) {
                    unsigned long long *m = reinterpret_cast<unsigned long long *>(r + C.off_min);
                    *m = key < *m ? key : *m;
                }
                if (C.flags & F_MAX) {
                    unsigned long long *m = reinterpret_cast<unsigned long long *>(r + C.off_max);
                    *m = key > *m ? key : *m;
                }
            }
        } else if (C.type == (int)Type::Dec128) {
            const long long *p = static_cast<const long long *>(C.data) + 2 * i;
            if (C.flags & F_SUM) {
                unsigned long long *lo = reinterpret_cast<unsigned long long *>(r + C.off_sum);
                long long *hi = reinterpret_cast<long long *>(r + C.off_sum + 8);
                const unsigned long long old = *lo;
                *lo = old + (unsigned long long)p[0];
                *hi += p[1] + (long long)(*lo < old);
            }
            if (C.flags & F_WIDE) {
                if (C.flags & F_MIN) plain_minmax_i128(reinterpret_cast<unsigned long long *>(r + C.off_min), p[0], p[1], false);
                if (C.flags & F_MAX) plain_minmax_i128(reinterpret_cast<unsigned long long *>(r + C.off_max), p[0], p[1], true);
            } else {
                if (C.flags & F_MIN) {
                    long long *m = reinterpret_cast<long long *>(r + C.off_min);
                    *m = p[0] < *m ? p[0] : *m;
                }
                if (C.flags & F_MAX) {
                    long long *m = reinterpret_cast<long long *>(r + C.off_max);
                    *m = p[0] > *m ? p[0] : *m;
                }
            }
        } else {  // I64, Dec64
            const long long v = static_cast<const long long *>(C.data)[i];
            if (C.flags & F_SUM) {
                unsigned long long *lo = reinterpret_cast<unsigned long long *>(r + C.off_sum);
                long long *hi = reinterpret_cast<long long *>(r + C.off_sum + 8);
                const unsigned long long old = *lo;
                *lo = old + (unsigned long long)v;
                *hi += (v < 0 ? -1ll : 0ll) + (long long)(*lo < old);
            }
            if (C.flags & F_MIN) {
                long long *m = reinterpret_cast<long long *>(r + C.off_min);
                *m = v < *m ? v : *m;
            }
            if (C.flags & F_MAX) {
                long long *m = reinterpret_cast<long long *>(r + C.off_max);
                *m = v > *m ? v : *m;
            }
        }
    }
}

// Accumulator::merge (accumulator.rs:1159): folds the partial record `src`
// into `dst`.
__device__ __forceinline__ void merge_record(const AggPlanDev &P, uint8_t *dst, const uint8_t *src) {
    const unsigned long long rows = *reinterpret_cast<const unsigned long long *>(src + P.off_rows);
    if (!rows) return;
    atomicAdd(reinterpret_cast<unsigned long long *>(dst + P.off_rows), rows);
    for (int c = 0; c < P.ncols; c++) {
        const AggColDev &C = P.c[c];
        const unsigned long long cnt = *reinterpret_cast<const unsigned long long *>(src + C.off_count);
        if (!cnt) continue;
        atomicAdd(reinterpret_cast<unsigned long long *>(dst + C.off_count), cnt);
        if (C.flags & F_STR) {
            if (C.flags & F_MIN) atomic_minmax_str(C, dst + C.off_min, *reinterpret_cast<const long long *>(src + C.off_min), false);
            if (C.flags & F_MAX) atomic_minmax_str(C, dst + C.off_max, *reinterpret_cast<const long long *>(src + C.off_max), true);
            continue;
        }
        if (C.type == (int)Type::I32 || C.type == (int)Type::Date32) {
            if (C.flags & F_SUM)
                atomicAdd(reinterpret_cast<unsigned long long *>(dst + C.off_sum),
                          *reinterpret_cast<const unsigned long long *>(src + C.off_sum));
            if (C.flags & F_MIN) atomicMin(reinterpret_cast<int *>(dst + C.off_min), *reinterpret_cast<const int *>(src + C.off_min));
            if (C.flags & F_MAX) atomicMax(reinterpret_cast<int *>(dst + C.off_max), *reinterpret_cast<const int *>(src + C.off_max));
        } else if (C.type == (int)Type::F64) {
            if (C.flags & F_SUM)
                atomic_add_dd2(reinterpret_cast<double *>(dst + C.off_sum), reinterpret_cast<double *>(dst + C.off_sum + 8),
                               *reinterpret_cast<const double *>(src + C.off_sum),
                               *reinterpret_cast<const double *>(src + C.off_sum + 8));
            if (C.flags & F_MIN)
                atomicMin(reinterpret_cast<unsigned long long *>(dst + C.off_min),
                          *reinterpret_cast<const unsigned long long *>(src + C.off_min));
            if (C.flags & F_MAX)
                atomicMax(reinterpret_cast<unsigned long long *>(dst + C.off_max),
                          *reinterpret_cast<const unsigned long long *>(src + C.off_max));
        } else {
            if (C.flags & F_SUM)
                atomic_add_i128(reinterpret_cast<unsigned long long *>(dst + C.off_sum),
                                reinterpret_cast<long long *>(dst + C.off_sum + 8),
                                *reinterpret_cast<const long long *>(src + C.off_sum),
                                *reinterpret_cast<const long long *>(src + C.off_sum + 8));
            if (C.flags & F_WIDE) {
                if (C.flags & F_MIN) {
                    const long long *m = reinterpret_cast<const long long *>(src + C.off_min);
                    atomic_minmax_i128(reinterpret_cast<unsigned long long *>(dst + C.off_min), (unsigned long long)m[0], m[1], false);
                }
                if (C.flags & F_MAX) {
                    const long long *m = reinterpret_cast<const long long *>(src + C.off_max);
                    atomic_minmax_i128(reinterpret_cast<unsigned long long *>(dst + C.off_max), (unsigned long long)m[0], m[1], true);
                }
                continue;
            }
            if (C.flags & F_MIN)
                atomicMin(reinterpret_cast<long long *>(dst + C.off_min), *reinterpret_cast<const long long *>(src + C.off_min));
            if (C.flags & F_MAX)
                atomicMax(reinterpret_cast<long long *>(dst + C.off_max), *reinterpret_cast<const long long *>(src + C.off_max));
        }
    }
}

// A claimed slot's group id, published by its claimer right after the claim.
// The wait is bounded: past the limit the kernel reports ST_TIMEOUT.
__device__ __forceinline__ uint32_t wait_gid(const TableDev &T, uint64_t pos) {
    for (int it = 0; it < (1 << 22); it++) {
        const uint32_t g = *reinterpret_cast<volatile uint32_t *>(T.gids + pos);
        if (g != kPending) {
            __threadfence();
            return g;
        }
        __nanosleep(20);
    }
    atomicOr(T.status, ST_TIMEOUT);
    return kOverflowGid;
}

// The group of key k: found, or inserted with a fresh dense id. kOverflowGid
// when the table is past its load limit (the row is deferred to a bigger
// table).
__device__ uint32_t find_or_insert(const TableDev &T, const AggPlanDev &P, long long k) {
    uint64_t pos = hash_word((uint64_t)k) & T.mask;
    for (uint64_t p = 0; p <= T.mask; p++) {
        const long long cur = __ldcg(T.keys + pos);
        if (cur == k) return wait_gid(T, pos);
        if (cur == kEmptyKey) {
            if (__ldcg(T.ngroups) >= T.limit) return kOverflowGid;
            const long long old = (long long)atomicCAS(reinterpret_cast<unsigned long long *>(T.keys + pos),
                                                       (unsigned long long)kEmptyKey, (unsigned long long)k);
            if (old == kEmptyKey) {
                const uint32_t g = (uint32_t)atomicAdd(T.ngroups, 1ull);
                init_record(P, T.states + (size_t)g * P.rec);
                T.gkeys[g] = k;
                __threadfence();
                atomicExch(T.gids + pos, g);
                return g;
            }
            if (old == k) return wait_gid(T, pos);
        }
        pos = (pos + 1) & T.mask;
    }
    return kOverflowGid;
}

// The group of key k when the table has it, else kPending (a lookup only).
__device__ __forceinline__ uint32_t table_find(const TableDev &T, long long k) {
    uint64_t pos = hash_word((uint64_t)k) & T.mask;
    for (uint64_t p = 0; p <= T.mask; p++) {
        const long long cur = __ldcg(T.keys + pos);
        if (cur == k) return wait_gid(T, pos);
        if (cur == kEmptyKey) return kPending;
        pos = (pos + 1) & T.mask;
    }
    return kPending;
}
// Key k of group g inserted into the hash table by the one thread that
// handles k (its partition's CTA), which looks it up only after a barrier.
__device__ __forceinline__ void table_index_owned(const TableDev &T, long long k, uint32_t g) {
    uint64_t pos = hash_word((uint64_t)k) & T.mask;
    for (uint64_t p = 0; p <= T.mask; p++) {
        if (__ldcg(T.keys + pos) == kEmptyKey &&
            atomicCAS(reinterpret_cast<unsigned long long *>(T.keys + pos), (unsigned long long)kEmptyKey,
                      (unsigned long long)k) == (unsigned long long)kEmptyKey) {
            T.gids[pos] = g;
            return;
        }
        pos = (pos + 1) & T.mask;
    }
}

// Groups [from, to), whose keys and records exist but which the hash table
// may not index yet, inserted into it: each key once (a key has one group).
__global__ void index_groups_kernel(const long long *gkeys, uint64_t from, uint64_t to, long long *keys, uint32_t *gids,
                                    uint64_t mask) {
    for (uint64_t g = from + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < to;
         g += (uint64_t)gridDim.x * blockDim.x) {
        const long long k = gkeys[g];
        uint64_t pos = hash_word((uint64_t)k) & mask;
        for (uint64_t p = 0; p <= mask; p++) {
            const long long old = (long long)atomicCAS(reinterpret_cast<unsigned long long *>(keys + pos),
                                                       (unsigned long long)kEmptyKey, (unsigned long long)k);
            if (old == kEmptyKey) {
                gids[pos] = (uint32_t)g;
                break;
            }
            if (old == k) break;  // agg_part_kernel indexed it already
            pos = (pos + 1) & mask;
        }
    }
}

__device__ __forceinline__ uint32_t group_of(const TableDev &T, const AggPlanDev &P, const KeyIn &key, int64_t r,
                                             long long &k) {
    if (!bit_get(key.valid, key.voff, r)) return kNullGid;
    k = key_at(key, r);
    if (k == kEmptyKey) return kMarkerGid;
    return find_or_insert(T, P, k);
}

__device__ __forceinline__ void defer(uint32_t *ovf_rows, unsigned long long *ovf_count, int64_t r) {
    const unsigned long long at = atomicAdd(ovf_count, 1ull);
    ovf_rows[at] = (uint32_t)r;
}

// Global mode: every row goes to the global table.
__global__ void __launch_bounds__(256) agg_global_kernel(AggPlanDev P, TableDev T, KeyIn key, int64_t n,
                                                         const uint32_t *rows_idx, uint32_t *ovf_rows,
                                                         unsigned long long *ovf_count) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += stride) {
        const int64_t r = rows_idx ? (int64_t)rows_idx[i] : i;
        long long k = 0;
        const uint32_t g = group_of(T, P, key, r, k);
        if (g == kOverflowGid) {
            defer(ovf_rows, ovf_count, r);
            continue;
        }
        update_record(P, T.states + (size_t)g * P.rec, r);
    }
}

// Shared-memory pre-aggregation: a CTA-private table of `E` (power of two)
// entries filled up to `fill` keys; rows of other keys go to the global table.
// The `H` hottest keys (sampled on the host) also get one record per warp:
// the lanes of a warp that hold rows of one hot key take turns updating
// their warp's record of it with plain arithmetic (no atomics, no
// compare-and-swap float adds), lanes of different hot keys in the same turn,
// so a key that takes a large share of the rows is no longer updated by every
// thread of the CTA through one record. The row loop runs the same number of
// iterations on every lane, so the turns are taken by whole warps.
constexpr int kHotKeys = 16;
constexpr int kAggThreads = 1024;
__global__ void __launch_bounds__(kAggThreads) agg_shared_kernel(AggPlanDev P, TableDev T, KeyIn key, int64_t n,
                                                                 const uint32_t *rows_idx, uint32_t *ovf_rows,
                                                                 unsigned long long *ovf_count, int E, int fill,
                                                                 const long long *hot, int H) {
    extern __shared__ __align__(16) uint8_t smem[];
    constexpr int kWarps = kAggThreads / 32;
    uint8_t *wrec = smem;                                                          // kWarps * H * rec
    uint8_t *srec = smem + (size_t)kWarps * H * P.rec;                             // E * rec
    long long *skeys = reinterpret_cast<long long *>(srec + (size_t)E * P.rec);    // E
    uint32_t *sgid = reinterpret_cast<uint32_t *>(skeys + E);                      // E
    int *sfill = reinterpret_cast<int *>(sgid + E);
    __shared__ long long s_hot[kHotKeys];
    __shared__ uint32_t s_hot_gid[kHotKeys];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int e = threadIdx.x; e < E; e += blockDim.x) {
        skeys[e] = kEmptyKey;
        init_record(P, srec + (size_t)e * P.rec);
    }
    for (int e = threadIdx.x; e < kWarps * H; e += blockDim.x) init_record(P, wrec + (size_t)e * P.rec);
    if (threadIdx.x < H) {
        // A hot key the global table has no room for is not hot in this CTA.
        const long long k = hot[threadIdx.x];
        const uint32_t g = find_or_insert(T, P, k);
        s_hot[threadIdx.x] = k;
        s_hot_gid[threadIdx.x] = g;
    }
    if (threadIdx.x == 0) *sfill = 0;
    __syncthreads();
    const int emask = E - 1;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < n; base += stride) {
        const int64_t i = base + threadIdx.x;
        const bool live = i < n;
        const int64_t r = !live ? 0 : rows_idx ? (int64_t)rows_idx[i] : i;
        const bool valid_key = live && bit_get(key.valid, key.voff, r);
        const long long k = valid_key ? key_at(key, r) : 0;
        int h = -1;
        if (valid_key && k != kEmptyKey) {
#pragma unroll
            for (int j = 0; j < kHotKeys; j++)
                if (j < H && h < 0 && s_hot[j] == k && s_hot_gid[j] < kOverflowGid) h = j;
        }
        if (__ballot_sync(0xFFFFFFFFu, h >= 0)) {
            // Lanes of one hot key take turns; lanes of different hot keys
            // update their records in the same turn.
            const unsigned peers = __match_any_sync(0xFFFFFFFFu, h);
            const unsigned rank = __popc(peers & ((1u << lane) - 1u));
            const unsigned turns = __reduce_max_sync(0xFFFFFFFFu, h >= 0 ? (unsigned)__popc(peers) : 0u);
            for (unsigned t = 0; t < turns; t++) {
                if (h >= 0 && rank == t) update_record_plain(P, wrec + ((size_t)warp * H + h) * P.rec, r);
                __syncwarp();
            }
        }
        if (!live || h >= 0) continue;
        if (!valid_key) {
            update_record(P, T.states + (size_t)kNullGid * P.rec, r);
            continue;
        }
        if (k == kEmptyKey) {
            update_record(P, T.states + (size_t)kMarkerGid * P.rec, r);
            continue;
        }
        int slot = -1;
        uint32_t g = kPending;
        int pos = (int)(hash_word((uint64_t)k) & (uint64_t)emask);
        for (int p = 0; p < 16; p++) {
            const long long cur = *reinterpret_cast<volatile long long *>(skeys + pos);
            if (cur == k) {
                slot = pos;
                break;
            }
            if (cur == kEmptyKey) {
                if (*reinterpret_cast<volatile int *>(sfill) >= fill) break;
                if (g == kPending) {
                    g = find_or_insert(T, P, k);
                    if (g == kOverflowGid) break;
                }
                const long long old = (long long)atomicCAS(reinterpret_cast<unsigned long long *>(skeys + pos),
                                                           (unsigned long long)kEmptyKey, (unsigned long long)k);
                if (old == kEmptyKey) {
                    sgid[pos] = g;
                    atomicAdd(sfill, 1);
                    slot = pos;
                    break;
                }
                if (old == k) {
                    slot = pos;
                    break;
                }
            }
            pos = (pos + 1) & emask;
        }
        if (slot >= 0) {
            update_record(P, srec + (size_t)slot * P.rec, r);
            continue;
        }
        if (g == kPending) g = find_or_insert(T, P, k);
        if (g == kOverflowGid) {
            defer(ovf_rows, ovf_count, r);
            continue;
        }
        update_record(P, T.states + (size_t)g * P.rec, r);
    }
    __syncthreads();
    for (int e = threadIdx.x; e < E; e += blockDim.x)
        if (skeys[e] != kEmptyKey) merge_record(P, T.states + (size_t)sgid[e] * P.rec, srec + (size_t)e * P.rec);
    for (int e = threadIdx.x; e < kWarps * H; e += blockDim.x) {
        const int h = e % H;
        if (s_hot_gid[h] < kOverflowGid)
            merge_record(P, T.states + (size_t)s_hot_gid[h] * P.rec, wrec + (size_t)e * P.rec);
    }
}

// ---- partitioned aggregation ------------------------------------------------------
// Two passes over a batch, so that no row updates a record through a global
// atomic:
//  1. agg_split_kernel streams every row once. Rows of the hot keys (sampled
//     from the first batch), of the NULL key and of the marker key are combined
//     within the warp (lanes of one key reduce to one leader) and folded into
//     the CTA's shared-memory records of those keys; every other row is written
//     as one fixed-size row record into its hash partition.
//  2. agg_part_kernel runs one CTA per partition: the partition's rows are
//     folded into a shared-memory table of its keys (each cold key lives in one
//     partition only), and each key's record is merged once into the global
//     record of its group. A full local table is merged and emptied (a window);
//     a window whose keys find no room in the global table is not merged at all,
//     and the partition stops there to run again after the host grows the table.
// Row records: key (8 B) at 0, the validity word (bit c: plan column c valid)
// at 8, values at off_val[c] (4-byte values from 12, then 8- and 16-byte ones).
// Shared-memory records are laid out P.rec + 8 bytes apart: an odd number of
// 8-byte words, so one field of 32 different records falls in 32 different
// 8-byte bank pairs.
__host__ __device__ __forceinline__ int smem_stride(const AggPlanDev &P) { return P.rec + 8; }
constexpr int kHotMax = 512;
constexpr int kSplitThreads = 512;
constexpr int kPartThreads = 512;
constexpr int kCntStride = 32;  // partition counters one 128-byte line apart
constexpr unsigned kFullMask = 0xFFFFFFFFu;

struct SplitDev {
    const long long *hot_keys;  // H distinct keys, none equal to kEmptyKey
    const uint32_t *hot_gids;   // H + 2 global group ids (then the NULL and marker groups)
    int H;
    int hot_slots;  // the hot table: hot_slots / kHotWays buckets (a power of two; 0 when H == 0)
    const long long *hot_tab;   // its keys (kEmptyKey: free), bucket by bucket
    const int16_t *hot_tab_idx; // their indexes in hot_keys
    int part_bits;  // >= 1
    int row_bytes;
    int16_t off_val[kMaxValueCols];
    int ctas;                   // CTAs of the count and split kernels: CTA b takes the tiles of
                                // kSplitThreads rows b, b + ctas, b + 2 ctas, ...
    unsigned *cta_rows;         // [p * ctas + b]: partition p's cold rows of CTA b (count), then
                                // the rows of p before CTA b's (after part_offsets_kernel)
    uint8_t *part_buf;          // partition p: rows [base_p, base_p + rows_p)
    const unsigned int *part_info;  // partition p's line at p * kCntStride: [0] rows, [1] rows, [2..3] base_p
    unsigned long long cold;    // rows in part_buf (the bound of every write)
};

// Shared-memory accumulators. On the SM a 32-bit shared atomic add is one
// instruction, while 64-bit adds (integer or float) are compare-and-swap
// loops that retry whenever lanes meet on one word. So shared-memory records
// count in the low word of their 64-bit counters (one CTA folds fewer than
// 2^32 rows: batches are shorter) and add integer sums limb by limb, each
// 32-bit limb's carry taken from the value its own add returned. The limb
// adds of concurrent updaters commute, so the field is exact once they are
// all done (after a barrier).
__device__ __forceinline__ void s_count(uint8_t *field, unsigned v) {
    atomicAdd(reinterpret_cast<unsigned *>(field), v);
}
// Adds the N-limb two's-complement value `a` (least significant limb first)
// to the N-limb field at f.
template <int N>
__device__ __forceinline__ void s_add_limbs(uint8_t *f, const unsigned (&a)[N]) {
    unsigned *w = reinterpret_cast<unsigned *>(f);
    unsigned carry = 0;
#pragma unroll
    for (int i = 0; i < N; i++) {
        const unsigned x = a[i] + carry;
        carry = x < carry ? 1u : 0u;  // a[i] + carry wrapped (x is 0 then)
        if (x) {
            const unsigned old = atomicAdd(w + i, x);
            carry = old + x < old ? 1u : 0u;
        }
    }
}
// A signed 64-bit value added to a 64-bit field.
__device__ __forceinline__ void s_add_i64(uint8_t *f, long long v) {
    const unsigned a[2] = {(unsigned)v, (unsigned)((unsigned long long)v >> 32)};
    s_add_limbs<2>(f, a);
}
// A 128-bit value (lo, hi) added to a 128-bit field.
__device__ __forceinline__ void s_add_i128(uint8_t *f, uint64_t lo, uint64_t hi) {
    const unsigned a[4] = {(unsigned)lo, (unsigned)(lo >> 32), (unsigned)hi, (unsigned)(hi >> 32)};
    s_add_limbs<4>(f, a);
}

// A value as the accumulators take it: `lo`/`hi` the 128-bit sum operand of
// integer and decimal types (f64: the value's bits in lo); `mm` a signed
// 64-bit key whose order is the value's (f64: the order key with its top bit
// flipped; decimal128: the low word, MIN/MAX being for precision <= 18).
__device__ __forceinline__ void value_words(const AggColDev &C, const void *data, int64_t i, uint64_t &lo,
                                            uint64_t &hi) {
    if (C.type == (int)Type::I32 || C.type == (int)Type::Date32) {
        const long long v = static_cast<const int *>(data)[i];
        lo = (uint64_t)v;
        hi = v < 0 ? ~0ull : 0ull;
    } else if (C.type == (int)Type::Dec128) {
        const long long *p = static_cast<const long long *>(data) + 2 * i;
        lo = (uint64_t)p[0];
        hi = (uint64_t)p[1];
    } else {  // I64, Dec64, F64 (bits)
        const long long v = static_cast<const long long *>(data)[i];
        lo = (uint64_t)v;
        hi = v < 0 ? ~0ull : 0ull;
    }
}
// One row's inputs, loaded a warp step ahead of their use: the loads of a
// step do not depend on one another, so a warp waits for memory once per
// step and the wait overlaps the previous step's work. NV bounds the value
// columns held in registers (the plan's first NV columns; ncols <= NV).
template <int NV>
struct RowIn {
    long long k;
    uint64_t lo[NV];  // the low word of value_words of each value column (the high
                      // word: the sign, or for decimal128 read where it is used)
    uint32_t valid;   // bit c: value column c valid; bit 31: the key valid
};
constexpr uint32_t kKeyValid = 1u << 31;
// The high word of value_words for row r's value `lo` of column C.
__device__ __forceinline__ uint64_t value_hi(const AggColDev &C, int64_t r, uint64_t lo) {
    if (C.type == (int)Type::Dec128) return (uint64_t) static_cast<const long long *>(C.data)[2 * r + 1];
    return (long long)lo < 0 ? ~0ull : 0ull;
}

template <int NV>
__device__ __forceinline__ void load_row(const AggPlanDev &P, const KeyIn &key, int64_t r, bool live, RowIn<NV> &in) {
    in.k = 0;
    in.valid = 0;
#pragma unroll
    for (int c = 0; c < NV; c++) in.lo[c] = 0;
    if (!live) return;
    in.k = key_at(key, r);
    uint8_t vb[NV + 1];
    vb[NV] = key.valid ? key.valid[(key.voff + r) >> 3] : 0xFF;
#pragma unroll
    for (int c = 0; c < NV; c++) {
        vb[c] = 0;
        if (c >= P.ncols) continue;
        const AggColDev &C = P.c[c];
        vb[c] = C.valid ? C.valid[(C.voff + r) >> 3] : 0xFF;
        if (C.flags & (F_SUM | F_MIN | F_MAX)) {
            if (C.type == (int)Type::I32 || C.type == (int)Type::Date32)
                in.lo[c] = (uint64_t)(long long) static_cast<const int *>(C.data)[r];
            else if (C.type == (int)Type::Dec128) in.lo[c] = (uint64_t) static_cast<const long long *>(C.data)[2 * r];
            else in.lo[c] = (uint64_t) static_cast<const long long *>(C.data)[r];
        }
    }
    uint32_t bits = ((vb[NV] >> ((key.voff + r) & 7)) & 1u) ? kKeyValid : 0u;
#pragma unroll
    for (int c = 0; c < NV; c++)
        if (c < P.ncols) bits |= ((uint32_t)(vb[c] >> ((P.c[c].voff + r) & 7)) & 1u) << c;
    in.valid = bits;
}

// The hot rows of one warp step (`hi`: the lane's hot key, -1 when none),
// folded into the CTA's shared-memory records. Counts of a key's lanes go in
// one update (population counts of the warp's ballots); integer sums (32-bit
// limbs) and MIN/MAX go in per lane; float64 sums, which must stay
// compensated, are reduced to the key's lowest lane first (TwoSum over the
// other lanes' values) and added as one double-double.
template <int NV>
__device__ __forceinline__ void hot_rows(const AggPlanDev &P, uint8_t *hrec, const RowIn<NV> &in, int64_t r, int hi,
                                         unsigned lane) {
    const bool hot = hi >= 0;
    const unsigned peers = __match_any_sync(kFullMask, hot ? hi : 0x40000 + (int)lane);
    const unsigned lead_lane = __ffs(peers) - 1;
    const bool lead = hot && lane == lead_lane;
    uint8_t *rec = hrec + (size_t)(hot ? hi : 0) * smem_stride(P);
    if (lead) s_count(rec + P.off_rows, (unsigned)__popc(peers));
    unsigned turns = 0;  // the largest key group of the warp, for the float sums
#pragma unroll
    for (int c = 0; c < NV; c++) {
        if (c >= P.ncols) break;
        const AggColDev &C = P.c[c];
        const bool v = hot && ((in.valid >> c) & 1u);
        const unsigned vm = __ballot_sync(kFullMask, v) & peers;
        if (lead && vm) s_count(rec + C.off_count, (unsigned)__popc(vm));
        if (!(C.flags & (F_SUM | F_MIN | F_MAX))) continue;
        const uint64_t lo = in.lo[c];
        const bool i32 = C.type == (int)Type::I32 || C.type == (int)Type::Date32;
        if (C.type == (int)Type::F64) {
            if (C.flags & F_SUM) {
                if (!turns) turns = __reduce_max_sync(kFullMask, hot ? (unsigned)__popc(peers) : 1u);
                double ds = v ? __longlong_as_double((long long)lo) : 0.0, de = 0.0;
                unsigned rest = peers & (peers - 1u);
                for (unsigned t = 1; t < turns; t++) {
                    const unsigned src = rest ? (unsigned)__ffs(rest) - 1u : lane;
                    rest &= rest - 1u;
                    const double x = __shfl_sync(kFullMask, __longlong_as_double((long long)lo), src);
                    if (src != lane && ((vm >> src) & 1u)) {
                        double sum, err;
                        two_sum(ds, x, sum, err);
                        ds = sum;
                        de = __dadd_rn(de, err);
                    }
                }
                if (lead && vm)
                    atomic_add_dd2(reinterpret_cast<double *>(rec + C.off_sum),
                                   reinterpret_cast<double *>(rec + C.off_sum + 8), ds, de);
            }
            if (v && (C.flags & (F_MIN | F_MAX))) {
                const unsigned long long key = f64_order_key(__longlong_as_double((long long)lo));
                if (C.flags & F_MIN) atomicMin(reinterpret_cast<unsigned long long *>(rec + C.off_min), key);
                if (C.flags & F_MAX) atomicMax(reinterpret_cast<unsigned long long *>(rec + C.off_max), key);
            }
            continue;
        }
        if (!v) continue;
        if (C.flags & F_SUM) {
            if (i32) s_add_i64(rec + C.off_sum, (long long)lo);
            else s_add_i128(rec + C.off_sum, lo, value_hi(C, r, lo));
        }
        if (C.flags & F_MIN) {
            if (i32) atomicMin(reinterpret_cast<int *>(rec + C.off_min), (int)lo);
            else atomicMin(reinterpret_cast<long long *>(rec + C.off_min), (long long)lo);
        }
        if (C.flags & F_MAX) {
            if (i32) atomicMax(reinterpret_cast<int *>(rec + C.off_max), (int)lo);
            else atomicMax(reinterpret_cast<long long *>(rec + C.off_max), (long long)lo);
        }
    }
}

// The cold rows of one warp step, each written as a row record into its
// partition at the CTA's cursor for it (one shared-memory update per
// partition and warp step). The count pass gave every CTA its exact share of
// each partition, so a write past the buffer only follows a miscount: it is
// skipped and reported.
template <int NV>
__device__ __forceinline__ void cold_rows(const AggPlanDev &P, const SplitDev &S, const int16_t *off_val,
                                          unsigned *cursor, const RowIn<NV> &in, int64_t r, uint64_t h,
                                          bool cold, unsigned lane, uint32_t *status) {
    const int p = cold ? (int)(h >> (64 - S.part_bits)) : -1 - (int)lane;
    const unsigned peers = __match_any_sync(kFullMask, p);
    const unsigned lead_lane = __ffs(peers) - 1;
    unsigned base = 0;
    if (cold && lane == lead_lane) base = atomicAdd(cursor + p, (unsigned)__popc(peers));
    base = __shfl_sync(kFullMask, base, lead_lane);
    if (!cold) return;
    const unsigned at = base + __popc(peers & ((1u << lane) - 1u));
    if (at >= S.cold) {
        atomicOr(status, ST_MISCOUNT);
        return;
    }
    uint8_t *row = S.part_buf + (size_t)at * S.row_bytes;
    *reinterpret_cast<long long *>(row) = in.k;
    *reinterpret_cast<uint32_t *>(row + 8) = in.valid & ~kKeyValid;
#pragma unroll
    for (int c = 0; c < NV; c++) {
        if (c >= P.ncols) break;
        const AggColDev &C = P.c[c];
        if (!((in.valid >> c) & 1u) || !(C.flags & (F_SUM | F_MIN | F_MAX))) continue;
        uint8_t *dst = row + off_val[c];
        if (C.type == (int)Type::I32 || C.type == (int)Type::Date32) *reinterpret_cast<int *>(dst) = (int)in.lo[c];
        else if (C.type == (int)Type::Dec128)
            *reinterpret_cast<longlong2 *>(dst) =
                make_longlong2((long long)in.lo[c], (long long)value_hi(C, r, in.lo[c]));
        else *reinterpret_cast<long long *>(dst) = (long long)in.lo[c];
    }
}

// The hot-key table: kHotWays keys per bucket, every key in one of its two
// buckets (hot_buckets), placed on the host (a key that fits neither is left
// cold). A lookup reads both buckets whole: no probe loop, so the lanes of a
// warp do not diverge on it.
constexpr int kHotWays = 4;
__host__ __device__ __forceinline__ void hot_buckets(uint64_t h, int nbuckets, int &b1, int &b2) {
    b1 = (int)(h & (uint64_t)(nbuckets - 1));
    b2 = (int)((h >> 32) & (uint64_t)(nbuckets - 1));
    if (b2 == b1) b2 = b1 ^ 1;
}
// The CTA's copy of the table in shared memory (the indexes when hidx).
__device__ __forceinline__ void hot_table_init(const SplitDev &S, long long *hkeys, int16_t *hidx) {
    for (int e = threadIdx.x; e < S.hot_slots; e += blockDim.x) {
        hkeys[e] = S.hot_tab[e];
        if (hidx) hidx[e] = S.hot_tab_idx[e];
    }
    __syncthreads();
}
// The index of hot key k, -1 when it is not hot (0 for a hot key when hidx
// is null).
__device__ __forceinline__ int hot_index(const SplitDev &S, const long long *hkeys, const int16_t *hidx, long long k,
                                         uint64_t h) {
    if (!S.H) return -1;
    int b1, b2;
    hot_buckets(h, S.hot_slots / kHotWays, b1, b2);
    const longlong2 *t = reinterpret_cast<const longlong2 *>(hkeys);
    const longlong2 x0 = t[2 * b1], x1 = t[2 * b1 + 1], y0 = t[2 * b2], y1 = t[2 * b2 + 1];
    int slot = -1;
    slot = x0.x == k ? 4 * b1 : slot;
    slot = x0.y == k ? 4 * b1 + 1 : slot;
    slot = x1.x == k ? 4 * b1 + 2 : slot;
    slot = x1.y == k ? 4 * b1 + 3 : slot;
    slot = y0.x == k ? 4 * b2 : slot;
    slot = y0.y == k ? 4 * b2 + 1 : slot;
    slot = y1.x == k ? 4 * b2 + 2 : slot;
    slot = y1.y == k ? 4 * b2 + 3 : slot;
    if (slot < 0) return -1;
    return hidx ? hidx[slot] : 0;
}
// A row's place in the split: hot index (>= 0, then H for the NULL key and
// H + 1 for the marker key), -1 for a cold row (partition from h), -2 past
// the end.
__device__ __forceinline__ int classify(const SplitDev &S, const long long *hkeys, const int16_t *hidx, bool live,
                                        bool kv, long long k, uint64_t h) {
    if (!live) return -2;
    if (!kv) return S.H;
    if (k == kEmptyKey) return S.H + 1;
    return hot_index(S, hkeys, hidx, k, h);
}

template <int NV>
__global__ void __launch_bounds__(kSplitThreads, 2) agg_split_kernel(AggPlanDev P, TableDev T, KeyIn key, int64_t n,
                                                                     SplitDev S) {
    extern __shared__ __align__(16) uint8_t smem[];
    const int NH = S.H + 2;
    const int nparts = 1 << S.part_bits;
    uint8_t *hrec = smem;                                                                  // NH records
    long long *hkeys = reinterpret_cast<long long *>(hrec + ((size_t)NH * smem_stride(P) + 15) / 16 * 16);  // hot_slots
    unsigned *cursor = reinterpret_cast<unsigned *>(hkeys + S.hot_slots);                  // nparts
    int16_t *hidx = reinterpret_cast<int16_t *>(cursor + nparts);                          // hot_slots
    const unsigned lane = threadIdx.x & 31u;
    __shared__ int16_t s_off[kMaxValueCols];  // row record offsets (read with a varying index)
    if (threadIdx.x < kMaxValueCols) s_off[threadIdx.x] = S.off_val[threadIdx.x];
    for (int e = threadIdx.x; e < NH; e += blockDim.x) init_record(P, hrec + (size_t)e * smem_stride(P));
    for (int q = threadIdx.x; q < nparts; q += blockDim.x) {
        const unsigned int *line = S.part_info + (size_t)q * kCntStride;
        cursor[q] = (unsigned)*reinterpret_cast<const unsigned long long *>(line + 2) +
                    S.cta_rows[(size_t)q * S.ctas + blockIdx.x];
    }
    hot_table_init(S, hkeys, hidx);
    // Tiles of blockDim rows, CTA b taking tiles b, b + ctas, ... (the
    // count kernel's assignment).
    const int64_t step = (int64_t)gridDim.x * blockDim.x;
    int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    RowIn<NV> cur;
    load_row(P, key, r, r < n, cur);
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < n; base += step, r += step) {
        RowIn<NV> nxt;
        load_row(P, key, r + step, r + step < n, nxt);
        const bool live = r < n;
        const uint64_t h = hash_word((uint64_t)cur.k);
        const int cls = classify(S, hkeys, hidx, live, (cur.valid & kKeyValid) != 0, cur.k, h);
        if (__any_sync(kFullMask, cls >= 0)) hot_rows(P, hrec, cur, r, cls, lane);
        const bool cold = cls == -1;
        if (__any_sync(kFullMask, cold)) cold_rows(P, S, s_off, cursor, cur, r, h, cold, lane, T.status);
        cur = nxt;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < NH; e += blockDim.x) {
        if (S.hot_gids[e] < kOverflowGid)
            merge_record(P, T.states + (size_t)S.hot_gids[e] * P.rec, hrec + (size_t)e * smem_stride(P));
        else atomicOr(T.status, ST_CAPACITY);
    }
}

// Cold rows per partition and CTA, by the split kernel's own test over the
// split kernel's tiles: cta_rows[p * ctas + b] (zeroed first) gets the rows of
// partition p in split CTA b's tiles. Two CTAs share each split CTA's tiles
// (twice the warps to hide the loads); four rows per thread and step, their
// loads issued together.
__global__ void __launch_bounds__(kSplitThreads) agg_count_kernel(KeyIn key, int64_t n, SplitDev S) {
    extern __shared__ __align__(16) uint8_t smem[];
    const int nparts = 1 << S.part_bits;
    unsigned int *s_hist = reinterpret_cast<unsigned int *>(smem);                    // nparts
    long long *hkeys = reinterpret_cast<long long *>(s_hist + ((nparts + 1) & ~1));  // hot_slots
    for (int q = threadIdx.x; q < nparts; q += blockDim.x) s_hist[q] = 0;
    hot_table_init(S, hkeys, nullptr);
    // gridDim.x = K * ctas: CTA (b, q) takes every K-th of split CTA b's
    // tiles from its q-th on.
    const int G = S.ctas, K = (int)gridDim.x / G, b = (int)blockIdx.x % G, q0 = (int)blockIdx.x / G;
    const int64_t step = (int64_t)K * G * blockDim.x;  // rows between this CTA's tiles
    constexpr int U = 4;
    for (int64_t base = ((int64_t)b + (int64_t)G * q0) * blockDim.x + threadIdx.x; base < n; base += U * step) {
        long long k[U];
        uint8_t vb[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int64_t r = base + u * step;
            k[u] = r < n ? key_at(key, r) : 0;
            vb[u] = r < n ? (key.valid ? key.valid[(key.voff + r) >> 3] : 0xFF) : 0;
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int64_t r = base + u * step;
            const bool kv = (vb[u] >> ((key.voff + r) & 7)) & 1u;
            const uint64_t h = hash_word((uint64_t)k[u]);
            if (classify(S, hkeys, nullptr, r < n, kv, k[u], h) == -1)
                atomicAdd(&s_hist[(int)(h >> (64 - S.part_bits))], 1u);
        }
    }
    __syncthreads();
    for (int q = threadIdx.x; q < nparts; q += blockDim.x)
        if (s_hist[q]) atomicAdd(&S.cta_rows[(size_t)q * G + b], s_hist[q]);
}

// Per partition (one warp each): the exclusive running count of its rows over
// the CTAs, in place, and the partition's total.
__global__ void part_offsets_kernel(unsigned *cta_rows, int ctas, int nparts, unsigned *total) {
    const int p = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
    const unsigned lane = threadIdx.x & 31u;
    if (p >= nparts) return;
    unsigned *row = cta_rows + (size_t)p * ctas;
    unsigned carry = 0;
    for (int b0 = 0; b0 < ctas; b0 += 32) {
        const int b = b0 + (int)lane;
        const unsigned x = b < ctas ? row[b] : 0u;
        unsigned incl = x;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const unsigned y = __shfl_up_sync(kFullMask, incl, d);
            if ((int)lane >= d) incl += y;
        }
        if (b < ctas) row[b] = carry + incl - x;
        carry += __shfl_sync(kFullMask, incl, 31);
    }
    if (lane == 0) total[p] = carry;
}

// The partitions laid out back to back: each partition's line [rows, rows,
// base] and the rows of all (one CTA of 1024 threads).
__global__ void __launch_bounds__(1024) part_bases_kernel(const unsigned *total, int nparts, unsigned *info,
                                                          unsigned long long *cold) {
    __shared__ unsigned long long s_warp[32];
    const int per = (nparts + blockDim.x - 1) / blockDim.x;
    const int q0 = threadIdx.x * per;
    unsigned long long mine = 0;
    for (int q = q0; q < q0 + per && q < nparts; q++) mine += total[q];
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    unsigned long long incl = mine;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const unsigned long long y = __shfl_up_sync(kFullMask, incl, d);
        if ((int)lane >= d) incl += y;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const unsigned long long w = lane < blockDim.x / 32 ? s_warp[lane] : 0ull;
        unsigned long long wi = w;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const unsigned long long y = __shfl_up_sync(kFullMask, wi, d);
            if ((int)lane >= d) wi += y;
        }
        s_warp[lane] = wi - w;  // exclusive over the warps
        if (lane == 31) *cold = wi;
    }
    __syncthreads();
    unsigned long long base = s_warp[warp] + incl - mine;
    for (int q = q0; q < q0 + per && q < nparts; q++) {
        unsigned *line = info + (size_t)q * kCntStride;
        line[0] = line[1] = total[q];
        *reinterpret_cast<unsigned long long *>(line + 2) = base;
        base += total[q];
    }
}

struct PartDev {
    const uint8_t *part_buf;
    const unsigned int *part_info;  // as SplitDev::part_info
    int row_bytes;
    int16_t off_val[kMaxValueCols];
    const int *todo;   // the partitions to run: CTA b runs partition todo[b] (all, in order, when null)
    uint32_t *start;   // per partition: its first row not yet merged (read and written)
    int *failed;       // partitions that stopped for want of room in the global table
    unsigned long long id_limit;  // new group ids only while the count is at most this
    unsigned long long first_new; // the first group id this launch hands out
    int lookup;                   // the global table may hold keys of these partitions
};

// agg_part_kernel works through a partition in chunks of at most kChunkRows
// rows:
//  1. the chunk's row records are copied into shared memory, and every row's
//     key gets a local slot (claimed when new) and its rank among the chunk's
//     rows of that slot (the value a 32-bit shared atomic add returned);
//  2. the slot counts are scanned and the used slots listed by size;
//  3. each row is placed at its slot's offset plus its rank (a counting sort);
//     keys new to the local table get their group ids in one step per chunk:
//     a lookup each (none while the global table holds no cold key), then one
//     reservation of ids for those it lacks (all or none: a chunk whose keys
//     find no room is not merged, and the partition stops there to run again
//     after the host grows the table); a new group's key goes to gkeys, and
//     the host indexes the new groups in the hash table (index_groups_kernel)
//     before anything looks keys up again;
//  4. each key's rows are reduced in registers by a team sized to them (a
//     lane below kTeamRows rows, kTeamLanes lanes below kWarpRows, a warp
//     per kSegRows rows from there on), and the sums merged into the key's
//     global record with plain loads and stores: a cold key lives in one
//     partition only, so its record has one writer, and the chunks of a
//     partition run in turn. Only a key of more than kSegRows rows, whose
//     segments several warps reduce at once, merges through atomics.
// The local table and its group ids carry over from chunk to chunk, until
// its keys pass a quarter of its slots.
constexpr int kChunkRows = 1024;
constexpr int kChunkSlots = 2048;
constexpr int kTeamRows = 8, kTeamLanes = 8, kWarpRows = 64, kSegRows = 128;
constexpr int kAccCols = 2;  // value columns reduced per pass over a key's rows (three spill at 64 registers)
constexpr uint32_t kNoGid = 0xFFFFFFFFu, kNewGid = 0x80000000u;

__host__ __device__ __forceinline__ size_t part_smem_bytes(int row_bytes) {
    return (size_t)kChunkRows * row_bytes + (size_t)kChunkSlots * (8 + 4 + 4 + 2) + (size_t)kChunkRows * 2 * 5;
}

// The accumulators of up to kAccCols value columns: the record's fields in
// registers. Sums: int32 columns in s0 (64-bit); int64 and decimal columns as
// 128 bits (s0 low, s1 high); float64 as a double-double (s0 high, s1 low,
// as bits). MIN/MAX: float64 as order keys (unsigned), the rest signed.
struct ColAcc {
    uint32_t cnt;  // a chunk has fewer than 2^32 rows
    uint64_t s0, s1;
    uint64_t mn, mx;
};
struct RowAcc {
    uint32_t rows;
    ColAcc c[kAccCols];
};

__device__ __forceinline__ bool acc_f64(const AggColDev &C) { return C.type == (int)Type::F64; }
__device__ __forceinline__ bool acc_i32(const AggColDev &C) {
    return C.type == (int)Type::I32 || C.type == (int)Type::Date32;
}

__device__ __forceinline__ void acc_init(const AggPlanDev &P, int cb, RowAcc &a) {
    a.rows = 0;
#pragma unroll
    for (int u = 0; u < kAccCols; u++) {
        ColAcc &x = a.c[u];
        x.cnt = 0;
        x.s0 = x.s1 = 0;
        const bool f = cb + u < P.ncols && acc_f64(P.c[cb + u]);
        x.mn = f ? ~0ull : (uint64_t)LLONG_MAX;
        x.mx = f ? 0ull : (uint64_t)LLONG_MIN;
    }
}

__device__ __forceinline__ void acc_min_max(bool f64, ColAcc &x, uint64_t mn, uint64_t mx) {
    if (f64) {
        x.mn = mn < x.mn ? mn : x.mn;
        x.mx = mx > x.mx ? mx : x.mx;
    } else {
        x.mn = (long long)mn < (long long)x.mn ? mn : x.mn;
        x.mx = (long long)mx > (long long)x.mx ? mx : x.mx;
    }
}
// x += the sums of another partial y (counts apart).
__device__ __forceinline__ void acc_add(const AggColDev &C, ColAcc &x, const ColAcc &y) {
    if (C.flags & F_SUM) {
        if (acc_f64(C)) {
            double s, e;
            two_sum(__longlong_as_double((long long)x.s0), __longlong_as_double((long long)y.s0), s, e);
            const double lo = __dadd_rn(__dadd_rn(__longlong_as_double((long long)x.s1),
                                                  __longlong_as_double((long long)y.s1)), e);
            x.s0 = (uint64_t)__double_as_longlong(s);
            x.s1 = (uint64_t)__double_as_longlong(lo);
        } else if (acc_i32(C)) {
            x.s0 += y.s0;
        } else {
            const uint64_t lo = x.s0 + y.s0;
            x.s1 += y.s1 + (lo < x.s0 ? 1ull : 0ull);
            x.s0 = lo;
        }
    }
    if (C.flags & (F_MIN | F_MAX)) acc_min_max(acc_f64(C), x, y.mn, y.mx);
}

// One row record's columns [cb, cb + kAccCols) folded into the accumulators.
__device__ __forceinline__ void acc_row(const AggPlanDev &P, const int16_t *off_val, int cb, RowAcc &a,
                                        const uint8_t *row) {
    a.rows++;
    const uint32_t bits = *reinterpret_cast<const uint32_t *>(row + 8);
#pragma unroll
    for (int u = 0; u < kAccCols; u++) {
        const int c = cb + u;
        if (c >= P.ncols) break;
        if (!((bits >> c) & 1u)) continue;
        const AggColDev &C = P.c[c];
        ColAcc &x = a.c[u];
        x.cnt++;
        if (!(C.flags & (F_SUM | F_MIN | F_MAX))) continue;
        uint64_t lo, hi;
        value_words(C, row + off_val[c], 0, lo, hi);
        if (acc_f64(C)) {
            const double v = __longlong_as_double((long long)lo);
            if (C.flags & F_SUM) {
                double s, e;
                two_sum(__longlong_as_double((long long)x.s0), v, s, e);
                x.s0 = (uint64_t)__double_as_longlong(s);
                x.s1 = (uint64_t)__double_as_longlong(__dadd_rn(__longlong_as_double((long long)x.s1), e));
            }
            if (C.flags & (F_MIN | F_MAX)) {
                const uint64_t k = f64_order_key(v);
                acc_min_max(true, x, k, k);
            }
            continue;
        }
        if (C.flags & F_SUM) {
            if (acc_i32(C)) {
                x.s0 += lo;
            } else {
                const uint64_t s = x.s0 + lo;
                x.s1 += hi + (s < x.s0 ? 1ull : 0ull);
                x.s0 = s;
            }
        }
        if (C.flags & (F_MIN | F_MAX)) acc_min_max(false, x, lo, lo);
    }
}

// A team's accumulators summed into its first lane's (teams of `width`
// lanes, aligned; every lane of the warp takes part).
__device__ __forceinline__ void acc_team_sum(const AggPlanDev &P, int cb, RowAcc &a, int width) {
    for (int d = width >> 1; d >= 1; d >>= 1) {
        a.rows += __shfl_down_sync(kFullMask, a.rows, d, width);
#pragma unroll
        for (int u = 0; u < kAccCols; u++) {
            if (cb + u >= P.ncols) break;
            ColAcc y;
            y.cnt = __shfl_down_sync(kFullMask, a.c[u].cnt, d, width);
            y.s0 = __shfl_down_sync(kFullMask, a.c[u].s0, d, width);
            y.s1 = __shfl_down_sync(kFullMask, a.c[u].s1, d, width);
            y.mn = __shfl_down_sync(kFullMask, a.c[u].mn, d, width);
            y.mx = __shfl_down_sync(kFullMask, a.c[u].mx, d, width);
            a.c[u].cnt += y.cnt;
            acc_add(P.c[cb + u], a.c[u], y);
        }
    }
}

// The accumulators merged into a global record that nothing else writes
// meanwhile (Accumulator::merge, accumulator.rs:1159). Every field is read
// before any is written: the field offsets are runtime values, so loads
// placed after stores would each wait for the stores before them.
__device__ __forceinline__ void acc_merge(const AggPlanDev &P, int cb, const RowAcc &a, uint8_t *r) {
    unsigned long long rows = 0, cnt[kAccCols];
    ColAcc x[kAccCols];
    if (cb == 0) rows = *reinterpret_cast<const unsigned long long *>(r + P.off_rows);
#pragma unroll
    for (int u = 0; u < kAccCols; u++) {
        const int c = cb + u;
        cnt[u] = 0;
        x[u].cnt = 0;
        x[u].s0 = x[u].s1 = x[u].mn = x[u].mx = 0;
        if (c >= P.ncols || !a.c[u].cnt) continue;
        const AggColDev &C = P.c[c];
        cnt[u] = *reinterpret_cast<const unsigned long long *>(r + C.off_count);
        if (C.flags & F_SUM) {
            x[u].s0 = *reinterpret_cast<const uint64_t *>(r + C.off_sum);
            if (!acc_i32(C)) x[u].s1 = *reinterpret_cast<const uint64_t *>(r + C.off_sum + 8);
        }
        if (acc_i32(C)) {
            x[u].mn = (uint64_t)(long long)((C.flags & F_MIN) ? *reinterpret_cast<const int *>(r + C.off_min) : INT_MAX);
            x[u].mx = (uint64_t)(long long)((C.flags & F_MAX) ? *reinterpret_cast<const int *>(r + C.off_max) : INT_MIN);
        } else {
            x[u].mn = (C.flags & F_MIN) ? *reinterpret_cast<const uint64_t *>(r + C.off_min) : a.c[u].mn;
            x[u].mx = (C.flags & F_MAX) ? *reinterpret_cast<const uint64_t *>(r + C.off_max) : a.c[u].mx;
        }
    }
    if (cb == 0) *reinterpret_cast<unsigned long long *>(r + P.off_rows) = rows + a.rows;
#pragma unroll
    for (int u = 0; u < kAccCols; u++) {
        const int c = cb + u;
        if (c >= P.ncols || !a.c[u].cnt) continue;
        const AggColDev &C = P.c[c];
        *reinterpret_cast<unsigned long long *>(r + C.off_count) = cnt[u] + a.c[u].cnt;
        if (!(C.flags & (F_SUM | F_MIN | F_MAX))) continue;
        acc_add(C, x[u], a.c[u]);
        if (C.flags & F_SUM) {
            *reinterpret_cast<uint64_t *>(r + C.off_sum) = x[u].s0;
            if (!acc_i32(C)) *reinterpret_cast<uint64_t *>(r + C.off_sum + 8) = x[u].s1;
        }
        if (acc_i32(C)) {
            if (C.flags & F_MIN) *reinterpret_cast<int *>(r + C.off_min) = (int)(long long)x[u].mn;
            if (C.flags & F_MAX) *reinterpret_cast<int *>(r + C.off_max) = (int)(long long)x[u].mx;
        } else {
            if (C.flags & F_MIN) *reinterpret_cast<uint64_t *>(r + C.off_min) = x[u].mn;
            if (C.flags & F_MAX) *reinterpret_cast<uint64_t *>(r + C.off_max) = x[u].mx;
        }
    }
}

// The accumulators merged into a global record that other warps update at
// the same time (the segments of one key): global atomics.
__device__ __forceinline__ void acc_merge_atomic(const AggPlanDev &P, int cb, const RowAcc &a, uint8_t *r) {
    if (cb == 0) atomicAdd(reinterpret_cast<unsigned long long *>(r + P.off_rows), (unsigned long long)a.rows);
#pragma unroll
    for (int u = 0; u < kAccCols; u++) {
        const int c = cb + u;
        if (c >= P.ncols || !a.c[u].cnt) continue;
        const AggColDev &C = P.c[c];
        const ColAcc &y = a.c[u];
        atomicAdd(reinterpret_cast<unsigned long long *>(r + C.off_count), (unsigned long long)y.cnt);
        if (C.flags & F_SUM) {
            if (acc_f64(C))
                atomic_add_dd2(reinterpret_cast<double *>(r + C.off_sum), reinterpret_cast<double *>(r + C.off_sum + 8),
                               __longlong_as_double((long long)y.s0), __longlong_as_double((long long)y.s1));
            else if (acc_i32(C)) atomicAdd(reinterpret_cast<unsigned long long *>(r + C.off_sum), (unsigned long long)y.s0);
            else
                atomic_add_i128(reinterpret_cast<unsigned long long *>(r + C.off_sum),
                                reinterpret_cast<long long *>(r + C.off_sum + 8), (int64_t)y.s0, (int64_t)y.s1);
        }
        if (acc_i32(C)) {
            if (C.flags & F_MIN) atomicMin(reinterpret_cast<int *>(r + C.off_min), (int)(long long)y.mn);
            if (C.flags & F_MAX) atomicMax(reinterpret_cast<int *>(r + C.off_max), (int)(long long)y.mx);
        } else if (acc_f64(C)) {
            if (C.flags & F_MIN) atomicMin(reinterpret_cast<unsigned long long *>(r + C.off_min), (unsigned long long)y.mn);
            if (C.flags & F_MAX) atomicMax(reinterpret_cast<unsigned long long *>(r + C.off_max), (unsigned long long)y.mx);
        } else {
            if (C.flags & F_MIN) atomicMin(reinterpret_cast<long long *>(r + C.off_min), (long long)y.mn);
            if (C.flags & F_MAX) atomicMax(reinterpret_cast<long long *>(r + C.off_max), (long long)y.mx);
        }
    }
}

__global__ void __launch_bounds__(kPartThreads, 2) agg_part_kernel(AggPlanDev P, TableDev T, PartDev D) {
    extern __shared__ __align__(16) uint8_t smem[];
    uint8_t *srows = smem;                                                                       // kChunkRows rows
    long long *skeys = reinterpret_cast<long long *>(srows + (size_t)kChunkRows * D.row_bytes);  // slots
    uint32_t *sgid = reinterpret_cast<uint32_t *>(skeys + kChunkSlots);                          // slots
    uint32_t *scnt = sgid + kChunkSlots;                                                         // slots
    uint16_t *soff = reinterpret_cast<uint16_t *>(scnt + kChunkSlots);                           // slots
    uint16_t *slot_of = soff + kChunkSlots;  // per chunk row: its slot
    uint16_t *rank_of = slot_of + kChunkRows;  // per chunk row: its rank among its slot's rows
    uint16_t *order = rank_of + kChunkRows;    // chunk rows sorted by slot
    uint16_t *big = order + kChunkRows;        // warp keys from the front, team keys from the back
    uint16_t *small = big + kChunkRows;        // one-lane keys
    __shared__ uint32_t s_warp[kPartThreads / 32];
    __shared__ int s_seg[kChunkRows / kWarpRows + 1];  // warp keys' first segments (then their count)
    __shared__ int s_keys, s_nw, s_nt, s_n1, s_fail, s_new;
    __shared__ unsigned long long s_base;
    __shared__ int16_t s_off[kMaxValueCols];  // row record offsets (read with a varying index)
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    constexpr int kWarps = kPartThreads / 32;
    if (threadIdx.x < kMaxValueCols) s_off[threadIdx.x] = D.off_val[threadIdx.x];
    const int p = D.todo ? D.todo[blockIdx.x] : (int)blockIdx.x;
    const unsigned int *line = D.part_info + (size_t)p * kCntStride;
    const uint32_t cnt = line[0], cap = line[1];
    const uint32_t rows = cnt < cap ? cnt : cap;
    const uint8_t *buf = D.part_buf + *reinterpret_cast<const unsigned long long *>(line + 2) * D.row_bytes;
    constexpr int kMask = kChunkSlots - 1;
    bool fresh = true;  // the local table is empty
    bool lookup = D.lookup != 0;
    for (uint32_t c0 = D.start[p]; c0 < rows; c0 += kChunkRows) {
        const int n = (int)(rows - c0 < (uint32_t)kChunkRows ? rows - c0 : (uint32_t)kChunkRows);
        // the table: emptied when new, or when its keys passed a quarter of
        // its slots (a chunk adds at most kChunkRows more); the counts always
        const bool clear = fresh || s_keys > kChunkSlots / 4;
        __syncthreads();  // every thread has read s_keys
        if (clear) {
            if (!fresh) {
                // The keys this CTA gave new groups go into the hash table
                // before the local table forgets them: later chunks look
                // them up there.
                for (int s = threadIdx.x; s < kChunkSlots; s += blockDim.x)
                    if (skeys[s] != kEmptyKey && sgid[s] != kNoGid && sgid[s] >= D.first_new)
                        table_index_owned(T, skeys[s], sgid[s]);
                lookup = true;
                __syncthreads();
            }
            for (int s = threadIdx.x; s < kChunkSlots; s += blockDim.x) {
                skeys[s] = kEmptyKey;
                sgid[s] = kNoGid;
            }
            if (threadIdx.x == 0) s_keys = 0;
            fresh = false;
        }
        for (int s = threadIdx.x; s < kChunkSlots; s += blockDim.x) scnt[s] = 0;
        if (threadIdx.x == 0) {
            s_nw = s_nt = s_n1 = 0;
            s_fail = 0;
            s_new = 0;
            s_base = ~0ull;
        }
        // 1. the chunk's rows into shared memory (16-byte words), then slots and ranks
        {
            const uint4 *src = reinterpret_cast<const uint4 *>(buf + (size_t)c0 * D.row_bytes);
            uint4 *dst = reinterpret_cast<uint4 *>(srows);
            const int words = n * D.row_bytes / 16;
            for (int w = threadIdx.x; w < words; w += blockDim.x) dst[w] = src[w];
        }
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const long long k = *reinterpret_cast<const long long *>(srows + (size_t)i * D.row_bytes);
            int pos = (int)(hash_word((uint64_t)k) & (uint64_t)kMask);
            for (int t = 0; t < kChunkSlots; t++) {
                long long cur = skeys[pos];
                if (cur == kEmptyKey) {
                    cur = (long long)atomicCAS(reinterpret_cast<unsigned long long *>(skeys + pos),
                                               (unsigned long long)kEmptyKey, (unsigned long long)k);
                    if (cur == kEmptyKey) {
                        atomicAdd(&s_keys, 1);
                        break;
                    }
                }
                if (cur == k) break;
                pos = (pos + 1) & kMask;
            }
            slot_of[i] = (uint16_t)pos;
            rank_of[i] = (uint16_t)atomicAdd(&scnt[pos], 1u);
        }
        __syncthreads();
        // 2. exclusive scan of the slot counts, and the used slots listed by size
        constexpr int kPer = kChunkSlots / kPartThreads;
        const int s0 = threadIdx.x * kPer;
        uint32_t mine = 0;
#pragma unroll
        for (int j = 0; j < kPer; j++) mine += scnt[s0 + j];
        uint32_t incl = mine;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(kFullMask, incl, d);
            if ((int)lane >= d) incl += y;
        }
        if (lane == 31) s_warp[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            const uint32_t w = lane < kWarps ? s_warp[lane] : 0u;
            uint32_t wi = w;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const uint32_t y = __shfl_up_sync(kFullMask, wi, d);
                if ((int)lane >= d) wi += y;
            }
            if (lane < kWarps) s_warp[lane] = wi - w;
        }
        __syncthreads();
        uint32_t run = s_warp[warp] + incl - mine;
#pragma unroll
        for (int j = 0; j < kPer; j++) {
            const int s = s0 + j;
            const uint32_t c = scnt[s];
            soff[s] = (uint16_t)run;
            run += c;
            if (c >= (uint32_t)kWarpRows) big[atomicAdd(&s_nw, 1)] = (uint16_t)s;
            else if (c >= (uint32_t)kTeamRows) big[kChunkRows - 1 - atomicAdd(&s_nt, 1)] = (uint16_t)s;
            else if (c) small[atomicAdd(&s_n1, 1)] = (uint16_t)s;
        }
        __syncthreads();
        // 3. the counting sort's scatter, and group ids for keys new to the local table
        for (int i = threadIdx.x; i < n; i += blockDim.x) order[soff[slot_of[i]] + rank_of[i]] = (uint16_t)i;
        const int nw = s_nw, nt = s_nt, n1 = s_n1;
        const int nused = nw + nt + n1;
        auto used_slot = [&](int u) -> int {
            if (u < nw) return big[u];
            u -= nw;
            if (u < nt) return big[kChunkRows - 1 - u];
            return small[u - nt];
        };
        if (threadIdx.x == 0) {  // the warp keys' segments of kSegRows rows
            int acc = 0;
            for (int u = 0; u < nw; u++) {
                s_seg[u] = acc;
                acc += ((int)scnt[big[u]] + kSegRows - 1) / kSegRows;
            }
            s_seg[nw] = acc;
        }
        for (int u = threadIdx.x; u < nused; u += blockDim.x) {  // found, or kNewGid + local index
            const int s = used_slot(u);
            if (sgid[s] != kNoGid) continue;
            const uint32_t g = lookup ? table_find(T, skeys[s]) : kPending;
            if (g == kOverflowGid) {  // a wait that gave up (reported as ST_TIMEOUT)
                atomicOr(&s_fail, 1);
                continue;
            }
            sgid[s] = g != kPending ? g : kNewGid | (uint32_t)atomicAdd(&s_new, 1);
        }
        __syncthreads();
        if (threadIdx.x == 0 && s_new) {  // ids for the new keys, all or none
            // Checked, then added: CTAs that pass the check together take at
            // most D.id_room more ids than D.id_limit, which the table holds.
            if (__ldcg(T.ngroups) + (unsigned long long)s_new > D.id_limit) s_fail = 1;
            else s_base = atomicAdd(T.ngroups, (unsigned long long)s_new);
        }
        if (__syncthreads_or(s_fail)) {
            if (threadIdx.x == 0) {
                D.start[p] = c0;
                atomicAdd(D.failed, 1);
            }
            return;
        }
        if (s_new) {
            for (int u = threadIdx.x; u < nused; u += blockDim.x) {
                const int s = used_slot(u);
                const uint32_t v = sgid[s];
                if (v == kNoGid || !(v & kNewGid)) continue;
                const uint32_t g = (uint32_t)s_base + (v & ~kNewGid);
                init_record(P, T.states + (size_t)g * P.rec);
                T.gkeys[g] = skeys[s];
                sgid[s] = g;
            }
            __syncthreads();
        }
        // 4. reduce and merge
        for (int cb = 0; cb < P.ncols || cb == 0; cb += kAccCols) {
            const int nseg = s_seg[nw];
            for (int it = warp; it < nseg; it += kWarps) {  // a warp per kSegRows rows of a key
                int u = 0;
                while (s_seg[u + 1] <= it) u++;
                const int s = big[u];
                const int m = (int)scnt[s];
                const int j0 = (it - s_seg[u]) * kSegRows, j1 = j0 + kSegRows < m ? j0 + kSegRows : m;
                RowAcc a;
                acc_init(P, cb, a);
                for (int j = j0 + (int)lane; j < j1; j += 32)
                    acc_row(P, s_off, cb, a, srows + (size_t)order[soff[s] + j] * D.row_bytes);
                acc_team_sum(P, cb, a, 32);
                if (lane == 0) {
                    uint8_t *rec = T.states + (size_t)sgid[s] * P.rec;
                    if (m > kSegRows) acc_merge_atomic(P, cb, a, rec);
                    else acc_merge(P, cb, a, rec);
                }
            }
            // team keys from the warp after the warp keys' last one, one-lane
            // keys from the last warp down: the classes fall on different warps
            constexpr int kTeams = 32 / kTeamLanes;
            const int team = (int)(lane / kTeamLanes), tl = (int)(lane % kTeamLanes);
            const int twarp = (int)((warp + kWarps - (unsigned)(nseg % kWarps)) % kWarps);
            for (int u0 = twarp * kTeams; u0 < nt; u0 += kWarps * kTeams) {  // a team per key
                const int u = u0 + team;
                RowAcc a;
                acc_init(P, cb, a);
                int s = -1;
                if (u < nt) {
                    s = big[kChunkRows - 1 - u];
                    const int first = soff[s], m = (int)scnt[s];
                    for (int j = tl; j < m; j += kTeamLanes)
                        acc_row(P, s_off, cb, a, srows + (size_t)order[first + j] * D.row_bytes);
                }
                acc_team_sum(P, cb, a, kTeamLanes);
                if (tl == 0 && s >= 0) acc_merge(P, cb, a, T.states + (size_t)sgid[s] * P.rec);
            }
            for (int u = (int)(blockDim.x - 1 - threadIdx.x); u < n1; u += blockDim.x) {  // a lane per key
                const int s = small[u];
                const int first = soff[s], m = (int)scnt[s];
                RowAcc a;
                acc_init(P, cb, a);
                for (int j = 0; j < m; j++) acc_row(P, s_off, cb, a, srows + (size_t)order[first + j] * D.row_bytes);
                acc_merge(P, cb, a, T.states + (size_t)sgid[s] * P.rec);
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) D.start[p] = rows;
}

// Group ids of the hot keys (inserted into the global table), then the NULL
// and the marker group.
__global__ void hot_gid_kernel(AggPlanDev P, TableDev T, const long long *hot_keys, int H, uint32_t *hot_gids) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < H + 2; j += gridDim.x * blockDim.x)
        hot_gids[j] = j < H ? find_or_insert(T, P, hot_keys[j]) : (j == H ? kNullGid : kMarkerGid);
}

__global__ void init_special_kernel(AggPlanDev P, uint8_t *states) {
    if (threadIdx.x < 2) init_record(P, states + (size_t)threadIdx.x * P.rec);
}

// Re-inserts the (key, group id) pairs of an old table into a bigger one.
__global__ void rehash_kernel(const long long *okeys, const uint32_t *ogids, uint64_t on, long long *nkeys,
                              uint32_t *ngids, uint64_t nmask) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < on; i += (uint64_t)gridDim.x * blockDim.x) {
        const long long k = okeys[i];
        if (k == kEmptyKey) continue;
        uint64_t pos = hash_word((uint64_t)k) & nmask;
        for (uint64_t p = 0; p <= nmask; p++) {
            const unsigned long long old =
                atomicCAS(reinterpret_cast<unsigned long long *>(nkeys + pos), (unsigned long long)kEmptyKey,
                          (unsigned long long)k);
            if (old == (unsigned long long)kEmptyKey) {
                ngids[pos] = ogids[i];
                break;
            }
            pos = (pos + 1) & nmask;
        }
    }
}

// ---- results -------------------------------------------------------------------
// Output functions beyond KRV_AGG_*: the state columns of a partial
// aggregate and the merges of state columns.
enum : int32_t {
    F_SUM_AS_F64 = 100,  // AVG's partial sum of a non-decimal column, as float64
    F_NONEMPTY = 101,    // a decimal SUM's partial "nonempty" flag (Boolean)
    F_COUNT_MERGE = 102, // COUNT over count states: their sum
    F_AVG_MERGE = 103,   // AVG over (sum, count) states
};
struct OutExprDev {
    int32_t func;
    int32_t col;      // value column index in the plan (-1: COUNT(*))
    int32_t aux;      // SUM of decimal states: the overflowed-state count; AVG merge: the counts (-1: none)
    int32_t otype;    // result Type
    int32_t rp, rs;   // result precision/scale (decimals)
    int32_t in_type;
    int32_t in_scale;
    int32_t ansi;
    void *dst;
    uint32_t *dst_valid;
};
constexpr int kMaxExprs = KRV_MAX_AGGREGATES;
struct OutPlanDev {
    OutExprDev e[kMaxExprs];
    int32_t n;
    int32_t nspecial;
    uint32_t special[2];
};

__device__ __forceinline__ unsigned __int128 pow10_u128(int p) {
    unsigned __int128 v = 1;
    for (int i = 0; i < p && i < 38; i++) v *= 10;
    return v;
}

// avg_decimal (helpers.rs:539-590): HALF_UP to scale 39, then HALF_UP to s.
__device__ bool avg_decimal_slow(__int128 sum, int ss, long long count, int p, int s, __int128 &out) {
    const bool negative = (sum < 0) != (count < 0);
    const unsigned __int128 a = sum < 0 ? (unsigned __int128)(-sum) : (unsigned __int128)sum;
    const unsigned __int128 b = (unsigned __int128)(count < 0 ? -(__int128)count : (__int128)count);
    unsigned __int128 in = a / b, rem = a % b;
    const int nfrac = 39 - ss;
    uint8_t frac[40];
    for (int i = 0; i < nfrac; i++) {
        rem *= 10;
        frac[i] = (uint8_t)(rem / b);
        rem %= b;
    }
    rem *= 10;
    if ((uint8_t)(rem / b) >= 5) {
        int i = nfrac - 1;
        bool carry = true;
        while (i >= 0 && carry) {
            if (frac[i] == 9) frac[i] = 0;
            else {
                frac[i]++;
                carry = false;
            }
            i--;
        }
        if (carry) in += 1;
    }
    int keep = s - ss;
    if (keep < 0) keep = 0;
    const bool up = keep < nfrac && frac[keep] >= 5;
    unsigned __int128 v = in;
    const unsigned __int128 lim = ((unsigned __int128)1) << 126;
    for (int i = 0; i < keep; i++) {
        if (v > lim / 10) return false;
        v = v * 10 + frac[i];
    }
    v += up ? 1 : 0;
    if (v >= pow10_u128(p)) return false;
    out = negative ? -(__int128)v : (__int128)v;
    return true;
}

// avg_fast (helpers.rs:595-610): one HALF_UP division when the result scale is
// at most 19 and not below the sum's; else the digit loop.
__device__ bool avg_decimal(__int128 sum, int ss, long long count, int p, int s, __int128 &out) {
    if (count == 0) return false;
    if (s <= 19 && s >= ss) {
        const unsigned __int128 mag = sum < 0 ? (unsigned __int128)(-sum) : (unsigned __int128)sum;
        const unsigned __int128 mul = pow10_u128(s - ss);
        if (mag <= (~(unsigned __int128)0) / mul) {
            const unsigned __int128 nn = mag * mul;
            const unsigned __int128 d = (unsigned __int128)(count < 0 ? -(__int128)count : (__int128)count);
            unsigned __int128 q = nn / d;
            const unsigned __int128 r = nn % d;
            q += (r >= d - r) ? 1 : 0;
            if (q >= pow10_u128(p)) return false;
            out = ((sum < 0) != (count < 0)) ? -(__int128)q : (__int128)q;
            return true;
        }
    }
    return avg_decimal_slow(sum, ss, count, p, s, out);
}

__global__ void __launch_bounds__(256) finalize_kernel(AggPlanDev P, OutPlanDev O, const uint8_t *states,
                                                       const long long *gkeys, int64_t nout, int key_width,
                                                       void *key_out, uint32_t *key_valid, uint32_t *status) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t base = blockIdx.x * (int64_t)blockDim.x; base < nout; base += stride) {
        const int64_t r = base + threadIdx.x;
        const bool live = r < nout;
        uint32_t g = 0;
        if (live) g = r < O.nspecial ? O.special[r] : (uint32_t)(r - O.nspecial + kFirstGid);
        const uint8_t *rec = states + (size_t)g * P.rec;
        // Group key.
        bool kv = live && g != kNullGid;
        if (live) {
            const long long k = g == kNullGid ? 0 : g == kMarkerGid ? kEmptyKey : gkeys[g];
            if (key_width == 4) static_cast<int *>(key_out)[r] = (int)k;
            else static_cast<long long *>(key_out)[r] = k;
        }
        if (key_valid) {
            const unsigned w = __ballot_sync(0xFFFFFFFFu, kv);
            if ((threadIdx.x & 31) == 0 && live) key_valid[r >> 5] = w;
        }
        for (int e = 0; e < O.n; e++) {
            const OutExprDev &X = O.e[e];
            bool valid = false, bit = false;
            if (live) {
                const unsigned long long rows = *reinterpret_cast<const unsigned long long *>(rec + P.off_rows);
                // the states of an overflowed decimal sum seen in this group
                const long long poisoned = X.aux >= 0 && X.func != F_AVG_MERGE
                                               ? *reinterpret_cast<const long long *>(rec + P.c[X.aux].off_sum)
                                               : 0;
                if (X.func == KRV_AGG_COUNT_STAR) {
                    static_cast<long long *>(X.dst)[r] = (long long)rows;
                    valid = true;
                } else if (X.func == F_COUNT_MERGE) {
                    static_cast<long long *>(X.dst)[r] = *reinterpret_cast<const long long *>(rec + P.c[X.col].off_sum);
                    valid = true;
                } else if (X.func == F_NONEMPTY) {
                    const unsigned long long cnt =
                        *reinterpret_cast<const unsigned long long *>(rec + P.c[X.col].off_count);
                    bit = cnt > 0 || poisoned > 0;
                    valid = true;
                } else if (X.func == F_AVG_MERGE) {
                    const AggColDev &C = P.c[X.col];
                    const long long cnt = *reinterpret_cast<const long long *>(rec + P.c[X.aux].off_sum);
                    if (cnt > 0 && C.type == (int)Type::F64) {
                        const double hi = *reinterpret_cast<const double *>(rec + C.off_sum);
                        const double lo = *reinterpret_cast<const double *>(rec + C.off_sum + 8);
                        static_cast<double *>(X.dst)[r] = __ddiv_rn(isfinite(hi) ? __dadd_rn(hi, lo) : hi, (double)cnt);
                        valid = true;
                    } else if (cnt > 0) {
                        const unsigned long long lo = *reinterpret_cast<const unsigned long long *>(rec + C.off_sum);
                        const long long hi = *reinterpret_cast<const long long *>(rec + C.off_sum + 8);
                        const __int128 sum = (__int128)(((unsigned __int128)(unsigned long long)hi << 64) | lo);
                        __int128 v = 0;
                        if (avg_decimal(sum, X.in_scale, cnt, X.rp, X.rs, v)) {
                            if (X.otype == (int)Type::Dec64) static_cast<long long *>(X.dst)[r] = (long long)v;
                            else {
                                long long *d = static_cast<long long *>(X.dst) + 2 * r;
                                d[0] = (long long)(unsigned long long)v;
                                d[1] = (long long)(v >> 64);
                            }
                            valid = true;
                        } else if (X.ansi) {
                            atomicOr(status, ST_OVERFLOW);
                        }
                    }
                    if (!valid) {
                        if (X.otype == (int)Type::Dec128) {
                            static_cast<long long *>(X.dst)[2 * r] = 0;
                            static_cast<long long *>(X.dst)[2 * r + 1] = 0;
                        } else {
                            static_cast<long long *>(X.dst)[r] = 0;
                        }
                    }
                } else {
                    const AggColDev &C = P.c[X.col];
                    const unsigned long long cnt = *reinterpret_cast<const unsigned long long *>(rec + C.off_count);
                    if (X.func == KRV_AGG_COUNT) {
                        static_cast<long long *>(X.dst)[r] = (long long)cnt;
                        valid = true;
                    } else if (X.func == F_SUM_AS_F64 && cnt > 0) {
                        const bool i32 = C.type == (int)Type::I32 || C.type == (int)Type::Date32;
                        double v;
                        if (C.type == (int)Type::F64) {
                            const double hi = *reinterpret_cast<const double *>(rec + C.off_sum);
                            const double lo = *reinterpret_cast<const double *>(rec + C.off_sum + 8);
                            v = isfinite(hi) ? __dadd_rn(hi, lo) : hi;
                        } else if (i32) {
                            v = (double)*reinterpret_cast<const long long *>(rec + C.off_sum);
                        } else {
                            const unsigned long long lo = *reinterpret_cast<const unsigned long long *>(rec + C.off_sum);
                            const long long hi = *reinterpret_cast<const long long *>(rec + C.off_sum + 8);
                            const bool fits64 = (hi == 0 && !(lo >> 63)) || (hi == -1 && (lo >> 63));
                            v = fits64 ? (double)(long long)lo : (double)hi * 18446744073709551616.0 + (double)lo;
                        }
                        static_cast<double *>(X.dst)[r] = v;
                        valid = true;
                    } else if (X.func == F_SUM_AS_F64) {
                        static_cast<double *>(X.dst)[r] = 0.0;
                    } else if (poisoned > 0) {
                        // a state's sum overflowed: NULL, or the ANSI error
                        if (X.ansi) atomicOr(status, ST_OVERFLOW);
                        if (X.otype == (int)Type::Dec128) {
                            static_cast<long long *>(X.dst)[2 * r] = 0;
                            static_cast<long long *>(X.dst)[2 * r + 1] = 0;
                        } else {
                            static_cast<long long *>(X.dst)[r] = 0;
                        }
                    } else if (cnt > 0) {
                        const bool i32 = C.type == (int)Type::I32 || C.type == (int)Type::Date32;
                        if (X.func == KRV_AGG_MIN || X.func == KRV_AGG_MAX) {
                            const int off = X.func == KRV_AGG_MIN ? C.off_min : C.off_max;
                            if (C.flags & F_WIDE) {
                                const long long *m = reinterpret_cast<const long long *>(rec + off);
                                static_cast<long long *>(X.dst)[2 * r] = m[0];
                                static_cast<long long *>(X.dst)[2 * r + 1] = m[1];
                            } else if (i32) static_cast<int *>(X.dst)[r] = *reinterpret_cast<const int *>(rec + off);
                            else if (C.type == (int)Type::F64)
                                static_cast<double *>(X.dst)[r] =
                                    f64_from_order_key(*reinterpret_cast<const unsigned long long *>(rec + off));
                            else if (X.otype == (int)Type::Dec128) {
                                const long long v = *reinterpret_cast<const long long *>(rec + off);
                                static_cast<long long *>(X.dst)[2 * r] = v;
                                static_cast<long long *>(X.dst)[2 * r + 1] = v < 0 ? -1 : 0;
                            } else static_cast<long long *>(X.dst)[r] = *reinterpret_cast<const long long *>(rec + off);
                            valid = true;
                        } else if (C.type == (int)Type::F64) {
                            const double hi = *reinterpret_cast<const double *>(rec + C.off_sum);
                            const double lo = *reinterpret_cast<const double *>(rec + C.off_sum + 8);
                            double s = isfinite(hi) ? __dadd_rn(hi, lo) : hi;
                            if (X.func == KRV_AGG_AVG) s = __ddiv_rn(s, (double)cnt);
                            static_cast<double *>(X.dst)[r] = s;
                            valid = true;
                        } else if (i32) {
                            const long long s = *reinterpret_cast<const long long *>(rec + C.off_sum);
                            if (X.func == KRV_AGG_SUM) static_cast<long long *>(X.dst)[r] = s;
                            else static_cast<double *>(X.dst)[r] = __ddiv_rn((double)s, (double)cnt);
                            valid = true;
                        } else {
                            const unsigned long long lo = *reinterpret_cast<const unsigned long long *>(rec + C.off_sum);
                            const long long hi = *reinterpret_cast<const long long *>(rec + C.off_sum + 8);
                            const __int128 sum = (__int128)(((unsigned __int128)(unsigned long long)hi << 64) | lo);
                            const bool fits64 = (hi == 0 && !(lo >> 63)) || (hi == -1 && (lo >> 63));
                            if (C.type == (int)Type::I64) {
                                if (X.func == KRV_AGG_SUM) {
                                    // SumInt: ANSI raises on overflow, else wraps (two's complement).
                                    if (!fits64 && X.ansi) atomicOr(status, ST_OVERFLOW);
                                    static_cast<long long *>(X.dst)[r] = (long long)lo;
                                    valid = true;
                                } else {
                                    const double s = fits64 ? (double)(long long)lo
                                                            : (double)hi * 18446744073709551616.0 + (double)lo;
                                    static_cast<double *>(X.dst)[r] = __ddiv_rn(s, (double)cnt);
                                    valid = true;
                                }
                            } else {
                                __int128 v = sum;
                                bool ok = true;
                                if (X.func == KRV_AGG_SUM) {
                                    const unsigned __int128 mag = sum < 0 ? (unsigned __int128)(-sum) : (unsigned __int128)sum;
                                    ok = mag < pow10_u128(X.rp);
                                } else {
                                    ok = avg_decimal(sum, X.in_scale, (long long)cnt, X.rp, X.rs, v);
                                }
                                if (!ok) {
                                    if (X.ansi) atomicOr(status, ST_OVERFLOW);
                                } else {
                                    if (X.otype == (int)Type::Dec64) static_cast<long long *>(X.dst)[r] = (long long)v;
                                    else {
                                        long long *d = static_cast<long long *>(X.dst) + 2 * r;
                                        d[0] = (long long)(unsigned long long)v;
                                        d[1] = (long long)(v >> 64);
                                    }
                                    valid = true;
                                }
                                if (!ok) {
                                    if (X.otype == (int)Type::Dec64) static_cast<long long *>(X.dst)[r] = 0;
                                    else {
                                        long long *d = static_cast<long long *>(X.dst) + 2 * r;
                                        d[0] = 0;
                                        d[1] = 0;
                                    }
                                }
                            }
                        }
                    } else {
                        // No non-NULL input: NULL result with a zeroed value.
                        const int w = X.otype == (int)Type::Dec128 ? 16
                                      : (X.otype == (int)Type::I32 || X.otype == (int)Type::Date32) ? 4
                                                                                                     : 8;
                        if (w == 4) static_cast<int *>(X.dst)[r] = 0;
                        else if (w == 8) static_cast<long long *>(X.dst)[r] = 0;
                        else {
                            static_cast<long long *>(X.dst)[2 * r] = 0;
                            static_cast<long long *>(X.dst)[2 * r + 1] = 0;
                        }
                    }
                }
            }
            if (X.func == F_NONEMPTY) {  // Boolean data: one bit per row
                const unsigned w = __ballot_sync(0xFFFFFFFFu, bit);
                if ((threadIdx.x & 31) == 0 && live) static_cast<uint32_t *>(X.dst)[r >> 5] = w;
            }
            if (X.dst_valid) {
                const unsigned w = __ballot_sync(0xFFFFFFFFu, valid);
                if ((threadIdx.x & 31) == 0 && live) X.dst_valid[r >> 5] = w;
            }
        }
    }
}

// The overflowed decimal SUM states of a batch: 1 where the state's sum is
// NULL but its `nonempty` flag is set (Boolean data, bit i = row i).
__global__ void poison_kernel(const uint8_t *sum_valid, int64_t sum_voff, const uint8_t *nonempty,
                              int64_t nonempty_off, int64_t n, long long *out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (!bit_get(sum_valid, sum_voff, i) && bit_get(nonempty, nonempty_off, i)) ? 1 : 0;
}

}  // namespace

class HashAggregate {
  public:
    HashAggregate(Runtime *rt, const krv_agg_spec &spec);
    void push(const DevBatch &b);
    void finish() { finished_ = true; }
    DevBatch result();
    int64_t groups() const { return known_groups_; }

  private:
    void plan(const DevBatch &b);
    void alloc_table(uint64_t slots);
    void grow(uint64_t need_groups);
    void launch(const DevBatch &b, const KeyIn &key, int64_t n, const uint32_t *rows_idx, uint32_t *ovf,
                unsigned long long *ovf_count);

    Runtime *rt_;
    krv_agg_spec spec_;
    bool planned_ = false, finished_ = false;
    // Group keys other than one int32/int64/date32/decimal(18) column: the
    // dictionary gives each key a dense int64 code, appended to every batch
    // as column key_col_ and aggregated as the key.
    KeyDict *dict_ = nullptr;
    std::vector<KeyDict *> vdicts_;  // per plan column: the value dictionary of a string MIN/MAX column
    std::vector<int> dict_cols_;
    int key_col_ = -1;
    // Plan columns of each aggregate (col, aux: see OutExprDev) and the
    // (sum, nonempty) columns of the decimal SUM states whose overflow flags
    // are appended to every batch after the code column.
    std::vector<int> expr_col_, expr_aux_;
    std::vector<std::pair<int, int>> poison_src_;

  public:
    ~HashAggregate() {
        if (dict_) key_dict_destroy(dict_);
        for (KeyDict *d : vdicts_)
            if (d) key_dict_destroy(d);
    }

  private:
    AggPlanDev P_{};
    std::vector<int> value_cols_;  // input column of each plan column
    std::vector<DType> input_types_;
    std::vector<std::string> input_names_;
    DType key_type_;
    std::string key_name_;
    DBuf keys_, gids_, states_, gkeys_, ngroups_;
    uint64_t slots_ = 0;
    unsigned long long limit_ = 0;
    int64_t known_groups_ = 2;     // exact after a sync
    int64_t pending_rows_ = 0;     // rows pushed since known_groups_ was read
    int mode_ = KRV_AGG_MODE_SHARED;
    int smem_entries_ = 0;
    // The hottest keys of the first batch (a strided sample), aggregated in
    // warp-private records by the shared-memory kernel.
    void sample_hot(const KeyIn &key, int64_t n);
    bool sampled_ = false;
    DBuf hot_;
    int hot_count_ = 0;
    // The partitioned path (agg_split_kernel + agg_part_kernel) for large
    // batches: its hot keys, their group ids and the estimate of distinct
    // keys, taken from the first large batch.
    bool use_partitioned(int64_t n) const;
    void push_partitioned(const DevBatch &b, const KeyIn &key, int64_t n);
    void plan_partitioned(const KeyIn &key, int64_t n);
    void plan_row_records();
    // Groups from unindexed_from_ on (when >= 0) have keys and records but no
    // hash table entry yet (agg_part_kernel appends them); index_pending
    // inserts them before anything looks keys up or rehashes the table.
    int64_t unindexed_from_ = -1;
    void index_pending();
    // agg_part_kernel's bound on new group ids: the table's limit, less the
    // ids that the resident CTAs may take past a check they passed together.
    uint64_t part_id_room(int part_blocks) const { return (uint64_t)part_blocks * rt_->sm_count * kChunkRows; }
    unsigned long long part_id_limit(int part_blocks) const {
        const uint64_t room = part_id_room(part_blocks), cap = slots_ / 8 * 7;
        return cap > room ? std::min<unsigned long long>(limit_, cap - room) : 0ull;
    }
    bool part_planned_ = false;
    DBuf part_hot_keys_, part_hot_gids_, part_hot_tab_, part_hot_tab_idx_;
    int part_hot_slots_ = 0;
    int part_hot_ = 0;
    double part_cold_frac_ = 1.0;
    int64_t part_groups_est_ = 0;
    int part_row_bytes_ = 0;
    int16_t part_off_val_[kMaxValueCols] = {};
};

HashAggregate::HashAggregate(Runtime *rt, const krv_agg_spec &spec) : rt_(rt), spec_(spec) {
    if (spec.n_group_by < 1 || spec.n_group_by > KRV_MAX_GROUP_KEYS)
        fail(KRV_UNSUPPORTED, "the GPU aggregate groups by 1 to 8 key columns");
    if (spec.n_aggregates < 0 || spec.n_aggregates > KRV_MAX_AGGREGATES)
        fail(KRV_INVALID_ARGUMENT, "aggregate count out of range");
    for (int e = 0; e < spec.n_aggregates; e++)
        if (spec.aggregates[e].function < KRV_AGG_COUNT_STAR || spec.aggregates[e].function > KRV_AGG_AVG)
            fail(KRV_UNSUPPORTED, "aggregate function " + std::to_string(spec.aggregates[e].function));
    mode_ = spec.mode == KRV_AGG_MODE_GLOBAL ? KRV_AGG_MODE_GLOBAL : KRV_AGG_MODE_SHARED;
}

void HashAggregate::plan(const DevBatch &b) {
    for (int k = 0; k < spec_.n_group_by; k++)
        if (spec_.group_by[k] < 0 || spec_.group_by[k] >= (int)b.cols.size())
            fail(KRV_INVALID_ARGUMENT, "group-by column out of range");
    const int kc = spec_.group_by[0];
    const Type t0 = b.cols[kc].type.id;
    if (spec_.n_group_by == 1 && (t0 == Type::I32 || t0 == Type::I64 || t0 == Type::Date32 || t0 == Type::Dec64)) {
        key_col_ = kc;
        key_type_ = b.cols[kc].type;
        key_name_ = b.cols[kc].name;
    } else {
        std::vector<DevCol> meta;
        for (int k = 0; k < spec_.n_group_by; k++) {
            dict_cols_.push_back(spec_.group_by[k]);
            DevCol m;
            m.type = b.cols[spec_.group_by[k]].type;
            m.name = b.cols[spec_.group_by[k]].name;
            m.nullable = b.cols[spec_.group_by[k]].nullable || b.cols[spec_.group_by[k]].valid;
            meta.push_back(m);
        }
        dict_ = make_key_dict(rt_, meta);
        key_col_ = (int)b.cols.size();
        key_type_ = DType{Type::I64, 0, 0};
        key_name_ = "#group";
    }
    for (const DevCol &c : b.cols) {
        input_types_.push_back(c.type);
        input_names_.push_back(c.name);
    }
    // One plan column per distinct input column; flags from its aggregates.
    // Merges of decimal SUM states add a hidden int64 column per state pair:
    // 1 where the state overflowed (its sum NULL, its nonempty flag set).
    const int hidden_base = (int)b.cols.size() + (dict_ ? 1 : 0);
    std::vector<int32_t> flags;
    auto type_of = [&](int col) -> DType {
        if (col >= hidden_base) return DType{Type::I64, 0, 0};
        // a UTF-8 / binary column: for MIN/MAX its value dictionary's int64
        // codes; counted by COUNT alone, its int32 offsets stand in for values
        // (never read: only the validity counts)
        if (b.cols[col].type.var()) {
            for (size_t i = 0; i < value_cols_.size(); i++)
                if (value_cols_[i] == col && (flags[i] & F_STR)) return DType{Type::I64, 0, 0};
            return DType{Type::I32, 0, 0};
        }
        return b.cols[col].type;
    };
    P_.ncols = 0;
    auto plan_col = [&](int col, int32_t flag) -> int {
        int at = -1;
        for (size_t i = 0; i < value_cols_.size(); i++)
            if (value_cols_[i] == col) at = (int)i;
        if (at < 0) {
            if ((int)value_cols_.size() == kMaxValueCols) fail(KRV_UNSUPPORTED, "more than 16 aggregated columns");
            value_cols_.push_back(col);
            flags.push_back(0);
            at = (int)value_cols_.size() - 1;
        }
        flags[at] |= flag;
        return at;
    };
    auto check_col = [&](int col) {
        if (col < 0 || col >= (int)b.cols.size()) fail(KRV_INVALID_ARGUMENT, "aggregate column out of range");
        const DType t = b.cols[col].type;
        if (t.id == Type::Bool || t.id == Type::U8 || t.var()) fail(KRV_UNSUPPORTED, "aggregate over " + t.format());
        return t;
    };
    // COUNT(column) also takes UTF-8 and binary columns (AggregateFunction::Count
    // counts the non-NULL values of any type, aggregate/mod.rs:134)
    auto check_counted = [&](int col) {
        if (col < 0 || col >= (int)b.cols.size()) fail(KRV_INVALID_ARGUMENT, "aggregate column out of range");
        if (!b.cols[col].type.var()) check_col(col);
    };
    expr_col_.assign(spec_.n_aggregates, -1);
    expr_aux_.assign(spec_.n_aggregates, -1);
    for (int e = 0; e < spec_.n_aggregates; e++) {
        const krv_agg_expr &x = spec_.aggregates[e];
        const bool state = x.input == KRV_AGG_INPUT_STATE;
        if (x.input != KRV_AGG_INPUT_RAW && !state) fail(KRV_INVALID_ARGUMENT, "unknown aggregate input");
        if (!state) {
            if (x.function == KRV_AGG_COUNT_STAR) continue;
            const bool var_arg = x.column >= 0 && x.column < (int)b.cols.size() && b.cols[x.column].type.var();
            if (x.function == KRV_AGG_COUNT && var_arg) {
                check_counted(x.column);
                expr_col_[e] = plan_col(x.column, 0);
                continue;
            }
            if ((x.function == KRV_AGG_MIN || x.function == KRV_AGG_MAX) && var_arg) {
                expr_col_[e] = plan_col(x.column, (x.function == KRV_AGG_MIN ? F_MIN : F_MAX) | F_STR);
                continue;
            }
            const DType t = check_col(x.column);
            int32_t f = 0;
            if (x.function == KRV_AGG_SUM || x.function == KRV_AGG_AVG) f = F_SUM;
            if (x.function == KRV_AGG_MIN) f = F_MIN;
            if (x.function == KRV_AGG_MAX) f = F_MAX;
            if (t.id == Type::Dec128 && t.precision > 18 && (f & (F_MIN | F_MAX))) f |= F_WIDE;
            expr_col_[e] = plan_col(x.column, f);
            continue;
        }
        // Partial states (AggregateExpr::merging, aggregate/mod.rs:561-569).
        if ((x.function == KRV_AGG_MIN || x.function == KRV_AGG_MAX) && x.column >= 0 &&
            x.column < (int)b.cols.size() && b.cols[x.column].type.var()) {
            expr_col_[e] = plan_col(x.column, (x.function == KRV_AGG_MIN ? F_MIN : F_MAX) | F_STR);
            continue;
        }
        const DType t = check_col(x.column);
        const bool dec = t.id == Type::Dec64 || t.id == Type::Dec128;
        switch (x.function) {
        case KRV_AGG_COUNT_STAR:
        case KRV_AGG_COUNT:
            if (t.id != Type::I64) fail(KRV_INVALID_ARGUMENT, "a COUNT state is an int64 column");
            expr_col_[e] = plan_col(x.column, F_SUM);
            break;
        case KRV_AGG_SUM:
            expr_col_[e] = plan_col(x.column, F_SUM);
            if (dec) {
                if (x.column2 < 0 || x.column2 >= (int)b.cols.size() || b.cols[x.column2].type.id != Type::Bool)
                    fail(KRV_INVALID_ARGUMENT, "a decimal SUM state is (sum, nonempty Boolean)");
                poison_src_.push_back({x.column, x.column2});
                expr_aux_[e] = plan_col(hidden_base + (int)poison_src_.size() - 1, F_SUM);
            }
            break;
        case KRV_AGG_AVG:
            if (!dec && t.id != Type::F64) fail(KRV_INVALID_ARGUMENT, "an AVG state's sum is decimal or float64");
            if (x.column2 < 0 || check_col(x.column2).id != Type::I64)
                fail(KRV_INVALID_ARGUMENT, "an AVG state is (sum, int64 count)");
            expr_col_[e] = plan_col(x.column, F_SUM);
            expr_aux_[e] = plan_col(x.column2, F_SUM);
            break;
        case KRV_AGG_MIN:
        case KRV_AGG_MAX:
            expr_col_[e] = plan_col(x.column, (x.function == KRV_AGG_MIN ? F_MIN : F_MAX) |
                                                  (t.id == Type::Dec128 && t.precision > 18 ? F_WIDE : 0));
            break;
        }
    }
    // Record layout: 16-byte sums first, then 8-byte fields, then 4-byte ones.
    int off = 0;
    P_.ncols = (int)value_cols_.size();
    for (int c = 0; c < P_.ncols; c++) {
        const DType t = type_of(value_cols_[c]);
        AggColDev &C = P_.c[c];
        C.type = (int)t.id;
        C.flags = flags[c];
        C.off_count = C.off_sum = C.off_min = C.off_max = -1;
        const bool wide = t.id == Type::I64 || t.id == Type::Dec64 || t.id == Type::Dec128 || t.id == Type::F64;
        if ((C.flags & F_SUM) && wide) {
            C.off_sum = off;
            off += 16;
        }
        if (C.flags & F_WIDE) {  // 128-bit MIN/MAX: 16-byte aligned pairs
            if (C.flags & F_MIN) {
                C.off_min = off;
                off += 16;
            }
            if (C.flags & F_MAX) {
                C.off_max = off;
                off += 16;
            }
        }
    }
    P_.off_rows = off;
    off += 8;
    for (int c = 0; c < P_.ncols; c++) {
        AggColDev &C = P_.c[c];
        const bool i32 = C.type == (int)Type::I32 || C.type == (int)Type::Date32;
        C.off_count = off;
        off += 8;
        if ((C.flags & F_SUM) && i32) {
            C.off_sum = off;
            off += 8;
        }
        if (!i32 && !(C.flags & F_WIDE)) {
            if (C.flags & F_MIN) {
                C.off_min = off;
                off += 8;
            }
            if (C.flags & F_MAX) {
                C.off_max = off;
                off += 8;
            }
        }
    }
    for (int c = 0; c < P_.ncols; c++) {
        AggColDev &C = P_.c[c];
        const bool i32 = C.type == (int)Type::I32 || C.type == (int)Type::Date32;
        if (i32) {
            if (C.flags & F_MIN) {
                C.off_min = off;
                off += 4;
            }
            if (C.flags & F_MAX) {
                C.off_max = off;
                off += 4;
            }
        }
    }
    P_.rec = (off + 15) & ~15;
    // Shared-memory entries: the largest power of two whose records, keys
    // and ids fit the opt-in shared memory of one CTA.
    const int per = P_.rec + 12;
    int e = 1;
    while ((e * 2) * per + 64 <= std::min(rt_->max_smem_optin, 200 * 1024)) e *= 2;
    smem_entries_ = e >= 64 ? e : 0;
    if (smem_entries_ == 0) mode_ = KRV_AGG_MODE_GLOBAL;
    for (int c = 0; c < P_.ncols; c++)
        if (P_.c[c].flags & (F_WIDE | F_STR)) mode_ = KRV_AGG_MODE_GLOBAL;  // 128-bit or string MIN/MAX: global kernels
    // a value dictionary per string MIN/MAX column
    vdicts_.assign(P_.ncols, nullptr);
    for (int c = 0; c < P_.ncols; c++)
        if (P_.c[c].flags & F_STR) {
            DevCol m;
            m.type = b.cols[value_cols_[c]].type;
            m.name = b.cols[value_cols_[c]].name;
            m.nullable = true;
            vdicts_[c] = make_key_dict(rt_, {m});
        }
    plan_row_records();
    const uint64_t hint = spec_.expected_groups > 0 ? (uint64_t)spec_.expected_groups : 65536;
    alloc_table(std::max<uint64_t>(1024, next_pow2((uint64_t)(hint * 2))));
    planned_ = true;
}

void HashAggregate::alloc_table(uint64_t slots) {
    slots_ = slots;
    limit_ = (unsigned long long)(slots * 3 / 4);
    keys_ = DBuf(rt_, slots * 8);
    gids_ = DBuf(rt_, slots * 4);
    KRV_CUDA(cudaMemsetAsync(keys_.get(), 0x80, slots * 8, rt_->stream));
    KRV_CUDA(cudaMemsetAsync(gids_.get(), 0xFF, slots * 4, rt_->stream));
    const size_t gcap = slots + kFirstGid;
    DBuf states(rt_, gcap * (size_t)P_.rec);
    DBuf gkeys(rt_, gcap * 8);
    if (states_.get()) {
        KRV_CUDA(cudaMemcpyAsync(states.get(), states_.get(), (size_t)known_groups_ * P_.rec, cudaMemcpyDeviceToDevice,
                                 rt_->stream));
        KRV_CUDA(cudaMemcpyAsync(gkeys.get(), gkeys_.get(), (size_t)known_groups_ * 8, cudaMemcpyDeviceToDevice,
                                 rt_->stream));
    } else {
        init_special_kernel<<<1, 32, 0, rt_->stream>>>(P_, states.as<uint8_t>());
        rt_->launches++;
        check_launch("init_special_kernel");
        ngroups_ = DBuf(rt_, 8);
        const unsigned long long first = kFirstGid;
        KRV_CUDA(cudaMemcpyAsync(ngroups_.get(), &first, 8, cudaMemcpyHostToDevice, rt_->stream));
        KRV_CUDA(cudaStreamSynchronize(rt_->stream));
    }
    states_ = std::move(states);
    gkeys_ = std::move(gkeys);
}

void HashAggregate::grow(uint64_t need_groups) {
    // the records to carry over: every group the device has handed out
    known_groups_ = (int64_t)read_scalar<unsigned long long>(rt_, ngroups_.get());
    pending_rows_ = 0;
    DBuf okeys = std::move(keys_), ogids = std::move(gids_);
    const uint64_t oslots = slots_;
    uint64_t ns = next_pow2(std::max<uint64_t>(oslots * 2, need_groups * 2));
    alloc_table(ns);
    rehash_kernel<<<grid_for(rt_, (int64_t)oslots, 256, 8), 256, 0, rt_->stream>>>(
        okeys.as<long long>(), ogids.as<uint32_t>(), oslots, keys_.as<long long>(), gids_.as<uint32_t>(), slots_ - 1);
    rt_->launches++;
    check_launch("rehash_kernel");
    index_pending();
}

void HashAggregate::index_pending() {
    if (unindexed_from_ < 0) return;
    const uint64_t from = (uint64_t)unindexed_from_;
    const uint64_t to = read_scalar<unsigned long long>(rt_, ngroups_.get());
    unindexed_from_ = -1;
    if (to <= from) return;
    index_groups_kernel<<<grid_for(rt_, (int64_t)(to - from), 256, 8), 256, 0, rt_->stream>>>(
        gkeys_.as<long long>(), from, to, keys_.as<long long>(), gids_.as<uint32_t>(), slots_ - 1);
    rt_->launches++;
    check_launch("index_groups_kernel");
}

void HashAggregate::launch(const DevBatch &b, const KeyIn &key, int64_t n, const uint32_t *rows_idx, uint32_t *ovf,
                           unsigned long long *ovf_count) {
    AggPlanDev P = P_;
    for (int c = 0; c < P.ncols; c++) {
        const DevCol &col = b.cols[value_cols_[c]];
        P.c[c].data = col.data;
        P.c[c].valid = col.valid;
        P.c[c].voff = col.valid_off;
    }
    TableDev T{keys_.as<long long>(), gids_.as<uint32_t>(), slots_ - 1, states_.as<uint8_t>(), gkeys_.as<long long>(),
               ngroups_.as<unsigned long long>(), limit_, status_word(rt_)};
    if (mode_ == KRV_AGG_MODE_SHARED) {
        const int E = smem_entries_;
        // as many hot keys as the shared memory left beside the table holds
        const int64_t room = (int64_t)rt_->max_smem_optin - 1024 - (int64_t)E * (P.rec + 12) - 16;
        const int H = (int)std::max<int64_t>(0, std::min<int64_t>(hot_count_, room / ((kAggThreads / 32) * P.rec)));
        const size_t smem = (size_t)E * (P.rec + 12) + 16 + (size_t)(kAggThreads / 32) * H * P.rec;
        KRV_CUDA(cudaFuncSetAttribute(agg_shared_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        const int grid = (int)std::min<int64_t>(rt_->sm_count, ceil_div(std::max<int64_t>(n, 1), kAggThreads));
        agg_shared_kernel<<<grid, kAggThreads, smem, rt_->stream>>>(P, T, key, n, rows_idx, ovf, ovf_count, E, E * 5 / 8,
                                                                    hot_.as<long long>(), H);
    } else {
        agg_global_kernel<<<grid_for(rt_, n, 256, 8), 256, 0, rt_->stream>>>(P, T, key, n, rows_idx, ovf, ovf_count);
    }
    rt_->launches++;
    check_launch("aggregate kernel");
}

namespace {
// The sampled rows' keys counted in an open-addressing table (each key once,
// its count in tcnt); stats[0]: the sampled rows with a NULL or the marker key.
__global__ void sample_count_kernel(KeyIn key, int64_t n, int64_t step, int m, long long *tkeys, unsigned *tcnt,
                                    uint64_t mask, unsigned *stats) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < m; j += gridDim.x * blockDim.x) {
        const int64_t r = (int64_t)j * step;
        if (r >= n) continue;
        const long long k = bit_get(key.valid, key.voff, r) ? key_at(key, r) : kEmptyKey;
        if (k == kEmptyKey) {
            atomicAdd(stats, 1u);
            continue;
        }
        uint64_t pos = hash_word((uint64_t)k) & mask;
        for (uint64_t t = 0; t <= mask; t++) {
            const long long cur = (long long)atomicCAS(reinterpret_cast<unsigned long long *>(tkeys + pos),
                                                       (unsigned long long)kEmptyKey, (unsigned long long)k);
            if (cur == kEmptyKey || cur == k) {
                atomicAdd(tcnt + pos, 1u);
                break;
            }
            pos = (pos + 1) & mask;
        }
    }
}
// The counted keys: stats[1] distinct, stats[2] seen once, and those seen
// at least `at_least` times listed (stats[3] of them, at most `cap` kept).
__global__ void sample_runs_kernel(const long long *tkeys, const unsigned *tcnt, uint64_t slots, unsigned at_least,
                                   long long *okeys, unsigned *ocnt, unsigned cap, unsigned *stats) {
    for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < slots; s += (uint64_t)gridDim.x * blockDim.x) {
        const unsigned c = tcnt[s];
        if (!c) continue;
        atomicAdd(stats + 1, 1u);
        if (c == 1) atomicAdd(stats + 2, 1u);
        if (c >= at_least) {
            const unsigned i = atomicAdd(stats + 3, 1u);
            if (i < cap) {
                okeys[i] = tkeys[s];
                ocnt[i] = c;
            }
        }
    }
}
}  // namespace

// A strided sample of `m` keys of the batch, counted on the device: the keys
// seen at least `at_least` times (count, key), the distinct keys, those seen
// once, and the sampled rows with a NULL or the marker key. One host read.
struct KeySample {
    std::vector<std::pair<int, long long>> runs;  // the keys seen at least at_least times
    int special = 0;
    int distinct = 0;  // distinct valid keys (not the marker)
    int singles = 0;   // of them, seen once
    int m = 0;
};
static KeySample take_sample(Runtime *rt, const KeyIn &key, int64_t n, int m, int at_least) {
    KeySample S;
    S.m = m;
    if (m <= 0) return S;
    constexpr unsigned kCap = 8192;
    const int64_t step = std::max<int64_t>(1, n / m);
    const uint64_t slots = next_pow2((uint64_t)2 * m);
    DBuf tkeys(rt, slots * 8), tcnt(rt, slots * 4);
    DBuf out(rt, 16 + (size_t)kCap * 12);  // stats[4], then kCap keys, then kCap counts
    KRV_CUDA(cudaMemsetAsync(tkeys.get(), 0x80, slots * 8, rt->stream));
    KRV_CUDA(cudaMemsetAsync(tcnt.get(), 0, slots * 4, rt->stream));
    KRV_CUDA(cudaMemsetAsync(out.get(), 0, 16, rt->stream));
    unsigned *stats = out.as<unsigned>();
    long long *okeys = reinterpret_cast<long long *>(out.as<uint8_t>() + 16);
    unsigned *ocnt = reinterpret_cast<unsigned *>(okeys + kCap);
    sample_count_kernel<<<grid_for(rt, m, 256, 4), 256, 0, rt->stream>>>(key, n, step, m, tkeys.as<long long>(),
                                                                         tcnt.as<unsigned>(), slots - 1, stats);
    rt->launches++;
    check_launch("sample_count_kernel");
    sample_runs_kernel<<<grid_for(rt, (int64_t)slots, 256, 4), 256, 0, rt->stream>>>(
        tkeys.as<long long>(), tcnt.as<unsigned>(), slots, (unsigned)std::max(1, at_least), okeys, ocnt, kCap, stats);
    rt->launches++;
    check_launch("sample_runs_kernel");
    std::vector<uint8_t> h(out.bytes());
    KRV_CUDA(cudaMemcpyAsync(h.data(), out.get(), out.bytes(), cudaMemcpyDeviceToHost, rt->stream));
    KRV_CUDA(cudaStreamSynchronize(rt->stream));
    unsigned st[4];
    memcpy(st, h.data(), 16);
    S.special = (int)st[0];
    S.distinct = (int)st[1];
    S.singles = (int)st[2];
    const unsigned got = std::min(st[3], kCap);
    const long long *hk = reinterpret_cast<const long long *>(h.data() + 16);
    const unsigned *hc = reinterpret_cast<const unsigned *>(hk + kCap);
    for (unsigned i = 0; i < got; i++) S.runs.push_back({(int)hc[i], hk[i]});
    return S;
}
// The `most` keys seen at least `at_least` times, most frequent first.
static std::vector<long long> top_keys(const KeySample &S, int most, int at_least) {
    std::vector<std::pair<int, long long>> c;
    for (const auto &r : S.runs)
        if (r.first >= at_least) c.push_back(r);
    const auto by_count = [](const auto &x, const auto &y) { return x.first > y.first || (x.first == y.first && x.second < y.second); };
    if ((int)c.size() > most) {
        std::nth_element(c.begin(), c.begin() + most, c.end(), by_count);
        c.resize(most);
    }
    std::sort(c.begin(), c.end(), by_count);
    std::vector<long long> out;
    for (const auto &r : c) out.push_back(r.second);
    return out;
}

void HashAggregate::sample_hot(const KeyIn &key, int64_t n) {
    sampled_ = true;
    constexpr int kSample = 1 << 16;
    const int m = (int)std::min<int64_t>(n, kSample);
    if (m < 1024) return;  // too few rows for hot keys to matter
    // hot: at least 0.2% of the sample each
    const int at_least = std::max(1, (m + 499) / 500);
    const KeySample S = take_sample(rt_, key, n, m, at_least);
    const std::vector<long long> hot = top_keys(S, kHotKeys, at_least);
    hot_count_ = (int)hot.size();
    if (!hot_count_) return;
    hot_ = DBuf(rt_, hot.size() * 8);
    KRV_CUDA(cudaMemcpyAsync(hot_.get(), hot.data(), hot.size() * 8, cudaMemcpyHostToDevice, rt_->stream));
    KRV_CUDA(cudaStreamSynchronize(rt_->stream));  // `hot` is a stack vector
}

// ---- the partitioned path ----------------------------------------------------------
namespace {
constexpr int64_t kPartMinRows = 1 << 18;    // smaller batches take the one-pass kernels
constexpr int64_t kPartSliceRows = 1 << 27;  // rows per split + partition round
constexpr int kPartSample = 1 << 16;

// The plan's columns sliced to start at row `row0`.
AggPlanDev slice_plan(const AggPlanDev &P, int64_t row0, const std::vector<int> &widths) {
    AggPlanDev S = P;
    for (int c = 0; c < P.ncols; c++) {
        S.c[c].data = static_cast<const uint8_t *>(P.c[c].data) + row0 * widths[c];
        S.c[c].voff = P.c[c].voff + row0;
    }
    return S;
}
}  // namespace

bool HashAggregate::use_partitioned(int64_t n) const {
    return mode_ == KRV_AGG_MODE_SHARED && n >= kPartMinRows &&
           part_smem_bytes(part_row_bytes_) + 1024 <= (size_t)rt_->max_smem_optin;
}

// Row records of the partitioned path: key, validity word, then the values
// the accumulators read (4-, then 8-, then 16-byte ones), 16-byte aligned.
void HashAggregate::plan_row_records() {
    int off = 12;
    for (int c = 0; c < P_.ncols; c++) part_off_val_[c] = 0;
    for (int pass = 0; pass < 3; pass++) {
        const int want = pass == 0 ? 4 : pass == 1 ? 8 : 16;
        if (want > 4) off = (off + want - 1) / want * want;
        for (int c = 0; c < P_.ncols; c++) {
            const AggColDev &C = P_.c[c];
            if (!(C.flags & (F_SUM | F_MIN | F_MAX))) continue;
            const int w = (C.type == (int)Type::I32 || C.type == (int)Type::Date32) ? 4
                          : C.type == (int)Type::Dec128                             ? 16
                                                                                    : 8;
            if (w != want) continue;
            part_off_val_[c] = (int16_t)off;
            off += w;
        }
    }
    part_row_bytes_ = (off + 15) / 16 * 16;
}

void HashAggregate::plan_partitioned(const KeyIn &key, int64_t n) {
    part_planned_ = true;
    // The sample: a strided 64K rows of the first large batch.
    const int m = (int)std::min<int64_t>(n, kPartSample);
    const KeySample S = take_sample(rt_, key, n, m, 3);
    const int special = S.special;
    // Hot: seen at least 3 times, as many as the split kernel's shared memory
    // holds records for beside its lookup table.
    const int smem_cap = std::min(rt_->max_smem_optin - 2048, 72 * 1024);
    int hmax = kHotMax;
    while (hmax > 0 && (size_t)(hmax + 2) * smem_stride(P_) + (size_t)2 * next_pow2(hmax) * 10 > (size_t)smem_cap)
        hmax /= 2;
    const std::vector<long long> ranked = top_keys(S, hmax, 3);
    // The hot-key table: each key, most frequent first, into the emptier of
    // its two buckets; a key that finds both full stays cold.
    const int nb = ranked.empty() ? 0 : (int)std::max<uint64_t>(2, next_pow2((ranked.size() + 1) / 2));
    std::vector<long long> tab((size_t)nb * kHotWays, kEmptyKey);
    std::vector<int16_t> tidx((size_t)nb * kHotWays, -1);
    std::vector<int> fill(nb, 0);
    std::vector<long long> hot;
    for (long long k : ranked) {
        int b1, b2;
        hot_buckets(hash_word((uint64_t)k), nb, b1, b2);
        const int b = fill[b1] <= fill[b2] ? b1 : b2;
        if (fill[b] >= kHotWays) continue;
        tab[(size_t)b * kHotWays + fill[b]] = k;
        tidx[(size_t)b * kHotWays + fill[b]] = (int16_t)hot.size();
        fill[b]++;
        hot.push_back(k);
    }
    part_hot_slots_ = nb * kHotWays;
    part_hot_tab_ = DBuf(rt_, (size_t)std::max(1, part_hot_slots_) * 8);
    part_hot_tab_idx_ = DBuf(rt_, (size_t)std::max(1, part_hot_slots_) * 2);
    if (nb) {
        KRV_CUDA(cudaMemcpyAsync(part_hot_tab_.get(), tab.data(), tab.size() * 8, cudaMemcpyHostToDevice, rt_->stream));
        KRV_CUDA(cudaMemcpyAsync(part_hot_tab_idx_.get(), tidx.data(), tidx.size() * 2, cudaMemcpyHostToDevice,
                                 rt_->stream));
    }
    std::vector<long long> hot_sorted = hot;
    std::sort(hot_sorted.begin(), hot_sorted.end());
    int hot_rows = 0;
    for (const auto &r : S.runs)
        if (std::binary_search(hot_sorted.begin(), hot_sorted.end(), r.second)) hot_rows += r.first;
    part_hot_ = (int)hot.size();
    part_cold_frac_ = m ? std::max(0.0, 1.0 - (double)(hot_rows + special) / m) : 1.0;
    // Distinct cold keys (the guaranteed-error estimator: keys seen once in
    // the sample stand for sqrt(n / m) keys each; hot keys are seen 3 times
    // or more).
    const int64_t d = std::max<int64_t>(0, (int64_t)S.distinct - part_hot_), f1 = S.singles;
    const double est = (double)d + (double)f1 * (std::sqrt((double)n / std::max(1, m)) - 1.0);
    part_groups_est_ = std::max<int64_t>({(int64_t)est, spec_.expected_groups, 1});
    // Hot keys' group ids: the table first gets room for them.
    part_hot_keys_ = DBuf(rt_, (size_t)std::max(1, part_hot_) * 8);
    part_hot_gids_ = DBuf(rt_, (size_t)(part_hot_ + 2) * 4);
    if (part_hot_)
        KRV_CUDA(cudaMemcpyAsync(part_hot_keys_.get(), hot.data(), hot.size() * 8, cudaMemcpyHostToDevice, rt_->stream));
    if (known_groups_ + part_hot_ + 2 > (int64_t)limit_) grow((uint64_t)known_groups_ + part_hot_ + 2);
    TableDev T{keys_.as<long long>(), gids_.as<uint32_t>(), slots_ - 1, states_.as<uint8_t>(), gkeys_.as<long long>(),
               ngroups_.as<unsigned long long>(), limit_, status_word(rt_)};
    hot_gid_kernel<<<grid_for(rt_, part_hot_ + 2, 128, 1), 128, 0, rt_->stream>>>(P_, T, part_hot_keys_.as<long long>(),
                                                                                  part_hot_, part_hot_gids_.as<uint32_t>());
    rt_->launches++;
    check_launch("hot_gid_kernel");
    KRV_CUDA(cudaStreamSynchronize(rt_->stream));  // `hot`, `tab` and `tidx` are stack vectors
}

void HashAggregate::push_partitioned(const DevBatch &b, const KeyIn &key, int64_t n) {
    clear_status(rt_);
    pending_rows_ = 0;
    if (!part_planned_) plan_partitioned(key, n);
    AggPlanDev P = P_;
    std::vector<int> widths(P.ncols);
    for (int c = 0; c < P.ncols; c++) {
        const DevCol &col = b.cols[value_cols_[c]];
        P.c[c].data = col.data;
        P.c[c].valid = col.valid;
        P.c[c].voff = col.valid_off;
        widths[c] = col.type.var() ? 4 : col.type.width();  // a counted string column: its offsets
    }
    known_groups_ = (int64_t)read_scalar<unsigned long long>(rt_, ngroups_.get());  // the hot keys' groups too
    // Partitions: each to hold about kPartKeys distinct keys (at most 2^13
    // of them: every split CTA keeps a cursor per partition in shared memory).
    constexpr int kPartKeys = 256;
    int bits = 5;
    while (bits < 13 && ((int64_t)1 << bits) * kPartKeys < part_groups_est_) bits++;
    const int nparts = 1 << bits;
    const int H = part_hot_;
    const int hot_slots = H ? part_hot_slots_ : 0;
    const size_t split_smem = ((size_t)(H + 2) * smem_stride(P) + 15) / 16 * 16 + (size_t)hot_slots * 10 + (size_t)nparts * 4;
    const size_t count_smem = (size_t)((nparts + 1) & ~1) * 4 + (size_t)hot_slots * 8;
    // Value columns held in registers: as few as the plan has (fewer
    // registers for the row loaded ahead).
    const auto split_kernel = P.ncols <= 3   ? agg_split_kernel<3>
                              : P.ncols <= 4 ? agg_split_kernel<4>
                                             : agg_split_kernel<kMaxValueCols>;
    KRV_CUDA(cudaFuncSetAttribute(split_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)split_smem));
    KRV_CUDA(cudaFuncSetAttribute(agg_count_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)count_smem));
    const size_t part_smem = part_smem_bytes(part_row_bytes_);
    KRV_CUDA(cudaFuncSetAttribute(agg_part_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)part_smem));
    int split_blocks = 0, part_blocks = 0;
    KRV_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&split_blocks, split_kernel, kSplitThreads, split_smem));
    KRV_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&part_blocks, agg_part_kernel, kPartThreads, part_smem));
    if (split_blocks < 1 || part_blocks < 1) fail(KRV_INTERNAL, "aggregate: partitioned kernels do not fit an SM");
    const KeyIn key0 = key;
    for (int64_t row0 = 0; row0 < n; row0 += kPartSliceRows) {
        const int64_t ns = std::min<int64_t>(kPartSliceRows, n - row0);
        SplitDev S{};
        S.hot_keys = part_hot_keys_.as<long long>();
        S.hot_gids = part_hot_gids_.as<uint32_t>();
        S.H = H;
        S.hot_slots = hot_slots;
        S.hot_tab = part_hot_tab_.as<long long>();
        S.hot_tab_idx = part_hot_tab_idx_.as<int16_t>();
        S.part_bits = bits;
        S.row_bytes = part_row_bytes_;
        for (int c = 0; c < kMaxValueCols; c++) S.off_val[c] = part_off_val_[c];
        // The count and split kernels take the same tiles: one CTA per
        // resident split CTA.
        S.ctas = (int)std::min<int64_t>((int64_t)split_blocks * rt_->sm_count, ceil_div(ns, kSplitThreads));
        KeyIn ks = key0;
        ks.data = static_cast<const uint8_t *>(key0.data) + row0 * key0.width;
        ks.voff = key0.voff + row0;
        // Exact partition sizes, per partition and CTA: the split's own test
        // over its own tiles, then the partitions laid out back to back and
        // every CTA's share of each placed within it.
        DBuf cta_rows(rt_, (size_t)nparts * S.ctas * 4), totals(rt_, (size_t)nparts * 4);
        DBuf part_info(rt_, (size_t)nparts * kCntStride * 4);
        DBuf ctl(rt_, 16);  // [0] rows in the partitions (u64), [8] failed partitions (int)
        KRV_CUDA(cudaMemsetAsync(ctl.get(), 0, 16, rt_->stream));
        S.cta_rows = cta_rows.as<unsigned>();
        KRV_CUDA(cudaMemsetAsync(cta_rows.get(), 0, cta_rows.bytes(), rt_->stream));
        agg_count_kernel<<<2 * S.ctas, kSplitThreads, count_smem, rt_->stream>>>(ks, ns, S);
        rt_->launches++;
        check_launch("agg_count_kernel");
        part_offsets_kernel<<<(int)ceil_div((int64_t)nparts * 32, 256), 256, 0, rt_->stream>>>(
            cta_rows.as<unsigned>(), S.ctas, nparts, totals.as<unsigned>());
        rt_->launches++;
        check_launch("part_offsets_kernel");
        part_bases_kernel<<<1, 1024, 0, rt_->stream>>>(totals.as<unsigned>(), nparts, part_info.as<unsigned>(),
                                                      ctl.as<unsigned long long>());
        rt_->launches++;
        check_launch("part_bases_kernel");
        const unsigned long long cold = read_scalar<unsigned long long>(rt_, ctl.get());
        DBuf part_buf(rt_, (size_t)std::max<unsigned long long>(cold, 1) * part_row_bytes_);
        DBuf start(rt_, (size_t)nparts * 4);
        KRV_CUDA(cudaMemsetAsync(start.get(), 0, start.bytes(), rt_->stream));
        // Room in the table for the keys this slice may add (an estimate; a
        // partition that finds none stops and runs again after a grow).
        const int64_t want = known_groups_ + std::min<int64_t>(ns, part_groups_est_) + H + 2;
        if (want > (int64_t)part_id_limit(part_blocks)) grow((uint64_t)want + part_id_room(part_blocks));
        TableDev T{keys_.as<long long>(), gids_.as<uint32_t>(), slots_ - 1, states_.as<uint8_t>(), gkeys_.as<long long>(),
                   ngroups_.as<unsigned long long>(), limit_, status_word(rt_)};
        S.part_buf = part_buf.as<uint8_t>();
        S.part_info = part_info.as<unsigned int>();
        S.cold = cold;
        const AggPlanDev PS = slice_plan(P, row0, widths);
        split_kernel<<<S.ctas, kSplitThreads, split_smem, rt_->stream>>>(PS, T, ks, ns, S);
        rt_->launches++;
        check_launch("agg_split_kernel");
        PartDev D{};
        D.part_buf = part_buf.as<uint8_t>();
        D.part_info = part_info.as<unsigned int>();
        D.row_bytes = part_row_bytes_;
        for (int c = 0; c < kMaxValueCols; c++) D.off_val[c] = part_off_val_[c];
        D.todo = nullptr;
        D.start = start.as<uint32_t>();
        D.failed = reinterpret_cast<int *>(ctl.as<uint8_t>() + 8);
        D.id_limit = part_id_limit(part_blocks);
        // Cold keys already in the table (from earlier batches or slices)
        // are looked up; the first slice's are all new.
        D.lookup = known_groups_ > (int64_t)kFirstGid + H ? 1 : 0;
        D.first_new = (unsigned long long)known_groups_;
        unindexed_from_ = known_groups_;
        agg_part_kernel<<<nparts, kPartThreads, part_smem, rt_->stream>>>(P, T, D);
        rt_->launches++;
        check_launch("agg_part_kernel");
        DBuf todo;
        for (int round = 0;; round++) {
            const int failed = read_scalar<int>(rt_, ctl.as<uint8_t>() + 8);
            const uint32_t st = take_status(rt_);
            if (st & ST_TIMEOUT) fail(KRV_TIMEOUT, "aggregate: a wait for a group id gave up");
            if (st & ST_CAPACITY) fail(KRV_INTERNAL, "aggregate: a hot key has no group");
            if (st & ST_MISCOUNT) fail(KRV_INTERNAL, "aggregate: the split wrote more rows than were counted");
            known_groups_ = (int64_t)read_scalar<unsigned long long>(rt_, ngroups_.get());
            if (failed == 0) break;
            if (round == 16) fail(KRV_INTERNAL, "aggregate: table growth did not converge");
            // Partitions that stopped: their windows run again on a bigger table.
            std::vector<uint32_t> hs(nparts), hc((size_t)nparts * kCntStride);
            KRV_CUDA(cudaMemcpyAsync(hs.data(), start.get(), (size_t)nparts * 4, cudaMemcpyDeviceToHost, rt_->stream));
            KRV_CUDA(cudaMemcpyAsync(hc.data(), part_info.get(), part_info.bytes(), cudaMemcpyDeviceToHost, rt_->stream));
            KRV_CUDA(cudaStreamSynchronize(rt_->stream));
            std::vector<int> again;
            for (int p = 0; p < nparts; p++)
                if (hs[p] < std::min<uint32_t>(hc[(size_t)p * kCntStride], hc[(size_t)p * kCntStride + 1]))
                    again.push_back(p);
            grow((uint64_t)known_groups_ + (uint64_t)again.size() * kChunkRows + part_id_room(part_blocks) + 1);
            unindexed_from_ = known_groups_;  // grow indexed every group so far
            todo = DBuf(rt_, again.size() * 4);
            KRV_CUDA(cudaMemcpyAsync(todo.get(), again.data(), again.size() * 4, cudaMemcpyHostToDevice, rt_->stream));
            KRV_CUDA(cudaMemsetAsync(ctl.as<uint8_t>() + 8, 0, 4, rt_->stream));
            TableDev T2{keys_.as<long long>(), gids_.as<uint32_t>(), slots_ - 1, states_.as<uint8_t>(),
                        gkeys_.as<long long>(), ngroups_.as<unsigned long long>(), limit_, status_word(rt_)};
            D.todo = todo.as<int>();
            D.id_limit = part_id_limit(part_blocks);
            D.lookup = 1;
            D.first_new = (unsigned long long)known_groups_;
            agg_part_kernel<<<(int)again.size(), kPartThreads, part_smem, rt_->stream>>>(P, T2, D);
            rt_->launches++;
            check_launch("agg_part_kernel");
            KRV_CUDA(cudaStreamSynchronize(rt_->stream));  // `again` is a stack vector
        }
    }
    const uint32_t st = take_status(rt_);
    if (st & ST_TIMEOUT) fail(KRV_TIMEOUT, "aggregate: a wait for a group id gave up");
    known_groups_ = (int64_t)read_scalar<unsigned long long>(rt_, ngroups_.get());
}

void HashAggregate::push(const DevBatch &in) {
    if (finished_) fail(KRV_INVALID_ARGUMENT, "push after finish");
    DeviceGuard g(rt_);
    if (!planned_) plan(in);
    if (in.cols.size() != input_types_.size()) fail(KRV_INVALID_ARGUMENT, "batches differ in columns");
    for (size_t i = 0; i < in.cols.size(); i++)
        if (in.cols[i].type != input_types_[i]) fail(KRV_INVALID_ARGUMENT, "batches differ in types");
    const int64_t n = in.rows;
    if (n == 0) return;
    if (n >= (int64_t)0xFFFFFFF0ll) fail(KRV_UNSUPPORTED, "aggregate batches of 2^32 rows or more");
    DevBatch b = in;
    DBuf codes;
    if (dict_) {
        codes = key_dict_encode(dict_, in, dict_cols_);
        DevCol cc;
        cc.type = DType{Type::I64, 0, 0};
        cc.name = key_name_;
        cc.nullable = false;
        cc.length = n;
        cc.data = codes.get();
        b.cols.push_back(cc);
    }
    // string MIN/MAX columns: their values as codes of the column's value dictionary
    std::vector<DBuf> vcodes;
    for (int c = 0; c < P_.ncols; c++) {
        if (!(P_.c[c].flags & F_STR)) continue;
        const int col = value_cols_[c];
        vcodes.push_back(key_dict_encode(vdicts_[c], in, {col}, true));
        b.cols[col].data = vcodes.back().get();
        key_dict_strings(vdicts_[c], &P_.c[c].s_off, &P_.c[c].s_len, &P_.c[c].s_heap);
    }
    std::vector<DBuf> hidden;
    for (const auto &ps : poison_src_) {
        const DevCol &sc = in.cols[ps.first], &nc = in.cols[ps.second];
        hidden.emplace_back(rt_, (size_t)n * 8);
        poison_kernel<<<grid_for(rt_, n, 256, 8), 256, 0, rt_->stream>>>(
            sc.valid, sc.valid_off, static_cast<const uint8_t *>(nc.data), 0, n, hidden.back().as<long long>());
        rt_->launches++;
        check_launch("poison_kernel");
        DevCol hc;
        hc.type = DType{Type::I64, 0, 0};
        hc.name = "#overflowed";
        hc.nullable = false;
        hc.length = n;
        hc.data = hidden.back().get();
        b.cols.push_back(hc);
    }
    const DevCol &kc = b.cols[key_col_];
    KeyIn key{kc.data, kc.valid, kc.valid_off, kc.type.width(), 0};
    index_pending();
    if (use_partitioned(n)) {
        push_partitioned(b, key, n);
        return;
    }
    if (mode_ == KRV_AGG_MODE_SHARED && !sampled_) sample_hot(key, n);
    clear_status(rt_);
    DBuf ovf_count(rt_, 8);
    KRV_CUDA(cudaMemsetAsync(ovf_count.get(), 0, 8, rt_->stream));
    DBuf ovf(rt_, (size_t)n * 4);
    launch(b, key, n, nullptr, ovf.as<uint32_t>(), ovf_count.as<unsigned long long>());
    pending_rows_ += n;
    // No row can have been deferred while the table had room for every row
    // pushed since the last count: skip the synchronization then.
    const bool may_defer = known_groups_ + pending_rows_ > (int64_t)limit_;
    if (!may_defer) {
        const uint32_t st = take_status(rt_);
        if (st & ST_TIMEOUT) fail(KRV_TIMEOUT, "aggregate: a wait for a group id gave up");
        return;
    }
    DBuf idx;
    for (int round = 0; round < 16; round++) {
        const unsigned long long deferred = read_scalar<unsigned long long>(rt_, ovf_count.get());
        known_groups_ = (int64_t)read_scalar<unsigned long long>(rt_, ngroups_.get());
        pending_rows_ = 0;
        const uint32_t st = take_status(rt_);
        if (st & ST_TIMEOUT) fail(KRV_TIMEOUT, "aggregate: a wait for a group id gave up");
        if (deferred == 0) return;
        grow((uint64_t)known_groups_ + deferred);
        idx = DBuf(rt_, (size_t)deferred * 4);
        KRV_CUDA(cudaMemcpyAsync(idx.get(), ovf.get(), (size_t)deferred * 4, cudaMemcpyDeviceToDevice, rt_->stream));
        KRV_CUDA(cudaMemsetAsync(ovf_count.get(), 0, 8, rt_->stream));
        launch(b, key, (int64_t)deferred, idx.as<uint32_t>(), ovf.as<uint32_t>(), ovf_count.as<unsigned long long>());
        pending_rows_ = (int64_t)deferred;
    }
    fail(KRV_INTERNAL, "aggregate: table growth did not converge");
}

namespace {
// A code where the group has no value (validity bit clear): 0, which names
// some stored string, so that the gather reads inside the dictionary.
__global__ void str_code_clean_kernel(long long *codes, const uint8_t *valid, int64_t n) {
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x)
        if (!valid || !((valid[j >> 3] >> (j & 7)) & 1) || codes[j] < 0) codes[j] = 0;
}
}  // namespace

DevBatch HashAggregate::result() {
    DeviceGuard g(rt_);
    DevBatch out;
    if (!planned_) return out;
    known_groups_ = (int64_t)read_scalar<unsigned long long>(rt_, ngroups_.get());
    pending_rows_ = 0;
    // Which of the two special groups (NULL key, marker key) have rows.
    unsigned long long special_rows[2];
    for (int s = 0; s < 2; s++)
        special_rows[s] = read_scalar<unsigned long long>(rt_, states_.as<uint8_t>() + (size_t)s * P_.rec + P_.off_rows);
    OutPlanDev O{};
    O.nspecial = 0;
    for (uint32_t s = 0; s < 2; s++)
        if (special_rows[s]) O.special[O.nspecial++] = s;
    const int64_t nout = O.nspecial + (known_groups_ - kFirstGid);
    const bool key_nullable = special_rows[0] != 0;
    DevCol kcol = make_col(rt_, key_type_, nout, key_nullable, key_name_);
    out.cols.push_back(kcol);
    // Output expressions: one per aggregate (final), or each aggregate's
    // state columns (partial; AggregateExpr::state_fields, aggregate/mod.rs:747-800).
    struct OutSpec {
        int32_t func, col, aux;
        DType in, type;
        std::string name;
        bool nullable;
    };
    std::vector<OutSpec> outs;
    static const char *fname[] = {"count(1)", "count", "sum", "min", "max", "avg"};
    const bool partial = spec_.output == KRV_AGG_OUTPUT_PARTIAL;
    for (int e = 0; e < spec_.n_aggregates; e++) {
        const krv_agg_expr &x = spec_.aggregates[e];
        const bool state = x.input == KRV_AGG_INPUT_STATE;
        const int col = expr_col_[e], aux = expr_aux_[e];
        const DType it = col >= 0 ? input_types_[x.column] : DType{Type::I64, 0, 0};
        const std::string name = x.function == KRV_AGG_COUNT_STAR
                                     ? std::string("count(1)")
                                     : std::string(fname[x.function]) + "(" + input_names_[x.column] + ")";
        const bool dec = it.id == Type::Dec64 || it.id == Type::Dec128;
        const DType i64{Type::I64, 0, 0}, f64{Type::F64, 0, 0};
        // sum_decimal (aggregate/mod.rs:929-931) on decimal_on's carrier (:1018-1024); a
        // merge of decimal sums keeps the state's type
        auto sum_type = [&]() -> DType {
            if (dec && state) return it;
            if (dec) {
                const int p = std::min(38, it.precision + 10);
                return DType{(it.id == Type::Dec64 && p <= 18) ? Type::Dec64 : Type::Dec128, p, it.scale};
            }
            return it.id == Type::F64 ? f64 : i64;
        };
        // AVG of a decimal: (p + 4, s + 4) of the raw argument
        auto avg_type = [&]() -> DType {
            if (!dec) return f64;
            int rp = it.precision, rs = it.scale;
            bool r64 = it.id == Type::Dec64;
            if (state) {
                rp = x.arg_precision > 0 ? x.arg_precision : it.precision < 38 ? it.precision - 10 : -1;
                if (rp <= 0) fail(KRV_INVALID_ARGUMENT, "AVG over decimal states of precision 38 needs arg_precision");
                rs = x.arg_precision > 0 ? x.arg_scale : it.scale;
                r64 = x.arg_bits ? x.arg_bits == 64 : it.id == Type::Dec64;
            }
            const int p = std::min(38, rp + 4), sc = std::min(38, rs + 4);
            return DType{(r64 && p <= 18) ? Type::Dec64 : Type::Dec128, p, sc};
        };
        auto add = [&](int32_t func, int c, int a, DType type, const std::string &nm, bool nullable) {
            outs.push_back(OutSpec{func, c, a, it, type, nm, nullable});
        };
        const int32_t count_f = state ? F_COUNT_MERGE : x.function;
        switch (x.function) {
        case KRV_AGG_COUNT_STAR:
        case KRV_AGG_COUNT:
            add(count_f, col, -1, i64, partial ? name + "#count" : name, false);
            break;
        case KRV_AGG_MIN:
        case KRV_AGG_MAX:
            add(x.function, col, -1, it, partial ? name + "#value" : name, true);
            break;
        case KRV_AGG_SUM:
            add(KRV_AGG_SUM, col, aux, sum_type(), partial ? name + "#sum" : name, true);
            if (partial && dec) add(F_NONEMPTY, col, aux, DType{Type::Bool, 0, 0}, name + "#nonempty", false);
            break;
        case KRV_AGG_AVG:
            if (!partial) {
                add(state ? F_AVG_MERGE : KRV_AGG_AVG, col, aux, avg_type(), name, true);
            } else if (state) {
                add(KRV_AGG_SUM, col, -1, sum_type(), name + "#sum", true);
                add(F_COUNT_MERGE, aux, -1, i64, name + "#count", false);
            } else {
                add(dec ? KRV_AGG_SUM : F_SUM_AS_F64, col, -1, dec ? sum_type() : f64, name + "#sum", true);
                add(KRV_AGG_COUNT, col, -1, i64, name + "#count", false);
            }
            break;
        }
    }
    if ((int)outs.size() > kMaxExprs) fail(KRV_UNSUPPORTED, "more than 32 output columns of aggregates");
    O.n = (int)outs.size();
    // string MIN/MAX outputs: (position in out.cols, output spec, plan column),
    // finalized as codes and then gathered from the value dictionary
    std::vector<std::tuple<int, OutSpec, int>> str_outs;
    for (int e = 0; e < O.n; e++) {
        OutSpec o = outs[e];
        OutExprDev &X = O.e[e];
        if ((o.func == KRV_AGG_MIN || o.func == KRV_AGG_MAX) && o.col >= 0 && (P_.c[o.col].flags & F_STR)) {
            str_outs.emplace_back((int)out.cols.size(), o, o.col);
            o.type = DType{Type::I64, 0, 0};
        }
        X.func = o.func;
        X.col = o.col;
        X.aux = o.aux;
        X.ansi = spec_.ansi;
        X.in_type = (int)o.in.id;
        X.in_scale = o.in.scale;
        X.otype = (int)o.type.id;
        X.rp = o.type.precision;
        X.rs = o.type.scale;
        DevCol c;
        if (o.type.id == Type::Bool) {
            // whole 32-bit words: the kernel stores one word per 32 rows
            c.type = o.type;
            c.name = o.name;
            c.nullable = false;
            c.length = nout;
            c.hold_data = std::make_shared<DBuf>(rt_, (size_t)ceil_div(std::max<int64_t>(nout, 1), 32) * 4);
            c.data = c.hold_data->get();
        } else {
            c = make_col(rt_, o.type, nout, o.nullable, o.name);
        }
        X.dst = const_cast<void *>(c.data);
        X.dst_valid = o.nullable ? (uint32_t *)c.valid : nullptr;
        out.cols.push_back(c);
    }
    out.rows = nout;
    clear_status(rt_);
    if (nout > 0) {
        finalize_kernel<<<grid_for(rt_, nout, 256, 8), 256, 0, rt_->stream>>>(
            P_, O, states_.as<uint8_t>(), gkeys_.as<long long>(), nout, key_type_.width(), const_cast<void *>(kcol.data),
            key_nullable ? (uint32_t *)kcol.valid : nullptr, status_word(rt_));
        rt_->launches++;
        check_launch("finalize_kernel");
    }
    const uint32_t st = take_status(rt_);
    if (st & ST_OVERFLOW)
        fail(KRV_ARITHMETIC_OVERFLOW, "ARITHMETIC_OVERFLOW: an aggregate overflowed its result type (ANSI mode)");
    for (const auto &so : str_outs) {
        const int pos = std::get<0>(so);
        const OutSpec &o = std::get<1>(so);
        DevCol codes = out.cols[pos];
        DevCol col;
        if (nout > 0) {
            // groups with no value: a code that exists (their validity stays clear)
            str_code_clean_kernel<<<grid_for(rt_, nout, 256, 8), 256, 0, rt_->stream>>>(
                static_cast<long long *>(const_cast<void *>(codes.data)), codes.valid, nout);
            rt_->launches++;
            check_launch("str_code_clean_kernel");
            col = key_dict_decode(vdicts_[std::get<2>(so)], static_cast<const long long *>(codes.data), nout)[0];
            col.hold_valid = codes.hold_valid;
            col.valid = codes.valid;
            col.valid_off = 0;
        } else {
            col = var_gather(rt_, VarSrc{}, nullptr, 0, o.type, true, o.name);
        }
        col.name = o.name;
        col.nullable = true;
        out.cols[pos] = col;
    }
    if (!str_outs.empty()) KRV_CUDA(cudaStreamSynchronize(rt_->stream));  // the codes are read by the gathers
    if (dict_) {
        // the group-by columns in place of the codes
        std::vector<DevCol> keys = key_dict_decode(dict_, static_cast<const long long *>(out.cols[0].data), out.rows);
        DevCol codes = out.cols[0];
        out.cols.erase(out.cols.begin());
        out.cols.insert(out.cols.begin(), keys.begin(), keys.end());
        KRV_CUDA(cudaStreamSynchronize(rt_->stream));  // the codes are read by the decode
    }
    return out;
}

HashAggregate *make_aggregate(Runtime *rt, const krv_agg_spec &spec) {
    return new HashAggregate(rt, spec);
}
void agg_push(HashAggregate *a, const DevBatch &b) { a->push(b); }
void agg_finish(HashAggregate *a) { a->finish(); }
DevBatch agg_result(HashAggregate *a) { return a->result(); }
int64_t agg_groups(const HashAggregate *a) { return a->groups(); }
void agg_destroy(HashAggregate *a) { delete a; }

}  // namespace krv
