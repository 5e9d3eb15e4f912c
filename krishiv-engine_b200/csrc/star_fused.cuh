// star_fused.cuh -- the fused fact-side kernel of the star-join pipeline.
//
// Each runtime filter is first evaluated once for every value of its key
// range [lo, hi] into an answer bitmap (bit v - lo = whether the filter passes
// v: the Bloom's answer, false positives included), when the range is small
// enough; dimension B's bitmap is staged in shared memory, A's stays in
// L2. A row's filter test is then one bit. Without a bitmap the kernel
// probes the filter itself (range, then Bloom block or exact set).
//
// Per warp, two stages, so both run on full warps without block barriers:
//  1. each lane reads 8 consecutive fk_b values (64 bytes; the warp reads
//     2 KB contiguous, the next tile prefetched into registers) and tests
//     them against B's filter; passing rows go to the warp's queue in shared
//     memory (row, fk_b);
//  2. whenever the queue holds 32 entries, each lane takes one: reads fk_a
//     (only for these rows), tests A's filter, probes both hash tables and
//     adds price * (1 - discount) of each joined row to its group's
//     shared-memory accumulator.
// So the kernel reads all of fk_b, the 32-byte sectors of fk_a holding a row
// that passed B's filter, and price/discount only of joined rows.
#pragma once

#include "krv_device.cuh"
#include "krv_filter.cuh"
#include "ops.h"

namespace krv {

constexpr int kStarThreads = 1024;                        // threads per CTA
constexpr int kStarWarps = kStarThreads / 32;
constexpr int kStarRows = 8;                              // rows per lane per tile
constexpr int kStarTile = kStarThreads * kStarRows;       // 8192 rows
constexpr int kStarWarpQueue = 32 * 4 + 32;               // one half-tile's rows + one drain
constexpr uint32_t kStarNone = 0xFFFFFFFFu;
constexpr int kStarMaxSmemGroups = 1024;

struct StarTable {
    const unsigned long long *slots;
    uint64_t mask;
    const uint32_t *next;
    uint64_t seed;
    const long long *keys;  // build key column
    const int32_t *gid;     // dense group id of each build row's attribute
};

struct StarArgs {
    const long long *fk_a, *fk_b, *price;
    const double *disc;
    int64_t n;
    KeyFilterDev fa, fb;
    const uint32_t *bits_a, *bits_b;  // answer bitmaps over [lo, hi] (null: probe the filter)
    int use_filters;
    int group_by;  // 0: dim A's attribute, 1: dim B's
    StarTable ta, tb;
    int ngroups;
    int bits_b_smem_words;  // > 0: B's answer bitmap staged in shared memory
    double *sum_hi, *sum_lo;
    unsigned long long *cnt;
    unsigned long long *stats;  // [0] rows passing both filters, [1] joined rows, [2] fk_a sectors read
};

__device__ __forceinline__ uint32_t star_lookup(const StarTable &t, long long k) {
    const uint64_t g = finalize(hash_word((uint64_t)k), t.seed);
    const unsigned long long tag = g >> 32;
    uint64_t pos = g & t.mask;
    for (uint64_t p = 0; p <= t.mask; p++) {
        const unsigned long long s = __ldg(t.slots + pos);
        if (s == 0) return kStarNone;
        if ((s >> 32) == tag) {
            const uint32_t o = (uint32_t)(s & 0xFFFFFFFFull) - 1u;
            if (__ldg(t.keys + o) == k) return o;
        }
        pos = (pos + 1) & t.mask;
    }
    return kStarNone;
}

// The filter's answer for k from its bitmap over [lo, hi].
__device__ __forceinline__ bool star_bit(const uint32_t *bits, long long lo, long long hi, long long k) {
    if (k < lo || k > hi) return false;
    const uint64_t v = (uint64_t)(k - lo);
    return (bits[v >> 5] >> (v & 31)) & 1u;
}

template <bool VEC>
__device__ __forceinline__ void star_load_tile(const StarArgs &A, int64_t r0, long long (&v)[kStarRows]) {
    if (VEC && r0 + kStarRows <= A.n) {
        const longlong2 *p = reinterpret_cast<const longlong2 *>(A.fk_b + r0);
#pragma unroll
        for (int j = 0; j < kStarRows / 2; j++) {
            const longlong2 x = __ldcs(p + j);
            v[2 * j] = x.x;
            v[2 * j + 1] = x.y;
        }
    } else {
#pragma unroll
        for (int j = 0; j < kStarRows; j++) v[j] = r0 + j < A.n ? __ldcs(A.fk_b + r0 + j) : 0;
    }
}

// Stage 2 for one queue entry (one lane).
__device__ __forceinline__ void star_stage2(const StarArgs &A, uint32_t row, long long kb, int G, double *s_hi,
                                            double *s_lo, unsigned long long *s_cnt, unsigned &passed,
                                            unsigned &joined) {
    const long long ka = __ldcs(A.fk_a + row);
    if (A.use_filters) {
        const bool pa = A.bits_a ? star_bit(A.bits_a, A.fa.lo, A.fa.hi, ka) : filter_pass(A.fa, ka);
        if (!pa) return;
    }
    passed++;
    uint32_t ra = star_lookup(A.ta, ka);
    if (ra == kStarNone) return;
    const uint32_t rb0 = star_lookup(A.tb, kb);
    if (rb0 == kStarNone) return;
    const double price = (double)__ldcs(A.price + row);
    const double disc = __ldcs(A.disc + row);
    const double v = __dmul_rn(price, __dsub_rn(1.0, disc));
    for (int ca = 0; ra != kStarNone && ca < (1 << 20); ca++, ra = A.ta.next[ra]) {
        int cb = 0;
        for (uint32_t rb = rb0; rb != kStarNone && cb < (1 << 20); cb++, rb = A.tb.next[rb]) {
            joined++;
            const int g = A.group_by == 0 ? A.ta.gid[ra] : A.tb.gid[rb];
            if (g < G) {
                atomic_add_dd(s_hi + g, s_lo + g, v);
                atomicAdd(s_cnt + g, 1ull);
            } else {
                atomic_add_dd(A.sum_hi + g, A.sum_lo + g, v);
                atomicAdd(A.cnt + g, 1ull);
            }
        }
    }
}

// BMODE 1: B's answer bitmap in shared memory; 0: B's filter probed per row.
template <int BMODE, bool VEC>
__global__ void __launch_bounds__(kStarThreads, 1) star_fused_kernel(StarArgs A) {
    extern __shared__ __align__(16) uint8_t smem[];
    uint32_t *s_bits = reinterpret_cast<uint32_t *>(smem);
    uint32_t *q_row_all = reinterpret_cast<uint32_t *>(smem + (size_t)A.bits_b_smem_words * 4);
    long long *q_key_all = reinterpret_cast<long long *>(q_row_all + kStarWarps * kStarWarpQueue);
    const int G = A.ngroups < kStarMaxSmemGroups ? A.ngroups : kStarMaxSmemGroups;
    double *s_hi = reinterpret_cast<double *>(q_key_all + kStarWarps * kStarWarpQueue);
    double *s_lo = s_hi + G;
    unsigned long long *s_cnt = reinterpret_cast<unsigned long long *>(s_lo + G);
    __shared__ unsigned long long s_stat[3];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    uint32_t *q_row = q_row_all + warp * kStarWarpQueue;
    long long *q_key = q_key_all + warp * kStarWarpQueue;
    for (int g = tid; g < G; g += kStarThreads) {
        s_hi[g] = 0.0;
        s_lo[g] = 0.0;
        s_cnt[g] = 0;
    }
    if (BMODE == 1) {
        const uint4 *src = reinterpret_cast<const uint4 *>(A.bits_b);
        uint4 *dst = reinterpret_cast<uint4 *>(s_bits);
        for (int w = tid; w < A.bits_b_smem_words / 4; w += kStarThreads) dst[w] = src[w];
    }
    if (tid < 3) s_stat[tid] = 0;
    __syncthreads();
    unsigned passed = 0, joined = 0, sectors = 0;
    int qn = 0;  // entries in this warp's queue (the same on every lane)

    const int64_t tstride = (int64_t)gridDim.x * kStarTile;
    int64_t t0 = (int64_t)blockIdx.x * kStarTile;
    long long nxt[kStarRows];
    const int64_t lane_off = (int64_t)tid * kStarRows;
    if (t0 < A.n) star_load_tile<VEC>(A, t0 + lane_off, nxt);
    for (; t0 < A.n; t0 += tstride) {
        long long cur[kStarRows];
#pragma unroll
        for (int j = 0; j < kStarRows; j++) cur[j] = nxt[j];
        if (t0 + tstride < A.n) star_load_tile<VEC>(A, t0 + tstride + lane_off, nxt);
#pragma unroll
        for (int half = 0; half < 2; half++) {
            // ---- stage 1: B's filter over 4 rows of this lane ----
            const int64_t r0 = t0 + lane_off + half * 4;
            unsigned m = 0;
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const long long k = cur[half * 4 + u];
                bool p = r0 + u < A.n;
                if (p && A.use_filters) {
                    if (BMODE == 1) p = star_bit(s_bits, A.fb.lo, A.fb.hi, k);
                    else p = A.bits_b ? star_bit(A.bits_b, A.fb.lo, A.fb.hi, k) : filter_pass(A.fb, k);
                }
                m |= (unsigned)p << u;
            }
            if (m) {
                // fk_a's sector of these 4 rows will be read in stage 2: start
                // bringing it into L2 now, so the drain waits on L2, not HBM.
                sectors++;
                asm volatile("prefetch.global.L2 [%0];" ::"l"(A.fk_a + r0));
            }
            const int np = __popc(m);
            int incl = np;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const int y = __shfl_up_sync(0xFFFFFFFFu, incl, d);
                if (lane >= d) incl += y;
            }
            int off = qn + incl - np;
            qn += __shfl_sync(0xFFFFFFFFu, incl, 31);
#pragma unroll
            for (int u = 0; u < 4; u++)
                if ((m >> u) & 1u) {
                    q_row[off] = (uint32_t)(r0 + u);
                    q_key[off] = cur[half * 4 + u];
                    off++;
                }
            __syncwarp();
            // ---- stage 2: 32 entries at a time from the queue's end ----
            while (qn >= 32) {
                qn -= 32;
                const uint32_t row = q_row[qn + lane];
                const long long kb = q_key[qn + lane];
                __syncwarp();
                star_stage2(A, row, kb, G, s_hi, s_lo, s_cnt, passed, joined);
            }
        }
    }
    if (lane < qn) star_stage2(A, q_row[lane], q_key[lane], G, s_hi, s_lo, s_cnt, passed, joined);
    atomicAdd(&s_stat[0], (unsigned long long)passed);
    atomicAdd(&s_stat[1], (unsigned long long)joined);
    atomicAdd(&s_stat[2], (unsigned long long)sectors);
    __syncthreads();
    for (int g = tid; g < G; g += kStarThreads)
        if (s_cnt[g]) {
            atomic_add_dd2(A.sum_hi + g, A.sum_lo + g, s_hi[g], s_lo[g]);
            atomicAdd(A.cnt + g, s_cnt[g]);
        }
    if (tid < 3 && s_stat[tid]) atomicAdd(A.stats + tid, s_stat[tid]);
}

// Evaluates a key filter for every value of [lo, lo + 32 * words) into an
// answer bitmap (bit v - lo).
__global__ void filter_bitmap_kernel(KeyFilterDev f, long long lo, uint64_t words, uint64_t values, uint32_t *out) {
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < words; w += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t word = 0;
        for (int j = 0; j < 32; j++) {
            const uint64_t v = w * 32 + j;
            if (v < values && filter_pass(f, lo + (long long)v)) word |= 1u << j;
        }
        out[w] = word;
    }
}

// Shared memory of one CTA for `bits_words` staged words and G groups.
inline size_t star_smem_bytes(int bits_words, int ngroups) {
    const int G = ngroups < kStarMaxSmemGroups ? ngroups : kStarMaxSmemGroups;
    return (size_t)bits_words * 4 + (size_t)kStarWarps * kStarWarpQueue * (4 + 8) + (size_t)G * 24;
}

}  // namespace krv
