// star_fused.cuh -- the fact-side kernels of the star-join pipeline.
//
// Dimension B's runtime filter is first evaluated once for every value of
// its key range [lo, hi] into an answer bitmap (bit v - lo = whether the
// filter passes v: the Bloom's answer, false positives included), staged in
// shared memory when it fits; a row's B test is then one bit. Without a
// bitmap the kernels probe the filter itself (range, then Bloom block or
// exact set).
//
// A dimension with unique keys over a range of at most 2^26 values also gets a
// direct index: its attribute's group id at key - lo (one byte or two, -1 =
// absent), so a probe is one L2 read instead of a hash-slot read and a key
// read. Otherwise the join's hash table is probed.
//
// Two kernels, so neither waits on the other's latency:
//  1. star_scan_kernel streams fk_b (each lane 8 consecutive values, the
//     warp 2 KB contiguous, the next tile prefetched into registers), tests
//     B's filter, and appends the passing rows (row, fk_b) to its CTA's region
//     of a survivor list, prefetching their fk_a sectors into L2;
//  2. star_join_kernel takes one survivor per thread over many CTAs: reads
//     fk_a, tests A's filter, looks both dimensions up and adds
//     price * (1 - discount) of each joined row to its group's accumulator.
// The fact side moves all of fk_b, the 32-byte sectors of fk_a holding a row
// that passed B's filter, price/discount of joined rows, and the survivor
// list (written once, read once).
#pragma once

#include "krv_device.cuh"
#include "krv_filter.cuh"
#include "ops.h"

namespace krv {

constexpr int kScanThreads = 1024;                        // threads per scan CTA
constexpr int kScanRows = 8;                              // rows per lane per tile
constexpr int kScanTile = kScanThreads * kScanRows;       // 8192 rows
constexpr int kJoinThreads = 512;                         // threads per join CTA
constexpr uint32_t kStarNone = 0xFFFFFFFFu;

struct StarTable {
    const unsigned long long *slots;
    uint64_t mask;
    const uint32_t *next;
    uint64_t seed;
    const long long *keys;  // build key column
    const int32_t *gid;     // dense group id of each build row's attribute
};

// key -> group id of a dimension with unique keys: gid at key - lo.
struct StarDirect {
    const void *gid;  // int8_t or int16_t per key value, -1 = no row
    long long lo;
    unsigned long long span;  // hi - lo
    int width;                // 1 or 2 (0: none)
};

struct StarArgs {
    const long long *fk_a, *fk_b, *price;
    const double *disc;
    int64_t n;
    KeyFilterDev fa, fb;
    const uint32_t *bits_b;  // B's answer bitmap over [fb.lo, fb.hi]
    int use_filters;
    int group_by;  // 0: dim A's attribute, 1: dim B's
    StarTable ta, tb;
    StarDirect da, db;
    int ngroups;
    int bits_b_smem_words;  // B's answer bitmap words staged in shared memory
    double *sum_hi, *sum_lo;
    unsigned long long *cnt;
    unsigned long long *stats;  // [0] rows passing both filters, [1] joined rows, [2] fk_a sectors read
    // Survivor list: CTA c of the scan owns entries [c * region, (c + 1) * region).
    uint32_t *surv_row;
    uint32_t *surv_kb32;   // fk_b - fb.lo (when B's range is below 2^32)
    long long *surv_kb64;  // fk_b (otherwise)
    uint64_t region;
    unsigned long long *region_count;
    // Validity bitmaps of the fact columns (null: no NULLs) and the bit of
    // row 0 in each. A NULL key never joins (join/keys.rs:17-19); a NULL
    // price or discount makes the row's value NULL, which SUM skips: the row
    // still joins and counts, and adds one to its group's `nulls`.
    const uint8_t *v_fk_a, *v_fk_b, *v_price, *v_disc;
    int64_t o_fk_a, o_fk_b, o_price, o_disc;
    unsigned long long *nulls;
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

__device__ __forceinline__ int star_direct(const StarDirect &d, long long k) {
    const unsigned long long off = (unsigned long long)(k - d.lo);
    if (off > d.span) return -1;
    return d.width == 1 ? (int)__ldg(static_cast<const int8_t *>(d.gid) + off)
                        : (int)__ldg(static_cast<const int16_t *>(d.gid) + off);
}

__device__ __forceinline__ unsigned long long warp_sum(unsigned long long v) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, d);
    return v;
}

template <bool VEC>
__device__ __forceinline__ void star_load_tile(const StarArgs &A, int64_t r0, long long (&v)[kScanRows]) {
    if (VEC && r0 + kScanRows <= A.n) {
        const longlong2 *p = reinterpret_cast<const longlong2 *>(A.fk_b + r0);
#pragma unroll
        for (int j = 0; j < kScanRows / 2; j++) {
            const longlong2 x = __ldcs(p + j);
            v[2 * j] = x.x;
            v[2 * j + 1] = x.y;
        }
    } else {
#pragma unroll
        for (int j = 0; j < kScanRows; j++) v[j] = r0 + j < A.n ? __ldcs(A.fk_b + r0 + j) : 0;
    }
}

// ---- stage 1 ------------------------------------------------------------------------
// BMODE 1: B's answer bitmap in shared memory; 0: B's filter probed per row.
// KB32: survivors keep fk_b - lo in 32 bits.
// NULLS: fact columns with validity bitmaps (compiled apart, so the kernel for
// columns without NULLs tests no bits).
template <int BMODE, bool VEC, bool KB32, bool NULLS>
__global__ void __launch_bounds__(kScanThreads, 1) star_scan_kernel(StarArgs A) {
    extern __shared__ __align__(16) uint8_t smem[];
    uint32_t *s_bits = reinterpret_cast<uint32_t *>(smem);
    __shared__ unsigned s_fill;
    __shared__ unsigned long long s_sectors;
    const int tid = threadIdx.x, lane = tid & 31;
    if (BMODE == 1) {
        const uint4 *src = reinterpret_cast<const uint4 *>(A.bits_b);
        uint4 *dst = reinterpret_cast<uint4 *>(s_bits);
        for (int w = tid; w < A.bits_b_smem_words / 4; w += kScanThreads) dst[w] = src[w];
    }
    if (tid == 0) {
        s_fill = 0;
        s_sectors = 0;
    }
    __syncthreads();
    const long long blo = A.fb.lo;
    const unsigned long long bspan = (unsigned long long)(A.fb.hi - A.fb.lo);
    const uint64_t region0 = (uint64_t)blockIdx.x * A.region;
    unsigned long long sectors = 0;

    const int64_t tstride = (int64_t)gridDim.x * kScanTile;
    int64_t t0 = (int64_t)blockIdx.x * kScanTile;
    long long nxt[kScanRows];
    const int64_t lane_off = (int64_t)tid * kScanRows;
    if (t0 < A.n) star_load_tile<VEC>(A, t0 + lane_off, nxt);
    for (; t0 < A.n; t0 += tstride) {
        long long cur[kScanRows];
#pragma unroll
        for (int j = 0; j < kScanRows; j++) cur[j] = nxt[j];
        if (t0 + tstride < A.n) star_load_tile<VEC>(A, t0 + tstride + lane_off, nxt);
        const int64_t r0 = t0 + lane_off;
        const bool full = r0 + kScanRows <= A.n;
        unsigned m = 0;
#pragma unroll
        for (int u = 0; u < kScanRows; u++) {
            bool p;
            if (!A.use_filters) {
                p = true;
            } else if (BMODE == 1) {
                // In range and the bit set; the offset fits 32 bits (range < 2^28).
                const unsigned long long off = (unsigned long long)(cur[u] - blo);
                const uint32_t o32 = (uint32_t)off;
                p = off <= bspan && ((s_bits[o32 >> 5] >> (o32 & 31)) & 1u);
            } else {
                p = filter_pass(A.fb, cur[u]);
            }
            if (!full && r0 + u >= A.n) p = false;
            if (NULLS && p && !bit_get(A.v_fk_b, A.o_fk_b, r0 + u)) p = false;
            m |= (unsigned)p << u;
        }
        // fk_a's 32-byte sectors of the passing rows will be read by stage 2.
        sectors += (unsigned long long)((m & 0x0Fu) != 0) + (unsigned long long)((m & 0xF0u) != 0);
        // Append the passing rows to this CTA's region: one shared atomic per warp.
        const int np = __popc(m);
        int incl = np;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int y = __shfl_up_sync(0xFFFFFFFFu, incl, d);
            if (lane >= d) incl += y;
        }
        const int total = __shfl_sync(0xFFFFFFFFu, incl, 31);
        unsigned base = 0;
        if (lane == 31 && total) base = atomicAdd(&s_fill, (unsigned)total);
        base = __shfl_sync(0xFFFFFFFFu, base, 31);
        if (m) {
            uint64_t pos = region0 + base + (unsigned)(incl - np);
#pragma unroll
            for (int u = 0; u < kScanRows; u++)
                if ((m >> u) & 1u) {
                    A.surv_row[pos] = (uint32_t)(r0 + u);
                    if (KB32) A.surv_kb32[pos] = (uint32_t)(cur[u] - blo);
                    else A.surv_kb64[pos] = cur[u];
                    pos++;
                }
        }
    }
    sectors = warp_sum(sectors);
    if (lane == 0 && sectors) atomicAdd(&s_sectors, sectors);
    __syncthreads();
    if (tid == 0) {
        A.region_count[blockIdx.x] = s_fill;
        if (s_sectors) atomicAdd(A.stats + 2, s_sectors);
    }
}

// ---- stage 2 ------------------------------------------------------------------------
// price * (1 - discount) of a row is NULL.
__device__ __forceinline__ bool star_value_null(const StarArgs &A, uint32_t row) {
    return (A.v_price && !bit_get(A.v_price, A.o_price, row)) || (A.v_disc && !bit_get(A.v_disc, A.o_disc, row));
}

// Adds v to the group of one joined pair: this warp's own accumulators in
// shared memory (lanes take turns, plain compensated adds: float64 atomics
// in shared memory are compare-and-swap loops) or, past them, the global ones.
__device__ __forceinline__ void star_add_plain(const StarArgs &A, int g, double v, double *w_hi, double *w_lo,
                                               unsigned long long *w_cnt, int G) {
    if (g < G) {
        double s, e;
        two_sum(w_hi[g], v, s, e);
        w_hi[g] = s;
        w_lo[g] = __dadd_rn(w_lo[g], e);
        w_cnt[g] += 1;
    } else {
        atomic_add_dd(A.sum_hi + g, A.sum_lo + g, v);
        atomicAdd(A.cnt + g, 1ull);
    }
}

// A's filter test of K keys at once: with a Bloom form the K block loads
// are issued together.
template <int K>
__device__ __forceinline__ void star_filterk(const KeyFilterDev &f, const long long (&k)[K], const bool (&has)[K],
                                             bool (&pass)[K]) {
    if (f.form == KRV_FILTER_BLOOM) {
        uint4 w0[K], w1[K];
        uint32_t key[K];
        bool in[K];
#pragma unroll
        for (int j = 0; j < K; j++) {
            in[j] = has[j] && !(f.has_range && (k[j] < f.lo || k[j] > f.hi));
            const uint64_t h = xxh64_u64((uint64_t)k[j]);
            key[j] = (uint32_t)h;
            const uint32_t *blk = f.bloom + (size_t)__umulhi((uint32_t)(h >> 32), (uint32_t)f.nblocks) * 8;
            if (in[j]) {
                w0[j] = __ldg(reinterpret_cast<const uint4 *>(blk));
                w1[j] = __ldg(reinterpret_cast<const uint4 *>(blk) + 1);
            }
        }
#pragma unroll
        for (int j = 0; j < K; j++) {
            const uint32_t miss = (sbbf_bit(key[j], 0) & ~w0[j].x) | (sbbf_bit(key[j], 1) & ~w0[j].y) |
                                  (sbbf_bit(key[j], 2) & ~w0[j].z) | (sbbf_bit(key[j], 3) & ~w0[j].w) |
                                  (sbbf_bit(key[j], 4) & ~w1[j].x) | (sbbf_bit(key[j], 5) & ~w1[j].y) |
                                  (sbbf_bit(key[j], 6) & ~w1[j].z) | (sbbf_bit(key[j], 7) & ~w1[j].w);
            pass[j] = in[j] && miss == 0;
        }
    } else {
#pragma unroll
        for (int j = 0; j < K; j++) pass[j] = has[j] && filter_pass(f, k[j]);
    }
}

// DIRECT: both dimensions have direct indexes; KB32 as in the scan. Each
// thread takes two survivors per step, each stage's loads issued together,
// so a thread keeps two probe chains in flight.
template <bool DIRECT, bool KB32, bool NULLS>
__global__ void __launch_bounds__(kJoinThreads, 2) star_join_kernel(StarArgs A, int regions, int slices, int G) {
    extern __shared__ __align__(16) uint8_t smem[];
    constexpr int kWarps = kJoinThreads / 32;
    constexpr int kK = 2;
    constexpr int kStep = kK * kJoinThreads;
    double *s_hi = reinterpret_cast<double *>(smem);
    double *s_lo = s_hi + kWarps * G;
    unsigned long long *s_cnt = reinterpret_cast<unsigned long long *>(s_lo + kWarps * G);
    __shared__ unsigned long long s_stat[2];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int i = tid; i < kWarps * G; i += kJoinThreads) {
        s_hi[i] = 0.0;
        s_lo[i] = 0.0;
        s_cnt[i] = 0;
    }
    if (tid < 2) s_stat[tid] = 0;
    __syncthreads();
    double *w_hi = s_hi + warp * G, *w_lo = s_lo + warp * G;
    unsigned long long *w_cnt = s_cnt + warp * G;
    unsigned long long passed = 0, joined = 0;
    const int r = blockIdx.x % regions, slice = blockIdx.x / regions;
    const uint64_t base0 = (uint64_t)r * A.region;
    const unsigned long long count = A.region_count[r];
    for (unsigned long long b = (unsigned long long)slice * kStep; b < count; b += (unsigned long long)slices * kStep) {
        bool has[kK], pa[kK], hit[kK];
        uint32_t row[kK];
        long long ka[kK], kb[kK];
        int g[kK];
        double v[kK];
#pragma unroll
        for (int j = 0; j < kK; j++) {
            const unsigned long long e = b + (unsigned long long)j * kJoinThreads + tid;
            has[j] = e < count;
            row[j] = has[j] ? A.surv_row[base0 + e] : 0u;
            kb[j] = !has[j] ? 0 : KB32 ? A.fb.lo + (long long)A.surv_kb32[base0 + e] : A.surv_kb64[base0 + e];
        }
        // Loads are issued a level at a time for all four entries; B's direct
        // index needs only fk_b, A's runs beside A's filter.
        int ga[kK], gb[kK];
#pragma unroll
        for (int j = 0; j < kK; j++) {
            ka[j] = has[j] ? __ldcs(A.fk_a + row[j]) : 0;
            if (DIRECT) gb[j] = has[j] ? star_direct(A.db, kb[j]) : -1;
        }
        if (DIRECT) {
#pragma unroll
            for (int j = 0; j < kK; j++) ga[j] = has[j] ? star_direct(A.da, ka[j]) : -1;
        }
        if (A.use_filters) star_filterk<kK>(A.fa, ka, has, pa);
        else {
#pragma unroll
            for (int j = 0; j < kK; j++) pa[j] = has[j];
        }
        if (NULLS) {
#pragma unroll
            for (int j = 0; j < kK; j++) pa[j] = pa[j] && bit_get(A.v_fk_a, A.o_fk_a, row[j]);
        }
        if (DIRECT) {
#pragma unroll
            for (int j = 0; j < kK; j++) {
                passed += pa[j];
                hit[j] = pa[j] && ga[j] >= 0 && gb[j] >= 0;
                g[j] = A.group_by == 0 ? ga[j] : gb[j];
                v[j] = 0.0;
                if (hit[j]) {
                    if (NULLS && star_value_null(A, row[j])) atomicAdd(A.nulls + g[j], 1ull);
                    else v[j] = __dmul_rn((double)__ldcs(A.price + row[j]), __dsub_rn(1.0, __ldcs(A.disc + row[j])));
                }
            }
#pragma unroll
            for (int j = 0; j < kK; j++) {
                // Lanes with a joined row add it in turn to the warp's accumulators.
                unsigned pend = __ballot_sync(0xFFFFFFFFu, hit[j]);
                while (pend) {
                    const int l = __ffs(pend) - 1;
                    pend &= pend - 1;
                    if (lane == l) {
                        joined++;
                        star_add_plain(A, g[j], v[j], w_hi, w_lo, w_cnt, G);
                    }
                    __syncwarp();
                }
            }
        } else {
#pragma unroll
            for (int j = 0; j < kK; j++) {
                passed += pa[j];
                uint32_t ra = kStarNone, rb0 = kStarNone;
                if (pa[j]) {
                    ra = star_lookup(A.ta, ka[j]);
                    if (ra != kStarNone) rb0 = star_lookup(A.tb, kb[j]);
                }
                const bool h = ra != kStarNone && rb0 != kStarNone;
                const bool vnull = NULLS && h && star_value_null(A, row[j]);
                double vv = 0.0;
                if (h && !vnull) vv = __dmul_rn((double)__ldcs(A.price + row[j]), __dsub_rn(1.0, __ldcs(A.disc + row[j])));
                unsigned pend = __ballot_sync(0xFFFFFFFFu, h);
                while (pend) {
                    const int l = __ffs(pend) - 1;
                    pend &= pend - 1;
                    if (lane == l) {
                        // every (a, b) match pair (chains are one long for unique keys)
                        for (int ca = 0; ra != kStarNone && ca < (1 << 20); ca++, ra = A.ta.next[ra]) {
                            int cb = 0;
                            for (uint32_t rb = rb0; rb != kStarNone && cb < (1 << 20); cb++, rb = A.tb.next[rb]) {
                                joined++;
                                const int gg = A.group_by == 0 ? A.ta.gid[ra] : A.tb.gid[rb];
                                if (vnull) atomicAdd(A.nulls + gg, 1ull);
                                star_add_plain(A, gg, vv, w_hi, w_lo, w_cnt, G);
                            }
                        }
                    }
                    __syncwarp();
                }
            }
        }
    }
    passed = warp_sum(passed);
    joined = warp_sum(joined);
    if (lane == 0) {
        if (passed) atomicAdd(&s_stat[0], passed);
        if (joined) atomicAdd(&s_stat[1], joined);
    }
    __syncthreads();
    for (int gi = tid; gi < G; gi += kJoinThreads) {
        double H = 0.0, L = 0.0;
        unsigned long long C = 0;
        for (int w = 0; w < kWarps; w++) {
            const unsigned long long c = s_cnt[w * G + gi];
            if (!c) continue;
            double s, e;
            two_sum(H, s_hi[w * G + gi], s, e);
            H = s;
            L = __dadd_rn(L, __dadd_rn(e, s_lo[w * G + gi]));
            C += c;
        }
        if (C) {
            atomic_add_dd2(A.sum_hi + gi, A.sum_lo + gi, H, L);
            atomicAdd(A.cnt + gi, C);
        }
    }
    if (tid < 2 && s_stat[tid]) atomicAdd(A.stats + tid, s_stat[tid]);
}

// Evaluates a key filter for every value of [lo, lo + values) into an answer
// bitmap (bit v - lo), one value per thread, one word per warp.
__global__ void filter_bitmap_kernel(KeyFilterDev f, long long lo, uint64_t words, uint64_t values, uint32_t *out) {
    const uint64_t total = words * 32;
    for (uint64_t base = blockIdx.x * (uint64_t)blockDim.x; base < total; base += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t v = base + threadIdx.x;
        const bool p = v < values && filter_pass(f, lo + (long long)v);
        const unsigned w = __ballot_sync(0xFFFFFFFFu, p);
        if ((threadIdx.x & 31) == 0 && v < total) out[v >> 5] = w;
    }
}

// Writes each dimension row's group id at its key's place of a direct index
// (the index starts all -1).
template <class T>
__global__ void direct_index_kernel(const long long *keys, const int32_t *gid, int64_t n, long long lo, T *out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[keys[i] - lo] = (T)gid[i];
}

// Shared memory of the scan: the staged bitmap words.
inline size_t star_scan_smem(int bits_words) { return (size_t)bits_words * 4; }
// Shared memory of the join kernel: per-warp accumulators of G groups.
inline size_t star_join_smem(int G) { return (size_t)(kJoinThreads / 32) * G * 24; }

}  // namespace krv
