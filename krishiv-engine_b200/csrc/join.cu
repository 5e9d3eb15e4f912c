// join.cu -- the hash join operator: build arena, open-addressing table over
// the engine's key hash, warp-cooperative probe with warp-aggregated output
// compaction fused with the payload gather, and the right/full join tails.
//
// Reference: crates/krishiv-exec/src/join/ (HashJoin, join/mod.rs:1014;
// BuildSink, join/build.rs; ProbeOp, join/probe.rs; JoinIndex,
// crates/krishiv-exec/src/rows/index.rs).
//
// Table layout (one per join): `slots` is a power-of-two array of u64,
// each (tag << 32) | (row + 1) with tag the top 32 bits of g = fin(h ^ seed)
// and 0 = empty, probed linearly from g & mask; `next` chains the build rows
// of one key newest-first (the reference's salted directory keeps a 16-bit
// salt and row + 1 the same way, rows/index.rs:1-32, 211-283). A probe reads
// a build row's key only when the 32-bit tag matches.
#include <algorithm>
#include <string>

#include "krv_device.cuh"
#include "ops.h"

namespace krv {

namespace {

constexpr uint32_t kNone = 0xFFFFFFFFu;
constexpr unsigned kFull = 0xFFFFFFFFu;

__device__ __forceinline__ bool key_valid(const KeyColDev &c, int64_t i) {
    return bit_get(c.valid, c.voff, i);
}

__device__ __forceinline__ void key_words(const KeyColDev &c, int64_t i, uint64_t &w0, uint64_t &w1) {
    if (c.width == 4) {
        w0 = static_cast<const uint32_t *>(c.data)[i];
        w1 = 0;
    } else if (c.width == 8) {
        w0 = static_cast<const uint64_t *>(c.data)[i];
        if (c.is_float) w0 = normalize_f64_bits(w0);
        w1 = 0;
    } else {
        const uint64_t *p = static_cast<const uint64_t *>(c.data) + 2 * i;
        w0 = p[0];
        w1 = p[1];
    }
}

// Every `=` key valid (join/keys.rs:17-19: a NULL `=` key never matches).
__device__ __forceinline__ bool matchable(const KeysDev &k, int64_t i) {
    for (int c = 0; c < k.n; c++)
        if (!((k.null_safe >> c) & 1u) && !key_valid(k.c[c], i)) return false;
    return true;
}

// The seedless row hash h (rows/layout.rs:487-555): NULL under a validity bit
// (null-safe key) mixes NULL_HASH, a value mixes its 8-byte words.
__device__ __forceinline__ uint64_t row_hash(const KeysDev &k, int64_t i) {
    uint64_t h = 0;  // fold(SEEDLESS = 0, MIX)
    for (int c = 0; c < k.n; c++) {
        if (!key_valid(k.c[c], i)) {
            if ((k.null_safe >> c) & 1u) h = mix(h, kNullHash);
            continue;
        }
        uint64_t w0, w1;
        key_words(k.c[c], i, w0, w1);
        h = mix(h, w0);
        if (k.c[c].width == 16) h = mix(h, w1);
    }
    return fold(h, kFinish);
}

__device__ __forceinline__ bool keys_eq(const KeysDev &a, int64_t i, const KeysDev &b, int64_t j) {
    for (int c = 0; c < a.n; c++) {
        const bool va = key_valid(a.c[c], i), vb = key_valid(b.c[c], j);
        if (va != vb) return false;
        if (!va) continue;
        uint64_t a0, a1, b0, b1;
        key_words(a.c[c], i, a0, a1);
        key_words(b.c[c], j, b0, b1);
        if (a0 != b0 || a1 != b1) return false;
    }
    return true;
}

// FAST: one non-float int64 key column.
template <bool FAST>
__device__ __forceinline__ uint64_t hash_of(const KeysDev &k, int64_t i) {
    if (FAST) return hash_word(static_cast<const uint64_t *>(k.c[0].data)[i]);
    return row_hash(k, i);
}
template <bool FAST>
__device__ __forceinline__ bool eq_of(const KeysDev &a, int64_t i, const KeysDev &b, int64_t j) {
    if (FAST)
        return static_cast<const int64_t *>(a.c[0].data)[i] == static_cast<const int64_t *>(b.c[0].data)[j];
    return keys_eq(a, i, b, j);
}

template <bool FAST>
__global__ void __launch_bounds__(256) build_kernel(KeysDev keys, int64_t n, unsigned long long *slots,
                                                    uint64_t mask, uint32_t *next, uint64_t seed,
                                                    unsigned long long *ctr, uint32_t *status) {
    // ctr: [0] distinct keys, [1] a NULL `=` key seen, [2] min / [3] max of an
    // int64 key (FAST), [4] indexed rows.
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    unsigned long long heads = 0, rows = 0;
    long long lo = LLONG_MAX, hi = LLONG_MIN;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += stride) {
        uint32_t nx = kNone;
        if (!matchable(keys, i)) {
            next[i] = nx;
            ctr[1] = 1;  // a NULL `=` key in the build (null-aware anti join)
            continue;
        }
        rows++;
        if (FAST) {
            const long long k = static_cast<const long long *>(keys.c[0].data)[i];
            lo = k < lo ? k : lo;
            hi = k > hi ? k : hi;
        }
        const uint64_t g = finalize(hash_of<FAST>(keys, i), seed);
        const unsigned long long entry = ((g >> 32) << 32) | (unsigned long long)(i + 1);
        uint64_t pos = g & mask;
        for (uint64_t probes = 0;; probes++) {
            if (probes > mask) {
                atomicOr(status, ST_CAPACITY);
                break;
            }
            unsigned long long s = __ldcg(slots + pos);
            if (s == 0) {
                const unsigned long long old = atomicCAS(slots + pos, 0ull, entry);
                if (old == 0) {
                    heads++;
                    break;
                }
                s = old;
            }
            if ((s >> 32) == (entry >> 32) && eq_of<FAST>(keys, i, keys, (int64_t)(s & 0xFFFFFFFFull) - 1)) {
                // Same key: this row becomes the head, the old head its next.
                const unsigned long long old = atomicExch(slots + pos, entry);
                nx = (uint32_t)(old & 0xFFFFFFFFull) - 1u;
                break;
            }
            pos = (pos + 1) & mask;
        }
        next[i] = nx;
    }
    // One atomic per warp and counter.
    for (int d = 16; d > 0; d >>= 1) {
        heads += __shfl_xor_sync(0xFFFFFFFFu, heads, d);
        rows += __shfl_xor_sync(0xFFFFFFFFu, rows, d);
        const long long ol = __shfl_xor_sync(0xFFFFFFFFu, lo, d), oh = __shfl_xor_sync(0xFFFFFFFFu, hi, d);
        lo = ol < lo ? ol : lo;
        hi = oh > hi ? oh : hi;
    }
    if ((threadIdx.x & 31) == 0) {
        if (heads) atomicAdd(ctr, heads);
        if (rows) atomicAdd(ctr + 4, rows);
        if (FAST && rows) {
            atomicMin(reinterpret_cast<long long *>(ctr + 2), lo);
            atomicMax(reinterpret_cast<long long *>(ctr + 3), hi);
        }
    }
}

template <bool FAST>
__device__ __forceinline__ uint32_t lookup(const KeysDev &pk, int64_t i, const KeysDev &bk,
                                           const unsigned long long *slots, uint64_t mask, uint64_t seed) {
    const uint64_t g = finalize(hash_of<FAST>(pk, i), seed);
    const unsigned long long tag = g >> 32;
    uint64_t pos = g & mask;
    for (uint64_t probes = 0; probes <= mask; probes++) {
        const unsigned long long s = __ldg(slots + pos);
        if (s == 0) return kNone;
        if ((s >> 32) == tag) {
            const int64_t o = (int64_t)(s & 0xFFFFFFFFull) - 1;
            if (eq_of<FAST>(pk, i, bk, o)) return (uint32_t)o;
        }
        pos = (pos + 1) & mask;
    }
    return kNone;
}

// ---- residual filter (JoinSpec::filter, join/probe.rs:425-436) -------------------
__device__ __forceinline__ bool filter_operand(const FilterOpDev &o, int64_t p, uint32_t b, long long &iv, double &fv) {
    if (o.side == 2) {
        iv = o.ci;
        fv = o.is_float ? o.cf : (double)o.ci;
        return true;
    }
    const int64_t r = o.side == 0 ? p : (int64_t)b;
    if (!bit_get(o.valid, o.voff, r)) return false;
    if (o.width == 4) {
        iv = static_cast<const int *>(o.data)[r];
        fv = (double)iv;
    } else if (o.is_float) {
        fv = static_cast<const double *>(o.data)[r];
        iv = 0;
    } else {
        iv = static_cast<const long long *>(o.data)[r];
        fv = (double)iv;
    }
    return true;
}
template <class T>
__device__ __forceinline__ bool compare(int op, T a, T b) {
    switch (op) {
    case KRV_CMP_EQ: return a == b;
    case KRV_CMP_NE: return a != b;
    case KRV_CMP_LT: return a < b;
    case KRV_CMP_LE: return a <= b;
    case KRV_CMP_GT: return a > b;
    default: return a >= b;
    }
}
__device__ bool filter_true(const FilterDev &F, int64_t p, uint32_t b) {
    for (int t = 0; t < F.n; t++) {
        const FilterTermDev &T = F.t[t];
        long long li, ri;
        double lf, rf;
        if (!filter_operand(T.l, p, b, li, lf) || !filter_operand(T.r, p, b, ri, rf)) return false;
        const bool ok = T.as_float ? compare(T.op, f64_order_key(lf), f64_order_key(rf)) : compare(T.op, li, ri);
        if (!ok) return false;
    }
    return true;
}
// The first build row of the chain from `cur` (newest first) whose pair
// with probe row p passes the filter.
__device__ __forceinline__ uint32_t first_true(const FilterDev &F, int64_t p, uint32_t cur, const uint32_t *next) {
    while (cur != kNone && !filter_true(F, p, cur)) cur = next[cur];
    return cur;
}

struct OutColDev {
    const void *src;
    const uint8_t *src_valid;
    int64_t src_voff;
    void *dst;
    uint32_t *dst_valid;  // zeroed bitmap words, or null (non-nullable output)
    int32_t width;
    int32_t side;         // 0 probe row, 1 build row, 2 constant NULL; 3 / 4 the probe / build row
                          // index itself (int64, -1 for a NULL side): the rows string columns are gathered from
};
struct OutDev {
    OutColDev c[2 * KRV_MAX_OUT_COLUMNS];
    int32_t n;
};

__device__ __forceinline__ void copy_value(void *dst, const void *src, int64_t di, int64_t si, int w) {
    switch (w) {
    case 1: static_cast<uint8_t *>(dst)[di] = static_cast<const uint8_t *>(src)[si]; break;
    case 4: static_cast<uint32_t *>(dst)[di] = static_cast<const uint32_t *>(src)[si]; break;
    case 8: static_cast<uint64_t *>(dst)[di] = static_cast<const uint64_t *>(src)[si]; break;
    default:
        static_cast<uint4 *>(dst)[di] = static_cast<const uint4 *>(src)[si];
        break;
    }
}
__device__ __forceinline__ void zero_value(void *dst, int64_t di, int w) {
    switch (w) {
    case 1: static_cast<uint8_t *>(dst)[di] = 0; break;
    case 4: static_cast<uint32_t *>(dst)[di] = 0; break;
    case 8: static_cast<uint64_t *>(dst)[di] = 0; break;
    default: static_cast<uint4 *>(dst)[di] = make_uint4(0, 0, 0, 0); break;
    }
}

// Writes one round of a warp's output rows: lane `want` writes row `pos`
// from probe row `prow` and build row `brow` (kNone: NULL build side; a
// negative prow: NULL probe side). Validity bits of the round are combined in
// rank order and OR-ed in with at most two atomics per column.
__device__ __forceinline__ void emit_round(const OutDev &out, bool want, unsigned long long pos,
                                           unsigned long long first, int64_t prow, uint32_t brow,
                                           unsigned long long cap) {
    const unsigned ballot = __ballot_sync(kFull, want);
    const unsigned rank = __popc(ballot & lanemask_lt());
    for (int k = 0; k < out.n; k++) {
        const OutColDev &c = out.c[k];
        bool v = false;
        if (want && pos < cap) {
            if (c.side == 3) {
                static_cast<long long *>(c.dst)[pos] = prow >= 0 ? prow : -1;
            } else if (c.side == 4) {
                static_cast<long long *>(c.dst)[pos] = brow != kNone ? (long long)brow : -1;
            } else if (c.side == 0 && prow >= 0) {
                copy_value(c.dst, c.src, (int64_t)pos, prow, c.width);
                v = bit_get(c.src_valid, c.src_voff, prow);
            } else if (c.side == 1 && brow != kNone) {
                copy_value(c.dst, c.src, (int64_t)pos, brow, c.width);
                v = bit_get(c.src_valid, c.src_voff, brow);
            } else {
                zero_value(c.dst, (int64_t)pos, c.width);
            }
        }
        if (c.dst_valid) {
            const unsigned m = __reduce_or_sync(kFull, (want && v) ? (1u << rank) : 0u);
            if (lane_id() == 0 && m) {
                const unsigned long long w = first >> 5;
                const unsigned sh = (unsigned)(first & 31);
                const unsigned long long capw = (cap + 31) >> 5;
                if (w < capw) atomicOr(c.dst_valid + w, m << sh);
                if (sh && w + 1 < capw && (m >> (32 - sh))) atomicOr(c.dst_valid + w + 1, m >> (32 - sh));
            }
        }
    }
}

// Allocates this round's output rows for the warp: returns the first row of
// the round (same on every lane) and this lane's row.
__device__ __forceinline__ unsigned long long round_alloc(unsigned long long *count, bool want,
                                                          unsigned long long &pos) {
    const unsigned ballot = __ballot_sync(kFull, want);
    unsigned long long first = 0;
    if (lane_id() == 0 && ballot) first = atomicAdd(count, (unsigned long long)__popc(ballot));
    first = __shfl_sync(kFull, first, 0);
    pos = first + __popc(ballot & lanemask_lt());
    return first;
}

// Pairs: inner, left outer, right outer, full outer (join/probe.rs:266-502).
template <bool FAST, bool FILT>
__global__ void __launch_bounds__(256) probe_pairs_kernel(KeysDev pk, KeysDev bk, int64_t n,
                                                          const unsigned long long *slots, uint64_t mask,
                                                          const uint32_t *next, uint64_t seed, OutDev out,
                                                          unsigned long long cap, unsigned long long *count,
                                                          uint8_t *marks, int pads_probe, int single_match,
                                                          uint32_t *status, unsigned long long *max_chain,
                                                          FilterDev F) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t base = blockIdx.x * (int64_t)blockDim.x; base < n; base += stride) {
        const int64_t i = base + threadIdx.x;
        const bool live = i < n;
        uint32_t cur = kNone;
        if (live && matchable(pk, i)) cur = lookup<FAST>(pk, i, bk, slots, mask, seed);
        if (FILT) cur = first_true(F, i, cur, next);
        bool pad = live && cur == kNone && pads_probe;
        unsigned chain = 0;
        while (__any_sync(kFull, cur != kNone || pad)) {
            const bool want = cur != kNone || pad;
            unsigned long long pos;
            const unsigned long long first = round_alloc(count, want, pos);
            emit_round(out, want, pos, first, i, cur, cap);
            if (cur != kNone) {
                if (marks) marks[cur] = 1;
                chain++;
                cur = next[cur];
                if (FILT) cur = first_true(F, i, cur, next);
            } else {
                pad = false;
            }
        }
        if (single_match && chain > 1) atomicOr(status, ST_TOO_MANY);
        if (chain > 1) atomicMax(max_chain, (unsigned long long)chain);
    }
}

// Pairs of an inner or left outer join on one int64 `=` key over a build
// side with unique keys, with no build marks: every probe row has at most one
// output row, so the kernel has no chain walks and no per-row loops, and its
// warps stay converged. Every lane resolves kFastRows probe rows at once
// (their slot loads in flight together); the CTA scans its warps' counts in
// shared memory and reserves its run of the output with one atomic per
// kFastRows x 256 probe rows. Validity bits of nullable output columns are
// set with one atomicOr per valid value.
//
// DIRECT: the build keys are also dense (their span at most a few times the
// row count), and a direct index (key - lo -> build row) replaces the table:
// one load per probe row instead of a slot load and a key compare.
constexpr int kFastRows = 4;
constexpr int kFastThreads = 256;
struct DirectDev {
    const uint32_t *row;  // build row of key lo + i, kNone where no row has it
    long long lo;
    unsigned long long span;  // hi - lo
};

__global__ void direct_build_kernel(KeysDev bk, int64_t n, DirectDev d) {
    const long long *keys = static_cast<const long long *>(bk.c[0].data);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        if (!key_valid(bk.c[0], i)) continue;
        const unsigned long long off = (unsigned long long)keys[i] - (unsigned long long)d.lo;
        if (off <= d.span) const_cast<uint32_t *>(d.row)[off] = (uint32_t)i;
    }
}

template <bool DIRECT>
__global__ void __launch_bounds__(kFastThreads) probe_fast_kernel(KeysDev pk, KeysDev bk, int64_t n,
                                                                  const unsigned long long *slots, uint64_t mask,
                                                                  uint64_t seed, DirectDev dir, OutDev out,
                                                                  unsigned long long cap, unsigned long long *count,
                                                                  int pad) {
    constexpr int kWarps = kFastThreads / 32;
    __shared__ unsigned s_warp[kWarps];
    __shared__ unsigned long long s_base;
    const long long *pkeys = static_cast<const long long *>(pk.c[0].data);
    const long long *bkeys = static_cast<const long long *>(bk.c[0].data);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t tile = (int64_t)kFastThreads * kFastRows;
    for (int64_t base = (int64_t)blockIdx.x * tile; base < n; base += (int64_t)gridDim.x * tile) {
        int64_t row[kFastRows];
        uint32_t head[kFastRows];
        long long key[kFastRows];
        uint64_t pos[kFastRows];
        unsigned long long tag[kFastRows], slot[kFastRows];
        bool live[kFastRows];
#pragma unroll
        for (int u = 0; u < kFastRows; u++) {
            row[u] = base + (int64_t)u * kFastThreads + threadIdx.x;
            live[u] = row[u] < n && key_valid(pk.c[0], row[u]);
            key[u] = live[u] ? pkeys[row[u]] : 0;
            if (DIRECT) continue;
            const uint64_t g = finalize(hash_word((uint64_t)key[u]), seed);
            tag[u] = g >> 32;
            pos[u] = g & mask;
        }
        if (DIRECT) {
#pragma unroll
            for (int u = 0; u < kFastRows; u++) {
                const unsigned long long off = (unsigned long long)key[u] - (unsigned long long)dir.lo;
                head[u] = live[u] && off <= dir.span ? __ldg(dir.row + off) : kNone;
            }
        }
#pragma unroll
        for (int u = 0; u < kFastRows; u++) slot[u] = !DIRECT && live[u] ? __ldg(slots + pos[u]) : 0ull;
#pragma unroll
        for (int u = 0; u < kFastRows; u++) {
            if (DIRECT) break;
            head[u] = kNone;
            if (!live[u]) continue;
            unsigned long long sl = slot[u];
            uint64_t p = pos[u];
            for (uint64_t probes = 0; probes <= mask && sl != 0; probes++) {
                if ((sl >> 32) == tag[u]) {
                    const uint32_t o = (uint32_t)(sl & 0xFFFFFFFFull) - 1u;
                    if (__ldg(bkeys + o) == key[u]) {
                        head[u] = o;
                        break;
                    }
                }
                p = (p + 1) & mask;
                sl = __ldg(slots + p);
            }
        }
        bool emit[kFastRows];
        unsigned mine = 0;
#pragma unroll
        for (int u = 0; u < kFastRows; u++) {
            emit[u] = row[u] < n && (head[u] != kNone || pad);
            mine += emit[u];
        }
        unsigned incl = mine;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const unsigned y = __shfl_up_sync(kFull, incl, d);
            if (lane >= d) incl += y;
        }
        if (lane == 31) s_warp[warp] = incl;
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned acc = 0;
            for (int w = 0; w < kWarps; w++) {
                const unsigned c = s_warp[w];
                s_warp[w] = acc;
                acc += c;
            }
            s_base = acc ? atomicAdd(count, (unsigned long long)acc) : 0ull;
        }
        __syncthreads();
        unsigned long long at = s_base + s_warp[warp] + (incl - mine);
        __syncthreads();  // s_warp and s_base are rewritten by the next tile
#pragma unroll
        for (int u = 0; u < kFastRows; u++) {
            if (!emit[u]) continue;
            const unsigned long long a = at++;
            if (a >= cap) continue;
            const uint32_t b = head[u];
            for (int k = 0; k < out.n; k++) {
                const OutColDev &c = out.c[k];
                bool v = false;
                if (c.side == 3) {
                    static_cast<long long *>(c.dst)[a] = row[u];
                } else if (c.side == 4) {
                    static_cast<long long *>(c.dst)[a] = b != kNone ? (long long)b : -1;
                } else if (c.side == 0) {
                    copy_value(c.dst, c.src, (int64_t)a, row[u], c.width);
                    v = bit_get(c.src_valid, c.src_voff, row[u]);
                } else if (b != kNone) {
                    copy_value(c.dst, c.src, (int64_t)a, b, c.width);
                    v = bit_get(c.src_valid, c.src_voff, b);
                } else {
                    zero_value(c.dst, (int64_t)a, c.width);
                }
                if (c.dst_valid && v) atomicOr(c.dst_valid + (a >> 5), 1u << (a & 31));
            }
        }
    }
}

// Probe rows once: semi, anti, null-aware anti (join/mod.rs:27-34).
// kind 0 semi, 1 anti, 2 null-aware anti.
template <bool FAST, bool FILT>
__global__ void __launch_bounds__(256) probe_rows_kernel(KeysDev pk, KeysDev bk, int64_t n,
                                                         const unsigned long long *slots, uint64_t mask,
                                                         uint64_t seed, OutDev out, unsigned long long cap,
                                                         unsigned long long *count, int kind, int build_empty,
                                                         int build_has_null, const uint32_t *next, FilterDev F) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t base = blockIdx.x * (int64_t)blockDim.x; base < n; base += stride) {
        const int64_t i = base + threadIdx.x;
        const bool live = i < n;
        bool ok = false;
        if (live) {
            const bool m = matchable(pk, i);
            uint32_t c = m && !build_empty ? lookup<FAST>(pk, i, bk, slots, mask, seed) : kNone;
            if (FILT) c = first_true(F, i, c, next);
            const bool hit = c != kNone;
            if (kind == 0) ok = hit;
            else if (kind == 1) ok = !hit;
            else ok = build_empty || (!build_has_null && m && !hit);
        }
        unsigned long long pos;
        const unsigned long long first = round_alloc(count, ok, pos);
        emit_round(out, ok, pos, first, i, kNone, cap);
    }
}

// Existence: every probe row once plus `exists` (join/mod.rs:35-45). Rows
// keep their positions; the flag of rows [base, base + 32) is one word.
template <bool FAST, bool FILT>
__global__ void __launch_bounds__(256) probe_exists_kernel(KeysDev pk, KeysDev bk, int64_t n,
                                                           const unsigned long long *slots, uint64_t mask,
                                                           uint64_t seed, uint32_t *exists, int build_empty,
                                                           const uint32_t *next, FilterDev F) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t base = blockIdx.x * (int64_t)blockDim.x; base < n; base += stride) {
        const int64_t i = base + threadIdx.x;
        bool hit = false;
        if (i < n && !build_empty && matchable(pk, i)) {
            uint32_t c = lookup<FAST>(pk, i, bk, slots, mask, seed);
            if (FILT) c = first_true(F, i, c, next);
            hit = c != kNone;
        }
        const unsigned word = __ballot_sync(kFull, hit);
        if (lane_id() == 0 && (i < n)) exists[i >> 5] = word;
    }
}

// Build rows by their marks once the probe side is done (emit_build,
// join/probe.rs:610-): kind 0 right semi (marked rows with a matchable key),
// kind 1 unmatched rows (right anti, right outer, full outer).
__global__ void __launch_bounds__(256) tail_kernel(int64_t nb, const uint8_t *marks, KeysDev bk, int kind,
                                                   OutDev out, unsigned long long cap,
                                                   unsigned long long *count) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t base = blockIdx.x * (int64_t)blockDim.x; base < nb; base += stride) {
        const int64_t r = base + threadIdx.x;
        bool ok = false;
        if (r < nb) ok = kind == 0 ? (marks[r] != 0 && matchable(bk, r)) : marks[r] == 0;
        unsigned long long pos;
        const unsigned long long first = round_alloc(count, ok, pos);
        emit_round(out, ok, pos, first, -1, ok ? (uint32_t)r : kNone, cap);
    }
}

void zero(Runtime *rt, void *p, size_t bytes) {
    if (bytes) KRV_CUDA(cudaMemsetAsync(p, 0, bytes, rt->stream));
}

}  // namespace

KeysDev keys_of(const DevBatch &b, const int32_t *cols, int n, const int32_t *null_safe) {
    KeysDev k{};
    k.n = n;
    for (int i = 0; i < n; i++) {
        if (cols[i] < 0 || cols[i] >= (int)b.cols.size()) fail(KRV_INVALID_ARGUMENT, "key column out of range");
        const DevCol &c = b.cols[cols[i]];
        const int w = c.type.width();
        if (w != 4 && w != 8 && w != 16) fail(KRV_UNSUPPORTED, "key column of type " + c.type.format());
        k.c[i] = KeyColDev{c.data, c.valid, c.valid_off, w, c.type.id == Type::F64 ? 1 : 0};
        if (null_safe && null_safe[i]) k.null_safe |= 1u << i;
    }
    return k;
}

namespace {
// The join's own key hash for every row, as the build and probe kernels
// compute it: h (row_hash), g = fin(h ^ seed), and the partition at `depth`
// (0: the top `radix` bits of h; d >= 1: bits [48-3d, 51-3d) of g).
__global__ void __launch_bounds__(256) hash_rows_kernel(KeysDev k, int64_t n, uint64_t seed, int depth, int radix,
                                                        uint64_t *out_h, uint64_t *out_g, int32_t *out_part) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint64_t h = row_hash(k, i);
        const uint64_t g = finalize(h, seed);
        if (out_h) out_h[i] = h;
        if (out_g) out_g[i] = g;
        if (out_part) out_part[i] = depth == 0 ? (int32_t)(h >> (64 - radix)) : (int32_t)((g >> (48 - 3 * depth)) & 7u);
    }
}
}  // namespace

void hash_rows(Runtime *rt, const DevBatch &b, const int32_t *cols, int n, const int32_t *null_safe, uint64_t seed,
               int depth, int radix, uint64_t *out_h, uint64_t *out_g, int32_t *out_part) {
    if (n < 1 || n > KRV_MAX_KEYS) fail(KRV_INVALID_ARGUMENT, "1 to 4 key columns");
    // Hashing::partition (join/keys.rs:92-95, 118-128): radix 3..6, depth 0..6
    radix = std::min(6, std::max(3, radix));
    if (depth < 0) fail(KRV_INVALID_ARGUMENT, "negative partition depth");
    depth = std::min(depth, 6);
    const KeysDev k = keys_of(b, cols, n, null_safe);
    if (b.rows == 0) return;
    hash_rows_kernel<<<grid_for(rt, b.rows, 256, 8), 256, 0, rt->stream>>>(k, b.rows, seed, depth, radix, out_h, out_g,
                                                                          out_part);
    rt->launches++;
    check_launch("hash_rows_kernel");
}

static bool fast_keys(const KeysDev &k) { return k.n == 1 && k.c[0].width == 8 && !k.c[0].is_float; }

HashJoin::HashJoin(Runtime *rt, const krv_join_spec &spec) : rt_(rt), spec_(spec) {
    if (spec.n_keys < 1 || spec.n_keys > KRV_MAX_KEYS) fail(KRV_INVALID_ARGUMENT, "join needs 1..4 keys");
    if (spec.join_type < KRV_JOIN_INNER || spec.join_type > KRV_JOIN_FULL_OUTER)
        fail(KRV_INVALID_ARGUMENT, "unknown join type");
    if (spec.has_residual_filter && spec.join_type == KRV_JOIN_NULL_AWARE_ANTI)
        fail(KRV_UNSUPPORTED, "KRISHIV_UNSUPPORTED_FEATURE: null-aware anti join with a residual condition");
    if (spec.single_match && spec.join_type != KRV_JOIN_LEFT_OUTER)
        fail(KRV_INVALID_ARGUMENT, "single_match is for left outer joins only");
    if (spec.join_type == KRV_JOIN_NULL_AWARE_ANTI && (spec.n_keys != 1 || spec.null_safe[0]))
        fail(KRV_INVALID_ARGUMENT, "a null-aware anti join has one `=` key");
    if (spec.n_probe_out > KRV_MAX_OUT_COLUMNS || spec.n_build_out > KRV_MAX_OUT_COLUMNS)
        fail(KRV_INVALID_ARGUMENT, "too many output columns");
    if (spec_.max_load <= 0.f || spec_.max_load > 0.9f) spec_.max_load = 0.5f;
    if (spec_.seed == 0) spec_.seed = 0x4B52565F4A4F494EULL;  // fixed: results never depend on it
    counters_.partitions = 1;
}

void HashJoin::append_arena(const DevBatch &b) {
    if (!have_schema_) {
        for (const DevCol &c : b.cols) {
            DevCol a;
            a.type = c.type;
            a.name = c.name;
            a.nullable = c.nullable;
            arena_cols_.push_back(a);
        }
        arena_data_.resize(b.cols.size());
        arena_valid_.resize(b.cols.size());
        have_schema_ = true;
    } else {
        if (b.cols.size() != arena_cols_.size()) fail(KRV_INVALID_ARGUMENT, "build batches differ in columns");
        for (size_t i = 0; i < b.cols.size(); i++)
            if (b.cols[i].type != arena_cols_[i].type) fail(KRV_INVALID_ARGUMENT, "build batches differ in types");
    }
    const int64_t need = build_rows_ + b.rows;
    if (need > (int64_t)0xFFFFFFFEll) fail(KRV_UNSUPPORTED, "more than 2^32-2 build rows in one table");
    if (need > arena_cap_) {
        int64_t cap = std::max<int64_t>({need, arena_cap_ * 2, spec_.build_rows_hint, 1024});
        if (arena_var_.size() < arena_cols_.size()) arena_var_.resize(arena_cols_.size());
        for (size_t i = 0; i < arena_cols_.size(); i++) {
            const DType t = arena_cols_[i].type;
            // a string column keeps a start (int64) per row here and its length beside
            const size_t w = t.var() ? 8 : (size_t)t.width();
            const size_t bytes = t.id == Type::Bool ? (size_t)ceil_div(cap, 8) : (size_t)cap * w;
            auto nd = std::make_shared<DBuf>(rt_, bytes);
            auto nv = std::make_shared<DBuf>(rt_, (size_t)ceil_div(cap, 32) * 4 + 8);
            zero(rt_, nv->get(), nv->bytes());
            std::shared_ptr<DBuf> nl;
            if (t.var()) nl = std::make_shared<DBuf>(rt_, (size_t)cap * 4);
            if (build_rows_) {
                const size_t old = t.id == Type::Bool ? (size_t)ceil_div(build_rows_, 8) : (size_t)build_rows_ * w;
                KRV_CUDA(cudaMemcpyAsync(nd->get(), arena_data_[i]->get(), old, cudaMemcpyDeviceToDevice, rt_->stream));
                KRV_CUDA(cudaMemcpyAsync(nv->get(), arena_valid_[i]->get(), (size_t)ceil_div(build_rows_, 8),
                                         cudaMemcpyDeviceToDevice, rt_->stream));
                if (nl)
                    KRV_CUDA(cudaMemcpyAsync(nl->get(), arena_var_[i].lens->get(), (size_t)build_rows_ * 4,
                                             cudaMemcpyDeviceToDevice, rt_->stream));
            }
            arena_data_[i] = nd;
            arena_valid_[i] = nv;
            if (nl) {
                arena_var_[i].starts = nd;
                arena_var_[i].lens = nl;
            }
        }
        arena_cap_ = cap;
    }
    for (size_t i = 0; i < arena_cols_.size(); i++) {
        const DevCol &c = b.cols[i];
        const DType t = c.type;
        if (t.id == Type::Bool) fail(KRV_UNSUPPORTED, "boolean build columns");
        if (c.valid) arena_cols_[i].nullable = true;
        if (b.rows == 0) continue;  // an empty batch only fixes the schema
        if (t.var()) {
            var_arena_append(rt_, arena_var_[i], c, build_rows_, b.rows);
        } else {
            const size_t w = (size_t)t.width();
            KRV_CUDA(cudaMemcpyAsync(arena_data_[i]->as<uint8_t>() + build_rows_ * w, c.data, (size_t)b.rows * w,
                                     cudaMemcpyDeviceToDevice, rt_->stream));
        }
        append_bits(rt_, c.valid, c.valid_off, b.rows, arena_valid_[i]->as<uint8_t>(), build_rows_);
    }
    build_rows_ = need;
}

void HashJoin::build_adopt(DevBatch b) {
    if (built_ || have_schema_) fail(KRV_INVALID_ARGUMENT, "build_adopt takes the whole build side, before any push");
    if (b.rows > (int64_t)0xFFFFFFFEll) fail(KRV_UNSUPPORTED, "more than 2^32-2 build rows in one table");
    for (const DevCol &c : b.cols) {
        if (!c.hold_data || c.hold_data->get() != c.data) fail(KRV_INVALID_ARGUMENT, "build_adopt needs owned columns");
        if (c.type.id == Type::Bool) fail(KRV_UNSUPPORTED, "boolean build columns");
        DevCol m;
        m.type = c.type;
        m.name = c.name;
        m.nullable = c.nullable || c.valid;
        arena_cols_.push_back(m);
        arena_data_.push_back(c.hold_data);
        arena_valid_.push_back(c.valid && c.valid_off == 0 ? c.hold_valid : nullptr);
        if (c.valid && (c.valid_off != 0 || !c.hold_valid)) fail(KRV_INVALID_ARGUMENT, "build_adopt needs owned bitmaps");
    }
    have_schema_ = true;
    build_rows_ = b.rows;
    arena_cap_ = b.rows;
}

HashJoin::~HashJoin() = default;

VarSrc HashJoin::var_src(int side, int col, const DevBatch *probe) const {
    VarSrc v{};
    if (side == 0) {
        const DevCol &c = probe->cols[col];
        v.offs = static_cast<const int32_t *>(c.data);
        v.bytes = static_cast<const uint8_t *>(c.bytes);
        v.valid = c.valid;
        v.voff = c.valid_off;
        return v;
    }
    if (col >= (int)arena_var_.size() || !arena_var_[col].starts) return v;  // no build rows: never read
    const VarArena &a = arena_var_[col];
    v.starts = a.starts->as<long long>();
    v.lens = a.lens->as<int32_t>();
    v.bytes = a.heap ? a.heap->as<uint8_t>() : nullptr;
    v.valid = arena_cols_[col].nullable ? arena_valid_[col]->as<uint8_t>() : nullptr;
    return v;
}

DevCol HashJoin::empty_col(const DevCol &meta) const {
    if (meta.type.var()) return var_gather(rt_, VarSrc{}, nullptr, 0, meta.type, meta.nullable, meta.name);
    return make_col(rt_, meta.type, 0, meta.nullable, meta.name);
}

void HashJoin::set_filter(const krv_join_filter &f) {
    if (decided_) fail(KRV_INVALID_ARGUMENT, "krv_join_set_filter after the first build push");
    if (spec_.join_type == KRV_JOIN_NULL_AWARE_ANTI)
        fail(KRV_UNSUPPORTED, "KRISHIV_UNSUPPORTED_FEATURE: null-aware anti join with a residual condition");
    if (f.n_terms < 1 || f.n_terms > KRV_MAX_FILTER_TERMS)
        fail(KRV_INVALID_ARGUMENT, "a residual filter has 1 to 8 comparisons");
    for (int t = 0; t < f.n_terms; t++) {
        const krv_filter_term &T = f.terms[t];
        if (T.op < KRV_CMP_EQ || T.op > KRV_CMP_GE) fail(KRV_INVALID_ARGUMENT, "unknown comparison");
        for (const krv_filter_operand *o : {&T.left, &T.right})
            if (o->kind < KRV_OPERAND_PROBE || o->kind > KRV_OPERAND_CONST_F64)
                fail(KRV_INVALID_ARGUMENT, "unknown filter operand kind");
    }
    residual_ = f;
    residual_set_ = true;
    spec_.has_residual_filter = 1;
}

// The device form of the residual filter over probe batch `in` and the arena.
FilterDev HashJoin::filter_dev(const DevBatch &in) const {
    FilterDev F{};
    F.n = residual_.n_terms;
    auto operand = [&](const krv_filter_operand &o, FilterOpDev &d, DType &t) {
        d.side = o.kind == KRV_OPERAND_PROBE ? 0 : o.kind == KRV_OPERAND_BUILD ? 1 : 2;
        if (d.side == 2) {
            d.is_float = o.kind == KRV_OPERAND_CONST_F64;
            d.ci = o.i64;
            d.cf = o.f64;
            t = DType{d.is_float ? Type::F64 : Type::I64, 0, 0};
            return;
        }
        const int ncol = d.side == 0 ? (int)in.cols.size() : (int)arena_cols_.size();
        if (o.column < 0 || o.column >= ncol) fail(KRV_INVALID_ARGUMENT, "residual filter column out of range");
        const DevCol &meta = d.side == 0 ? in.cols[o.column] : arena_cols_[o.column];
        t = meta.type;
        if (t.id != Type::I32 && t.id != Type::Date32 && t.id != Type::I64 && t.id != Type::Dec64 && t.id != Type::F64)
            fail(KRV_UNSUPPORTED, "a residual filter over " + t.format() + " columns");
        d.width = t.width();
        d.is_float = t.id == Type::F64;
        if (d.side == 0) {
            d.data = meta.data;
            d.valid = meta.valid;
            d.voff = meta.valid_off;
        } else if (!arena_.cols.empty()) {
            const DevCol &c = arena_.cols[o.column];
            d.data = c.data;
            d.valid = meta.nullable ? c.valid : nullptr;
            d.voff = c.valid_off;
        }
    };
    for (int t = 0; t < F.n; t++) {
        const krv_filter_term &T = residual_.terms[t];
        FilterTermDev &D = F.t[t];
        D.op = T.op;
        DType lt, rt;
        operand(T.left, D.l, lt);
        operand(T.right, D.r, rt);
        D.as_float = D.l.is_float || D.r.is_float;
        const bool ldec = lt.id == Type::Dec64, rdec = rt.id == Type::Dec64;
        if (!D.as_float && D.l.side != 2 && D.r.side != 2 && ldec != rdec)
            fail(KRV_UNSUPPORTED, "a residual filter compares a decimal column with an integer column");
        if (ldec && rdec && lt.scale != rt.scale)
            fail(KRV_UNSUPPORTED, "a residual filter compares decimal columns of different scales");
    }
    return F;
}

// Whether the keys are coded: some key column of the first build batch is
// a string or binary column.
void HashJoin::decide(const DevBatch &b) {
    decided_ = true;
    bool var = false;
    for (int k = 0; k < spec_.n_keys; k++) {
        const int c = spec_.build_keys[k];
        if (c < 0 || c >= (int)b.cols.size()) fail(KRV_INVALID_ARGUMENT, "build key column out of range");
        var = var || b.cols[c].type.var();
    }
    if (!var) return;
    if (residual_set_) fail(KRV_UNSUPPORTED, "a residual filter on a join over string or binary keys");
    coded_.reset(new Coded());
    coded_->outer = spec_;
    std::vector<DevCol> meta;
    for (int k = 0; k < spec_.n_keys; k++) {
        const DevCol &c = b.cols[spec_.build_keys[k]];
        DevCol m;
        m.type = c.type;
        m.name = c.name;
        m.nullable = c.nullable || c.valid;
        meta.push_back(m);
    }
    coded_->dict = make_key_dict(rt_, meta);
    // the build side's columns (string key columns stay, as payload), then the code
    const krv_join_spec &o = coded_->outer;
    spec_.n_keys = 1;
    spec_.build_keys[0] = (int32_t)b.cols.size();
    spec_.null_safe[0] = 0;
    spec_.runtime_filter = 0;  // a filter over codes answers nothing outside
    const int nb = o.n_build_out < 0 ? (int)b.cols.size() : o.n_build_out;
    for (int i = 0; i < nb; i++) {
        const int c = o.n_build_out < 0 ? i : o.build_out[i];
        if (c < 0 || c >= (int)b.cols.size()) fail(KRV_INVALID_ARGUMENT, "projection column out of range");
        spec_.build_out[i] = c;
    }
    spec_.n_build_out = nb;
}

__global__ void code_valid_kernel(KeysDev k, int64_t n, uint32_t *bits) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i - (threadIdx.x & 31) < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        bool v = i < n;
        for (int c = 0; c < k.n && v; c++)
            if (!((k.null_safe >> c) & 1u) && !bit_get(k.c[c].valid, k.c[c].voff, i)) v = false;
        const unsigned w = __ballot_sync(0xFFFFFFFFu, v);
        if ((threadIdx.x & 31) == 0) bits[i >> 5] = w;
    }
}

// The batch the table sees: b's columns (string and binary ones included,
// as payload the output can carry), then the key code (NULL where an `=`
// key is NULL: such a row never matches).
DevBatch HashJoin::coded_batch(const DevBatch &b, bool build) {
    const krv_join_spec &o = coded_->outer;
    const int32_t *keys = build ? o.build_keys : o.probe_keys;
    std::vector<int> cols;
    for (int k = 0; k < o.n_keys; k++) {
        if (keys[k] < 0 || keys[k] >= (int)b.cols.size()) fail(KRV_INVALID_ARGUMENT, "key column out of range");
        cols.push_back(keys[k]);
    }
    auto codes = std::make_shared<DBuf>(key_dict_encode(coded_->dict, b, cols, build));
    DevBatch in;
    in.rows = b.rows;
    in.cols = b.cols;
    // validity of the code: every `=` key component valid
    KeysDev kd{};
    kd.n = o.n_keys;
    for (int k = 0; k < o.n_keys; k++) {
        const DevCol &c = b.cols[keys[k]];
        kd.c[k] = KeyColDev{c.data, c.valid, c.valid_off, 8, 0};
        if (o.null_safe[k]) kd.null_safe |= 1u << k;
    }
    auto bits = std::make_shared<DBuf>(rt_, (size_t)ceil_div(std::max<int64_t>(b.rows, 1), 32) * 4 + 8);
    if (b.rows > 0) {
        code_valid_kernel<<<grid_for(rt_, b.rows, 256, 8), 256, 0, rt_->stream>>>(kd, b.rows, bits->as<uint32_t>());
        rt_->launches++;
        check_launch("code_valid_kernel");
    }
    DevCol cc;
    cc.type = DType{Type::I64, 0, 0};
    cc.name = "#key";
    cc.nullable = true;
    cc.length = b.rows;
    cc.hold_data = codes;
    cc.data = codes->get();
    cc.hold_valid = bits;
    cc.valid = bits->as<uint8_t>();
    cc.valid_off = 0;
    in.cols.push_back(cc);
    if (!build && !coded_->probe_mapped) {
        coded_->probe_mapped = true;
        spec_.probe_keys[0] = (int32_t)b.cols.size();
        const int np = o.n_probe_out < 0 ? (int)b.cols.size() : o.n_probe_out;
        for (int i = 0; i < np; i++) {
            const int c = o.n_probe_out < 0 ? i : o.probe_out[i];
            if (c < 0 || c >= (int)b.cols.size()) fail(KRV_INVALID_ARGUMENT, "projection column out of range");
            spec_.probe_out[i] = c;
        }
        spec_.n_probe_out = np;
    }
    return in;
}

void HashJoin::build_push(DevBatch b) {
    if (built_) fail(KRV_INVALID_ARGUMENT, "build_push after build_finish");
    DeviceGuard g(rt_);
    if (!decided_) decide(b);
    if (coded_) b = coded_batch(b, true);
    append_arena(b);
}

DevBatch HashJoin::staged() const {
    DevBatch b;
    b.rows = build_rows_;
    for (size_t i = 0; i < arena_cols_.size(); i++) {
        DevCol c = arena_cols_[i];
        c.length = build_rows_;
        c.hold_data = arena_data_[i];
        c.data = c.hold_data ? c.hold_data->get() : nullptr;
        c.valid = nullptr;
        c.valid_off = 0;
        b.cols.push_back(c);
    }
    return b;
}

HashJoin::TableDev HashJoin::table_dev() const {
    return TableDev{slots_.as<unsigned long long>(), mask_, next_.as<uint32_t>(), spec_.seed};
}

void HashJoin::build_finish() {
    if (built_) fail(KRV_INVALID_ARGUMENT, "build_finish called twice");
    DeviceGuard g(rt_);
    built_ = true;
    arena_.rows = build_rows_;
    arena_.cols.clear();
    for (size_t i = 0; i < arena_cols_.size(); i++) {
        DevCol c = arena_cols_[i];
        c.length = build_rows_;
        c.hold_data = arena_data_[i];
        c.hold_valid = arena_valid_[i];
        c.data = c.hold_data ? c.hold_data->get() : nullptr;
        c.valid = c.hold_valid ? c.hold_valid->as<uint8_t>() : nullptr;
        c.valid_off = 0;
        arena_.cols.push_back(c);
    }
    const uint64_t want = (uint64_t)std::ceil((double)std::max<int64_t>(build_rows_, 1) / spec_.max_load);
    const uint64_t slots = std::max<uint64_t>(1024, next_pow2(want));
    mask_ = slots - 1;
    slots_ = DBuf(rt_, slots * 8);
    zero(rt_, slots_.get(), slots * 8);
    next_ = DBuf(rt_, (size_t)std::max<int64_t>(build_rows_, 1) * 4);
    counters_dev_ = DBuf(rt_, 64);
    {
        // [0] keys, [1] NULL seen, [2] min, [3] max, [4] indexed rows, [6] longest chain
        const unsigned long long init[8] = {0, 0, (unsigned long long)LLONG_MAX, (unsigned long long)LLONG_MIN, 0, 0, 0, 0};
        KRV_CUDA(cudaMemcpyAsync(counters_dev_.get(), init, 64, cudaMemcpyHostToDevice, rt_->stream));
    }
    const int jt = spec_.join_type;
    const bool preserved = jt == KRV_JOIN_RIGHT_SEMI || jt == KRV_JOIN_RIGHT_ANTI || jt == KRV_JOIN_RIGHT_OUTER ||
                           jt == KRV_JOIN_FULL_OUTER;
    if (preserved) {
        marks_ = DBuf(rt_, (size_t)std::max<int64_t>(build_rows_, 1));
        zero(rt_, marks_.get(), marks_.bytes());
    }
    clear_status(rt_);
    if (build_rows_ > 0) {
        if (arena_.cols.empty()) fail(KRV_INVALID_ARGUMENT, "build batches without columns");
        KeysDev k = keys_of(arena_, spec_.build_keys, spec_.n_keys, spec_.null_safe);
        const int threads = 256;
        const int grid = grid_for(rt_, build_rows_, threads, 8);
        auto *ctr = counters_dev_.as<unsigned long long>();
        if (fast_keys(k))
            build_kernel<true><<<grid, threads, 0, rt_->stream>>>(k, build_rows_, slots_.as<unsigned long long>(), mask_,
                                                                 next_.as<uint32_t>(), spec_.seed, ctr, status_word(rt_));
        else
            build_kernel<false><<<grid, threads, 0, rt_->stream>>>(k, build_rows_, slots_.as<unsigned long long>(), mask_,
                                                                  next_.as<uint32_t>(), spec_.seed, ctr, status_word(rt_));
        rt_->launches++;
        check_launch("build_kernel");
    }
    unsigned long long host_ctr[8];
    KRV_CUDA(cudaMemcpyAsync(host_ctr, counters_dev_.get(), 64, cudaMemcpyDeviceToHost, rt_->stream));
    const uint32_t st = take_status(rt_);  // synchronizes: host_ctr is ready too
    if (st & ST_CAPACITY) fail(KRV_INTERNAL, "join table full");
    counters_.build_rows = build_rows_;
    counters_.build_keys = (int64_t)host_ctr[0];
    counters_.table_slots = (int64_t)slots;
    any_null_build_ = host_ctr[1] != 0;
    indexed_rows_ = (int64_t)host_ctr[4];
    key_lo_ = (long long)host_ctr[2];
    key_hi_ = (long long)host_ctr[3];
    // Unique, dense int64 keys (a span of at most 4 values per row): a direct
    // index, 4 bytes per key value, for the probe of inner and left outer joins.
    direct_.reset();
    direct_span_ = 0;
    if (indexed_rows_ > 0 && counters_.build_keys == indexed_rows_ && spec_.n_keys == 1 && !spec_.null_safe[0] &&
        arena_.cols[spec_.build_keys[0]].type.id == Type::I64 &&
        (spec_.join_type == KRV_JOIN_INNER || spec_.join_type == KRV_JOIN_LEFT_OUTER)) {
        const __int128 span = (__int128)key_hi_ - (__int128)key_lo_;
        if (span >= 0 && span < ((__int128)1 << 31) && span < (__int128)4 * indexed_rows_ + 4096) {
            direct_span_ = (unsigned long long)span;
            direct_ = DBuf(rt_, (size_t)(span + 1) * 4);
            KRV_CUDA(cudaMemsetAsync(direct_.get(), 0xFF, direct_.bytes(), rt_->stream));
            KeysDev k = keys_of(arena_, spec_.build_keys, spec_.n_keys, spec_.null_safe);
            direct_build_kernel<<<grid_for(rt_, build_rows_, 256, 8), 256, 0, rt_->stream>>>(
                k, build_rows_, DirectDev{direct_.as<uint32_t>(), key_lo_, direct_span_});
            rt_->launches++;
            check_launch("direct_build_kernel");
        }
    }
    // The runtime filter of a one-key join (BuildSink::publish, join/build.rs:482).
    if (spec_.runtime_filter && spec_.n_keys == 1) {
        const DevCol &key = arena_.cols[spec_.build_keys[0]];
        if (key.type.id == Type::I64) {
            krv_key_filter_options o;
            krv_key_filter_options_default(&o);
            // The build already counted the kept rows, the distinct keys and
            // their range: the filter builder needs no pass of its own unless
            // an exact form may apply.
            KeyStats ks{(int64_t)host_ctr[4], (int64_t)host_ctr[0], (long long)host_ctr[2], (long long)host_ctr[3]};
            filter_ = build_key_filter(rt_, o, key, &ks);
        }
    }
}

static std::vector<int> projection(int n, const int32_t *cols, int ncols) {
    std::vector<int> v;
    if (n < 0) {
        for (int i = 0; i < ncols; i++) v.push_back(i);
    } else {
        for (int i = 0; i < n; i++) {
            if (cols[i] < 0 || cols[i] >= ncols) fail(KRV_INVALID_ARGUMENT, "projection column out of range");
            v.push_back(cols[i]);
        }
    }
    return v;
}

DevBatch HashJoin::probe(const DevBatch &outer_in) {
    if (!built_) fail(KRV_INVALID_ARGUMENT, "probe before build_finish");
    DeviceGuard g(rt_);
    DevBatch coded_in;
    if (coded_) coded_in = coded_batch(outer_in, false);
    const DevBatch &in = coded_ ? coded_in : outer_in;
    const int jt = spec_.join_type;
    const int64_t n = in.rows;
    counters_.probe_rows += n;
    if (probe_types_.empty()) {
        for (const DevCol &c : in.cols) {
            probe_types_.push_back(c.type);
            probe_names_.push_back(c.name);
            probe_nullable_.push_back(c.nullable);
        }
    }
    KeysDev pk = keys_of(in, spec_.probe_keys, spec_.n_keys, spec_.null_safe);
    KeysDev bk{};
    if (build_rows_ > 0) bk = keys_of(arena_, spec_.build_keys, spec_.n_keys, spec_.null_safe);
    else bk = pk;  // never dereferenced: the table is empty
    for (int c = 0; c < spec_.n_keys; c++) {
        const DevCol &pc = in.cols[spec_.probe_keys[c]];
        if (build_rows_ > 0 && pc.type != arena_.cols[spec_.build_keys[c]].type)
            fail(KRV_INVALID_ARGUMENT, "probe and build key types differ");
    }
    const bool fast = fast_keys(pk);
    if (spec_.has_residual_filter && !residual_set_)
        fail(KRV_INVALID_ARGUMENT, "has_residual_filter is set but no filter was given (krv_join_set_filter)");
    const bool filt = residual_set_;
    const FilterDev fd = filt ? filter_dev(in) : FilterDev{};
    auto launch_pairs = [&](bool fast_, bool filt_, int grid_, int threads_, const KeysDev &pk_, const KeysDev &bk_,
                            int64_t n_, const OutDev &od_, unsigned long long cap_, unsigned long long *count_,
                            uint8_t *marks_p, int pad_, int single_, unsigned long long *mc_, const FilterDev &fd_) {
        const auto *sl = slots_.as<unsigned long long>();
        const uint32_t *nx = next_.as<uint32_t>();
        uint32_t *st = status_word(rt_);
        if (fast_ && filt_)
            probe_pairs_kernel<true, true><<<grid_, threads_, 0, rt_->stream>>>(
                pk_, bk_, n_, sl, mask_, nx, spec_.seed, od_, cap_, count_, marks_p, pad_, single_, st, mc_, fd_);
        else if (fast_)
            probe_pairs_kernel<true, false><<<grid_, threads_, 0, rt_->stream>>>(
                pk_, bk_, n_, sl, mask_, nx, spec_.seed, od_, cap_, count_, marks_p, pad_, single_, st, mc_, fd_);
        else if (filt_)
            probe_pairs_kernel<false, true><<<grid_, threads_, 0, rt_->stream>>>(
                pk_, bk_, n_, sl, mask_, nx, spec_.seed, od_, cap_, count_, marks_p, pad_, single_, st, mc_, fd_);
        else
            probe_pairs_kernel<false, false><<<grid_, threads_, 0, rt_->stream>>>(
                pk_, bk_, n_, sl, mask_, nx, spec_.seed, od_, cap_, count_, marks_p, pad_, single_, st, mc_, fd_);
    };
    const auto pcols = projection(spec_.n_probe_out, spec_.probe_out, (int)in.cols.size());
    const auto bcols = projection(spec_.n_build_out, spec_.build_out, (int)arena_cols_.size());
    const int threads = 256;
    const int grid = grid_for(rt_, n, threads, 8);
    const auto *slots = slots_.as<unsigned long long>();
    DevBatch out;

    if (jt == KRV_JOIN_EXISTENCE) {
        out.rows = n;
        for (int pc : pcols) {
            const DevCol &s = in.cols[pc];
            if (s.type.var()) {
                out.cols.push_back(var_gather(rt_, var_src(0, pc, &in), nullptr, n, s.type, s.nullable || s.valid, s.name));
                continue;
            }
            DevCol d = make_col(rt_, s.type, n, s.nullable || s.valid, s.name);
            const size_t bytes = s.type.id == Type::Bool ? (size_t)ceil_div(n, 8) : (size_t)n * s.type.width();
            if (bytes) KRV_CUDA(cudaMemcpyAsync(const_cast<void *>(d.data), s.data, bytes, cudaMemcpyDeviceToDevice, rt_->stream));
            if (d.valid) {
                zero(rt_, const_cast<uint8_t *>(d.valid), d.hold_valid->bytes());
                append_bits(rt_, s.valid, s.valid_off, n, const_cast<uint8_t *>(d.valid), 0);
            }
            out.cols.push_back(d);
        }
        DevCol ex = make_col(rt_, DType{Type::Bool, 0, 0}, n, false, "exists");
        zero(rt_, const_cast<void *>(ex.data), ex.hold_data->bytes());
        if (n > 0) {
            const uint32_t *nx = next_.as<uint32_t>();
            uint32_t *exw = (uint32_t *)ex.data;
            const int empty = build_rows_ == 0;
            if (fast && filt)
                probe_exists_kernel<true, true><<<grid, threads, 0, rt_->stream>>>(pk, bk, n, slots, mask_, spec_.seed,
                                                                                   exw, empty, nx, fd);
            else if (fast)
                probe_exists_kernel<true, false><<<grid, threads, 0, rt_->stream>>>(pk, bk, n, slots, mask_, spec_.seed,
                                                                                    exw, empty, nx, fd);
            else if (filt)
                probe_exists_kernel<false, true><<<grid, threads, 0, rt_->stream>>>(pk, bk, n, slots, mask_, spec_.seed,
                                                                                    exw, empty, nx, fd);
            else
                probe_exists_kernel<false, false><<<grid, threads, 0, rt_->stream>>>(pk, bk, n, slots, mask_,
                                                                                     spec_.seed, exw, empty, nx, fd);
            rt_->launches++;
            check_launch("probe_exists_kernel");
        }
        out.cols.push_back(ex);
        counters_.output_rows += n;
        remember_shape(out);
        return out;
    }

    const bool pairs = jt == KRV_JOIN_INNER || jt == KRV_JOIN_LEFT_OUTER || jt == KRV_JOIN_RIGHT_OUTER ||
                       jt == KRV_JOIN_FULL_OUTER;
    if (!pairs && (jt == KRV_JOIN_RIGHT_SEMI || jt == KRV_JOIN_RIGHT_ANTI)) {
        // Probe only marks build rows; output comes at finish.
        if (n > 0 && build_rows_ > 0) {
            OutDev od{};
            od.n = 0;
            DBuf cnt(rt_, 8);
            zero(rt_, cnt.get(), 8);
            auto *mc = counters_dev_.as<unsigned long long>() + 6;
            launch_pairs(fast, filt, grid, threads, pk, bk, n, od, 0, cnt.as<unsigned long long>(), marks_.as<uint8_t>(), 0,
                         0, mc, fd);
            rt_->launches++;
            check_launch("probe_pairs_kernel");
        }
        // Nothing is emitted by this batch: an empty batch of the output shape.
        DevBatch empty;
        for (int bc : bcols) empty.cols.push_back(empty_col(arena_cols_[bc]));
        return empty;
    }

    const bool build_nullable = jt == KRV_JOIN_LEFT_OUTER || jt == KRV_JOIN_FULL_OUTER;
    const bool probe_nullable = jt == KRV_JOIN_RIGHT_OUTER || jt == KRV_JOIN_FULL_OUTER;
    // The output's size is known only after the kernel. Unique build keys
    // give at most one row per probe row; otherwise there is room for the
    // rows that the earlier batches' output ratio predicts (before any, the
    // build's mean rows per key), 5% more, and a batch with more output runs
    // again with room for all of it.
    unsigned long long cap = (unsigned long long)std::max<int64_t>(n, 1);
    const bool unique_keys = build_rows_ > 0 && counters_.build_keys == indexed_rows_;
    if (pairs && !unique_keys && n > 0) {
        const int64_t seen = counters_.probe_rows - n;
        double ratio = seen > 0 ? (double)counters_.output_rows / (double)seen
                       : counters_.build_keys > 0 ? (double)indexed_rows_ / (double)counters_.build_keys : 1.0;
        if (jt == KRV_JOIN_LEFT_OUTER || jt == KRV_JOIN_FULL_OUTER) ratio = std::max(ratio, 1.0);
        cap = std::max<unsigned long long>(1, (unsigned long long)((double)n * ratio * 1.05) + 1024);
    }
    DBuf cnt(rt_, 8);
    for (int attempt = 0; attempt < 4; attempt++) {
        out = DevBatch{};
        OutDev od{};
        std::vector<VarOut> vars;  // string columns, gathered once the row indexes are known
        for (int pc : pcols) {
            const DevCol &s = in.cols[pc];
            if (s.type.id == Type::Bool) fail(KRV_UNSUPPORTED, "boolean probe payload columns");
            const bool nullable = s.nullable || s.valid || probe_nullable;
            if (s.type.var()) {
                DevCol m;
                m.type = s.type;
                m.name = s.name;
                m.nullable = nullable;
                vars.push_back(VarOut{(int)out.cols.size(), 0, pc});
                out.cols.push_back(m);
                continue;
            }
            DevCol d = make_col(rt_, s.type, (int64_t)cap, nullable, s.name);
            if (d.valid) zero(rt_, const_cast<uint8_t *>(d.valid), d.hold_valid->bytes());
            od.c[od.n++] = OutColDev{s.data, s.valid, s.valid_off, const_cast<void *>(d.data),
                                     (uint32_t *)d.valid, s.type.width(), 0};
            out.cols.push_back(d);
        }
        if (pairs) {
            for (int bc : bcols) {
                const DevCol &s = arena_.cols.empty() ? DevCol{} : arena_.cols[bc];
                const DevCol &meta = arena_cols_[bc];
                const bool nullable = meta.nullable || build_nullable;
                if (meta.type.var()) {
                    DevCol m;
                    m.type = meta.type;
                    m.name = meta.name;
                    m.nullable = nullable;
                    vars.push_back(VarOut{(int)out.cols.size(), 1, bc});
                    out.cols.push_back(m);
                    continue;
                }
                DevCol d = make_col(rt_, meta.type, (int64_t)cap, nullable, meta.name);
                if (d.valid) zero(rt_, const_cast<uint8_t *>(d.valid), d.hold_valid->bytes());
                od.c[od.n++] = OutColDev{s.data, meta.nullable ? s.valid : nullptr, 0, const_cast<void *>(d.data),
                                         (uint32_t *)d.valid, meta.type.width(), 1};
                out.cols.push_back(d);
            }
        }
        DBuf idx[2];
        for (const VarOut &v : vars)
            if (!idx[v.side].get()) {
                idx[v.side] = DBuf(rt_, (size_t)cap * 8);
                od.c[od.n++] = OutColDev{nullptr, nullptr, 0, idx[v.side].get(), nullptr, 8, 3 + v.side};
            }
        zero(rt_, cnt.get(), 8);
        clear_status(rt_);
        if (n > 0) {
            auto *count = cnt.as<unsigned long long>();
            if (pairs) {
                if (build_rows_ > 0 || jt == KRV_JOIN_LEFT_OUTER || jt == KRV_JOIN_FULL_OUTER) {
                    // An empty build still has an all-empty table: every lookup misses.
                    auto *mc = counters_dev_.as<unsigned long long>() + 6;
                    uint8_t *marks = marks_.get() ? marks_.as<uint8_t>() : nullptr;
                    const int pad = jt == KRV_JOIN_LEFT_OUTER || jt == KRV_JOIN_FULL_OUTER;
                    // unique build keys: at most one output row per probe row
                    const bool unique = build_rows_ > 0 && counters_.build_keys == indexed_rows_;
                    if (fast && unique && !marks && pk.null_safe == 0 && !filt &&
                        (jt == KRV_JOIN_INNER || jt == KRV_JOIN_LEFT_OUTER)) {
                        const int fgrid = grid_for(rt_, ceil_div(n, kFastRows), kFastThreads, 8);
                        const DirectDev dd{direct_.as<uint32_t>(), key_lo_, direct_span_};
                        if (dd.row)
                            probe_fast_kernel<true><<<fgrid, kFastThreads, 0, rt_->stream>>>(
                                pk, bk, n, slots, mask_, spec_.seed, dd, od, cap, count, pad);
                        else
                            probe_fast_kernel<false><<<fgrid, kFastThreads, 0, rt_->stream>>>(
                                pk, bk, n, slots, mask_, spec_.seed, dd, od, cap, count, pad);
                    } else {
                        launch_pairs(fast, filt, grid, threads, pk, bk, n, od, cap, count, marks, pad,
                                     spec_.single_match, mc, fd);
                    }
                    rt_->launches++;
                    check_launch("probe_pairs_kernel");
                }
            } else {
                const int kind = jt == KRV_JOIN_LEFT_SEMI ? 0 : jt == KRV_JOIN_LEFT_ANTI ? 1 : 2;
                const unsigned long long *sl = slots;
                const uint64_t mask = mask_;
                const uint32_t *nx = next_.as<uint32_t>();
                const int empty = build_rows_ == 0, hn = any_null_build_;
                if (fast && filt)
                    probe_rows_kernel<true, true><<<grid, threads, 0, rt_->stream>>>(
                        pk, bk, n, sl, mask, spec_.seed, od, cap, count, kind, empty, hn, nx, fd);
                else if (fast)
                    probe_rows_kernel<true, false><<<grid, threads, 0, rt_->stream>>>(
                        pk, bk, n, sl, mask, spec_.seed, od, cap, count, kind, empty, hn, nx, fd);
                else if (filt)
                    probe_rows_kernel<false, true><<<grid, threads, 0, rt_->stream>>>(
                        pk, bk, n, sl, mask, spec_.seed, od, cap, count, kind, empty, hn, nx, fd);
                else
                    probe_rows_kernel<false, false><<<grid, threads, 0, rt_->stream>>>(
                        pk, bk, n, sl, mask, spec_.seed, od, cap, count, kind, empty, hn, nx, fd);
                rt_->launches++;
                check_launch("probe_rows_kernel");
            }
        }
        const unsigned long long got = read_scalar<unsigned long long>(rt_, cnt.get());
        const uint32_t st = take_status(rt_);
        if (st & ST_TOO_MANY) fail(KRV_TOO_MANY_ROWS, "SCALAR_SUBQUERY_TOO_MANY_ROWS: a probe row matched more than one build row");
        if (got <= cap) {
            out.rows = (int64_t)got;
            for (DevCol &c : out.cols) c.length = out.rows;
            for (const VarOut &v : vars) {
                const DevCol m = out.cols[v.pos];
                out.cols[v.pos] = var_gather(rt_, var_src(v.side, v.col, &in), idx[v.side].as<long long>(), out.rows,
                                             m.type, m.nullable, m.name);
            }
            counters_.output_rows += out.rows;
            remember_shape(out);
            return out;
        }
        cap = got;  // output larger than guessed: run again with room for all of it
    }
    fail(KRV_INTERNAL, "join output did not converge");
}

DevBatch HashJoin::finish() {
    if (!built_) fail(KRV_INVALID_ARGUMENT, "finish before build_finish");
    DeviceGuard g(rt_);
    const int jt = spec_.join_type;
    const bool tail = jt == KRV_JOIN_RIGHT_SEMI || jt == KRV_JOIN_RIGHT_ANTI || jt == KRV_JOIN_RIGHT_OUTER ||
                      jt == KRV_JOIN_FULL_OUTER;
    if (!tail || finished_) {
        // Nothing waits for the end: an empty batch of the probe output's shape.
        finished_ = true;
        DevBatch empty;
        for (const DevCol &m : out_meta_) empty.cols.push_back(empty_col(m));
        return empty;
    }
    finished_ = true;
    const bool with_probe = jt == KRV_JOIN_RIGHT_OUTER || jt == KRV_JOIN_FULL_OUTER;
    if (with_probe && probe_types_.empty())
        fail(KRV_INVALID_ARGUMENT, "an outer join's tail needs the probe schema: probe at least one batch");
    const auto bcols = projection(spec_.n_build_out, spec_.build_out, (int)arena_cols_.size());
    std::vector<int> pcols;
    if (with_probe) pcols = projection(spec_.n_probe_out, spec_.probe_out, (int)probe_types_.size());
    const unsigned long long cap = (unsigned long long)std::max<int64_t>(build_rows_, 1);
    DevBatch out;
    OutDev od{};
    std::vector<VarOut> vars;
    for (int pc : pcols) {
        if (probe_types_[pc].var()) {
            DevCol m;
            m.type = probe_types_[pc];
            m.name = probe_names_[pc];
            m.nullable = true;
            vars.push_back(VarOut{(int)out.cols.size(), 0, pc});
            out.cols.push_back(m);
            continue;
        }
        DevCol d = make_col(rt_, probe_types_[pc], (int64_t)cap, true, probe_names_[pc]);
        zero(rt_, const_cast<uint8_t *>(d.valid), d.hold_valid->bytes());
        od.c[od.n++] = OutColDev{nullptr, nullptr, 0, const_cast<void *>(d.data), (uint32_t *)d.valid,
                                 probe_types_[pc].width(), 2};
        out.cols.push_back(d);
    }
    for (int bc : bcols) {
        const DevCol &meta = arena_cols_[bc];
        const DevCol &s = arena_.cols[bc];
        const bool nullable = meta.nullable || jt == KRV_JOIN_FULL_OUTER;
        if (meta.type.var()) {
            DevCol m;
            m.type = meta.type;
            m.name = meta.name;
            m.nullable = nullable;
            vars.push_back(VarOut{(int)out.cols.size(), 1, bc});
            out.cols.push_back(m);
            continue;
        }
        DevCol d = make_col(rt_, meta.type, (int64_t)cap, nullable, meta.name);
        if (d.valid) zero(rt_, const_cast<uint8_t *>(d.valid), d.hold_valid->bytes());
        od.c[od.n++] = OutColDev{s.data, meta.nullable ? s.valid : nullptr, 0, const_cast<void *>(d.data),
                                 (uint32_t *)d.valid, meta.type.width(), 1};
        out.cols.push_back(d);
    }
    DBuf idx[2];
    for (const VarOut &v : vars)
        if (!idx[v.side].get()) {
            idx[v.side] = DBuf(rt_, (size_t)cap * 8);
            od.c[od.n++] = OutColDev{nullptr, nullptr, 0, idx[v.side].get(), nullptr, 8, 3 + v.side};
        }
    DBuf cnt(rt_, 8);
    zero(rt_, cnt.get(), 8);
    if (build_rows_ > 0) {
        KeysDev bk = keys_of(arena_, spec_.build_keys, spec_.n_keys, spec_.null_safe);
        const int threads = 256;
        tail_kernel<<<grid_for(rt_, build_rows_, threads, 8), threads, 0, rt_->stream>>>(
            build_rows_, marks_.as<uint8_t>(), bk, jt == KRV_JOIN_RIGHT_SEMI ? 0 : 1, od, cap,
            cnt.as<unsigned long long>());
        rt_->launches++;
        check_launch("tail_kernel");
    }
    out.rows = (int64_t)read_scalar<unsigned long long>(rt_, cnt.get());
    for (DevCol &c : out.cols) c.length = out.rows;
    for (const VarOut &v : vars) {
        const DevCol m = out.cols[v.pos];
        // the tail's probe side is all NULL: its string columns read nothing
        const VarSrc src = v.side == 1 ? var_src(1, v.col, nullptr) : VarSrc{};
        out.cols[v.pos] = var_gather(rt_, src, idx[v.side].as<long long>(), out.rows, m.type, m.nullable, m.name);
    }
    counters_.output_rows += out.rows;
    return out;
}

}  // namespace krv
