// krv_device.cuh -- device-side building blocks: the engine's key hashes,
// XXH64 of fixed-width keys, the split-block Bloom mask, validity bitmaps,
// 128-bit and compensated atomics, and warp-aggregated output allocation.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace krv {

// ---- the row layout's key hash (crates/krishiv-exec/src/rows/layout.rs) ----
// Constants of rows/layout.rs:43-50 (fractional digits of pi, e, sqrt(2));
// a hash must use them to agree with the engine's tables and sketches.
constexpr uint64_t kNullHash = 0xA5A55A5AC3C33C3CULL;
constexpr uint64_t kMix = 0x243F6A8885A308D3ULL;
constexpr uint64_t kFinish = 0xB7E151628AED2A6BULL;
constexpr uint64_t kFin = 0x6A09E667F3BCC909ULL;

// The folded multiply: low ^ high half of the 128-bit product
// (rows/layout.rs:1131-1139).
__host__ __device__ __forceinline__ uint64_t fold(uint64_t a, uint64_t b) {
#ifdef __CUDA_ARCH__
    return (a * b) ^ __umul64hi(a, b);
#else
    unsigned __int128 p = (unsigned __int128)a * b;
    return (uint64_t)p ^ (uint64_t)(p >> 64);
#endif
}
__host__ __device__ __forceinline__ uint64_t mix(uint64_t h, uint64_t v) { return fold(h ^ v, kMix); }
// h of one valid 8-byte key word: fold(0, MIX) = 0, one mix, the finish fold.
__host__ __device__ __forceinline__ uint64_t hash_word(uint64_t w) {
    return fold(fold(w, kMix), kFinish);
}
// g = fin(h ^ seed) (rows/layout.rs:1080-1082)
__host__ __device__ __forceinline__ uint64_t finalize(uint64_t h, uint64_t seed) {
    return fold(h ^ seed, kFin);
}
// Spark key normalization of a float64's bits (rows/layout.rs:1147-1149).
__host__ __device__ __forceinline__ uint64_t normalize_f64_bits(uint64_t bits) {
    const uint64_t exp = bits & 0x7FF0000000000000ULL, man = bits & 0x000FFFFFFFFFFFFFULL;
    if (exp == 0x7FF0000000000000ULL && man != 0) return 0x7FF8000000000000ULL;  // one NaN
    if (bits == 0x8000000000000000ULL) return 0;                                 // -0.0
    return bits;
}

// ---- XXH64 (seed 0) of fixed-width little-endian values --------------------
// The public XXH64 algorithm's short-input path for 8 bytes, as the engine's
// runtime filters hash int64 keys (crates/krishiv-kernels/src/hash/
// routing.rs:112-142, crates/krishiv-io/src/runtime_filter/hash.rs:56-65).
constexpr uint64_t kP1 = 0x9E3779B185EBCA87ULL;
constexpr uint64_t kP2 = 0xC2B2AE3D27D4EB4FULL;
constexpr uint64_t kP3 = 0x165667B19E3779F9ULL;
constexpr uint64_t kP4 = 0x85EBCA77C2B2AE63ULL;
constexpr uint64_t kP5 = 0x27D4EB2F165667C5ULL;
__host__ __device__ __forceinline__ uint64_t rotl64(uint64_t x, int r) {
    return (x << r) | (x >> (64 - r));
}
__host__ __device__ __forceinline__ uint64_t xxh64_u64(uint64_t k) {
    uint64_t h = kP5 + 8;
    uint64_t k1 = rotl64(k * kP2, 31) * kP1;
    h = rotl64(h ^ k1, 27) * kP1 + kP4;
    h ^= h >> 33;
    h *= kP2;
    h ^= h >> 29;
    h *= kP3;
    return h ^ (h >> 32);
}

// ---- split-block Bloom filter (crates/krishiv-io/src/runtime_filter/bloom.rs)
// The Parquet SBBF salts (bloom.rs:15-24; fixed by the Parquet format).
__host__ __device__ __forceinline__ uint32_t sbbf_salt(int i) {
    const uint32_t s[8] = {0x47b6137bu, 0x44974d91u, 0x8824ad5bu, 0xa2b7289du,
                           0x705495c7u, 0x2df1424bu, 0x9efc4947u, 0x5c6bfb31u};
    return s[i];
}
// block = (upper 32 bits of the hash * blocks) >> 32 (bloom.rs:129-132)
__host__ __device__ __forceinline__ uint64_t sbbf_block(uint64_t hash, uint64_t nblocks) {
#ifdef __CUDA_ARCH__
    return __umul64hi((hash >> 32) << 32, nblocks);
#else
    return (uint64_t)(((unsigned __int128)(hash >> 32) * nblocks) >> 32);
#endif
}
__host__ __device__ __forceinline__ uint32_t sbbf_bit(uint32_t key, int i) {
    return 1u << ((key * sbbf_salt(i)) >> 27);
}
// All eight bits of the hash set in the block at `blk` (8 words).
__device__ __forceinline__ bool sbbf_check_words(const uint32_t *blk, uint32_t key) {
    const uint4 a = *reinterpret_cast<const uint4 *>(blk);
    const uint4 b = *reinterpret_cast<const uint4 *>(blk + 4);
    uint32_t miss = (sbbf_bit(key, 0) & ~a.x) | (sbbf_bit(key, 1) & ~a.y) |
                    (sbbf_bit(key, 2) & ~a.z) | (sbbf_bit(key, 3) & ~a.w) |
                    (sbbf_bit(key, 4) & ~b.x) | (sbbf_bit(key, 5) & ~b.y) |
                    (sbbf_bit(key, 6) & ~b.z) | (sbbf_bit(key, 7) & ~b.w);
    return miss == 0;
}

// ---- validity bitmaps ----------------------------------------------------------
__device__ __forceinline__ bool bit_get(const uint8_t *bm, int64_t off, int64_t i) {
    if (!bm) return true;
    const int64_t b = off + i;
    return (bm[b >> 3] >> (b & 7)) & 1;
}

// ---- warp helpers ----------------------------------------------------------------
__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}
// Warp-aggregated allocation: every active lane with `want` reserves one slot
// of `*counter`; returns this lane's position (only meaningful if `want`).
// One atomic per warp (the warp-aggregated atomic compaction pattern).
__device__ __forceinline__ unsigned long long warp_alloc(unsigned long long *counter, bool want,
                                                         unsigned active) {
    const unsigned ballot = __ballot_sync(active, want);
    const int leader = __ffs(active) - 1;
    unsigned long long base = 0;
    if ((int)lane_id() == leader && ballot) base = atomicAdd(counter, (unsigned long long)__popc(ballot));
    base = __shfl_sync(active, base, leader);
    return base + __popc(ballot & lanemask_lt());
}

// ---- 128-bit integer accumulation with two 64-bit atomics ---------------------
// The 128-bit sum is exact once every addition finished: the low word wraps
// with its carry added to the high word by the same adder.
__device__ __forceinline__ void atomic_add_i128(unsigned long long *lo, long long *hi, int64_t vlo,
                                                int64_t vhi) {
    const unsigned long long old = atomicAdd(lo, (unsigned long long)vlo);
    const unsigned long long carry = (old + (unsigned long long)vlo) < old ? 1ull : 0ull;
    const long long add_hi = vhi + (long long)carry;
    if (add_hi) atomicAdd(reinterpret_cast<unsigned long long *>(hi), (unsigned long long)add_hi);
}
__device__ __forceinline__ void atomic_add_i128_from_i64(unsigned long long *lo, long long *hi,
                                                         int64_t v) {
    atomic_add_i128(lo, hi, v, v < 0 ? -1 : 0);
}

// ---- compensated float64 accumulation --------------------------------------------
// A double-double accumulator (hi, lo): atomicAdd on hi returns the value it
// added to, so TwoSum gives the exact rounding error of that addition, which
// goes to lo. hi + lo then equals the exact sum up to the rounding of the lo
// additions (relative error about n * eps^2), whatever the order.
__device__ __forceinline__ void two_sum(double a, double b, double &s, double &e) {
    s = __dadd_rn(a, b);
    const double bb = __dsub_rn(s, a);
    e = __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb));
}
__device__ __forceinline__ void atomic_add_dd(double *hi, double *lo, double v) {
    const double old = atomicAdd(hi, v);
    double s, e;
    two_sum(old, v, s, e);
    if (e != 0.0) atomicAdd(lo, e);
}
// Adds a double-double value (vh, vl).
__device__ __forceinline__ void atomic_add_dd2(double *hi, double *lo, double vh, double vl) {
    const double old = atomicAdd(hi, vh);
    double s, e;
    two_sum(old, vh, s, e);
    const double r = __dadd_rn(e, vl);
    if (r != 0.0) atomicAdd(lo, r);
}

// ---- order-preserving float keys for atomic MIN/MAX --------------------------------
// Spark orders doubles with NaN largest (aggregate/accumulator/helpers.rs:498);
// -0.0 is taken as 0.0. The map is monotone, so unsigned min/max of the keys
// is the float min/max.
__device__ __forceinline__ uint64_t f64_order_key(double d) {
    uint64_t b = normalize_f64_bits((uint64_t)__double_as_longlong(d));
    return (b & 0x8000000000000000ULL) ? ~b : (b | 0x8000000000000000ULL);
}
__host__ __device__ __forceinline__ double f64_from_order_key(uint64_t k) {
    const uint64_t b = (k & 0x8000000000000000ULL) ? (k & 0x7FFFFFFFFFFFFFFFULL) : ~k;
    double d;
    memcpy(&d, &b, 8);
    return d;
}

}  // namespace krv
