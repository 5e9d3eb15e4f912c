// gen.cu -- counter-based synthetic column generators for the benchmarks.
// value(seed, column, row) is a pure function, so any row range can be
// generated on any device in any order, and the CPU test oracle computes the
// same values.
#include <cmath>
#include <vector>

#include "krv_device.cuh"
#include "ops.h"

namespace krv {

namespace {

__host__ __device__ __forceinline__ uint64_t fmix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
// The SplitMix64 output at step row + 1 of the stream started by (seed, column).
__host__ __device__ __forceinline__ uint64_t rnd(uint64_t seed, uint32_t column, uint64_t row) {
    const uint64_t base = fmix64(seed ^ fmix64((uint64_t)column + 0x632BE59BD9B4E019ULL));
    return fmix64(base + (row + 1) * 0x9E3779B97F4A7C15ULL);
}
__device__ __forceinline__ uint64_t mulhi(uint64_t a, uint64_t b) { return __umul64hi(a, b); }
__device__ __forceinline__ double unit(uint64_t x) { return (double)(x >> 11) * 0x1.0p-53; }

// A permutation of [0, n): 4-round Feistel over 2^bits >= n (bits even),
// cycle-walking until the value falls below n.
__device__ __forceinline__ uint64_t permute(uint64_t seed, uint64_t n, uint64_t i) {
    int bits = 2;
    while ((1ULL << bits) < n) bits += 2;
    const int half = bits / 2;
    const uint64_t hmask = (1ULL << half) - 1;
    uint64_t x = i;
    for (int walk = 0; walk < 4096; walk++) {
        uint64_t l = x >> half, r = x & hmask;
        for (uint32_t round = 0; round < 4; round++) {
            const uint64_t f = rnd(seed, 0x70000000u + round, r) & hmask;
            const uint64_t nl = r;
            r = l ^ f;
            l = nl;
        }
        x = (l << half) | r;
        if (x < n) return x;
    }
    return i % n;  // unreachable for a 4-round Feistel (cycles are short)
}

__global__ void gen_kernel(krv_gen_spec s, int64_t n, void *out, uint32_t *valid, const double *cdf, int64_t cdf_n) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t base = blockIdx.x * (int64_t)blockDim.x; base < n; base += stride) {
        const int64_t i = base + threadIdx.x;
        bool v = true;
        if (i < n) {
            const uint64_t row = (uint64_t)(s.row0 + i);
            const uint64_t x = rnd(s.seed, s.column, row);
            switch (s.kind) {
            case KRV_GEN_UNIFORM_I64: {
                const uint64_t span = (uint64_t)(s.hi - s.lo) + 1;
                static_cast<int64_t *>(out)[i] = s.lo + (int64_t)mulhi(x, span);
                break;
            }
            case KRV_GEN_UNIFORM_I32: {
                const uint64_t span = (uint64_t)(s.hi - s.lo) + 1;
                static_cast<int32_t *>(out)[i] = (int32_t)(s.lo + (int64_t)mulhi(x, span));
                break;
            }
            case KRV_GEN_UNIT_F64:
                static_cast<double *>(out)[i] = __dadd_rn(s.x0, __dmul_rn(__dsub_rn(s.x1, s.x0), unit(x)));
                break;
            case KRV_GEN_PERMUTATION:
                static_cast<int64_t *>(out)[i] = s.lo + (int64_t)permute(s.seed, (uint64_t)s.hi, row);
                break;
            case KRV_GEN_ZIPF: {
                const double u = unit(x);
                int64_t lo = 0, hi = cdf_n - 1;
                while (lo < hi) {
                    const int64_t mid = lo + (hi - lo) / 2;
                    if (cdf[mid] > u) hi = mid;
                    else lo = mid + 1;
                }
                static_cast<int64_t *>(out)[i] = s.lo + (int64_t)permute(s.seed ^ 0x5A17F00DULL, (uint64_t)cdf_n, (uint64_t)lo);
                break;
            }
            default: break;
            }
            if (valid) v = unit(rnd(s.seed, s.column + 0x10000u, row)) >= s.null_fraction;
        }
        if (valid) {
            const unsigned w = __ballot_sync(0xFFFFFFFFu, v);
            if ((threadIdx.x & 31) == 0 && i < n) valid[i >> 5] = w;
        }
    }
}

}  // namespace

void gen_fill(Runtime *rt, const krv_gen_spec &s, int64_t n, void *out, void *out_valid) {
    if (n < 0) fail(KRV_INVALID_ARGUMENT, "negative row count");
    if (n == 0) return;
    if (s.kind < KRV_GEN_UNIFORM_I64 || s.kind > KRV_GEN_ZIPF) fail(KRV_INVALID_ARGUMENT, "unknown generator");
    if ((s.kind == KRV_GEN_UNIFORM_I64 || s.kind == KRV_GEN_UNIFORM_I32) && s.hi < s.lo)
        fail(KRV_INVALID_ARGUMENT, "empty integer range");
    if ((s.kind == KRV_GEN_PERMUTATION || s.kind == KRV_GEN_ZIPF) && s.hi <= 0)
        fail(KRV_INVALID_ARGUMENT, "a permutation or Zipf domain needs hi > 0");
    DeviceGuard g(rt);
    DBuf cdf;
    int64_t cdf_n = 0;
    if (s.kind == KRV_GEN_ZIPF) {
        // Zipf(s) cumulative table over ranks 1..N: plain IEEE double sums, in
        // rank order, normalized by the total (the CPU oracle computes the same).
        cdf_n = s.hi;
        std::vector<double> h((size_t)cdf_n);
        double acc = 0.0;
        for (int64_t k = 1; k <= cdf_n; k++) {
            acc += std::pow((double)k, -s.x0);
            h[(size_t)(k - 1)] = acc;
        }
        for (int64_t k = 0; k < cdf_n; k++) h[(size_t)k] /= acc;
        h[(size_t)(cdf_n - 1)] = 1.0;
        cdf = DBuf(rt, (size_t)cdf_n * 8);
        KRV_CUDA(cudaMemcpyAsync(cdf.get(), h.data(), (size_t)cdf_n * 8, cudaMemcpyHostToDevice, rt->stream));
        KRV_CUDA(cudaStreamSynchronize(rt->stream));
    }
    uint32_t *valid = (s.null_fraction > 0 && out_valid) ? static_cast<uint32_t *>(out_valid) : nullptr;
    gen_kernel<<<grid_for(rt, n, 256, 16), 256, 0, rt->stream>>>(s, n, out, valid, cdf.as<double>(), cdf_n);
    rt->launches++;
    check_launch("gen_kernel");
    if (cdf.get()) KRV_CUDA(cudaStreamSynchronize(rt->stream));
}

}  // namespace krv
