// bloom.cu -- the runtime key filter: min/max range, exact set of a few keys,
// or a split-block Bloom filter over XXH64(seed 0) of the key bytes, built on
// the device and evaluated over probe-side columns.
//
// Reference: crates/krishiv-io/src/runtime_filter/ (KeyFilterBuilder,
// filter.rs:157-593; KeyFilter::evaluate_keys, filter.rs:776-798; member
// evaluation, member.rs:423-560; RuntimeBloom, bloom.rs:70-247). The form
// choice and the Bloom's size follow the reference exactly, so a filter built
// here passes exactly the rows the reference's filter passes.
#include <cmath>

#include "krv_device.cuh"
#include "krv_filter.cuh"
#include "ops.h"

extern "C" void krv_key_filter_options_default(krv_key_filter_options *o) {
    // KeyFilterOptions::default (filter.rs:89-104); EXACT_SET_MAX (member.rs:38).
    o->max_values = 50;
    o->exact_max_values = 4096;
    o->bloom = 1;
    o->pad0 = 0;
    o->bloom_max_items = 4000000;
    o->bloom_max_bytes = 8ll << 20;
    o->bloom_fpp = 0.01;
    o->bloom_max_fpp = 0.05;
    o->bloom_bytes = 0;
}

namespace krv {

namespace {

constexpr int64_t kEmptyKey = (int64_t)0x8000000000000000ULL;
constexpr int kBlockBytes = 32;

// RuntimeBloom::bytes_for (bloom.rs:96-110): Parquet's sizing.
int64_t bloom_bytes_for(uint64_t items, double fpp) {
    fpp = std::fmin(std::fmax(fpp, 1e-9), 0.5);
    const double bits = -8.0 * (double)items / std::log(1.0 - std::pow(fpp, 1.0 / 8.0));
    const int64_t bytes = (int64_t)std::ceil(bits / 8.0);
    int64_t blocks = (bytes + kBlockBytes - 1) / kBlockBytes;
    if (blocks < 1) blocks = 1;
    return blocks * kBlockBytes;
}

// RuntimeBloom::expected_fpp (bloom.rs:275-): the Poisson-weighted estimate.
double bloom_expected_fpp(int64_t nbytes, uint64_t items) {
    const double blocks = (double)(nbytes / kBlockBytes);
    const double lambda = (double)items / blocks;
    if (lambda == 0.0) return 0.0;
    if (lambda > 1024.0) return std::pow(1.0 - std::pow(31.0 / 32.0, lambda), 8);
    const double spread = 10.0 * std::sqrt(lambda) + 20.0;
    const double lo = std::floor(std::fmax(lambda - spread, 0.0)), hi = lambda + spread;
    double ln_p = -lambda;
    double k = 1.0;
    while (k <= lo) {
        ln_p += std::log(lambda) - std::log(k);
        k += 1.0;
    }
    double total = 0.0;
    k = lo;
    while (k <= hi) {
        const double word = 1.0 - std::pow(31.0 / 32.0, k);
        total += std::exp(ln_p) * std::pow(word, 8);
        k += 1.0;
        ln_p += std::log(lambda) - std::log(k);
    }
    return total;
}

struct Stats {
    unsigned long long rows;
    long long lo, hi;
    unsigned long long distinct;
    unsigned int overflow;  // more distinct keys than the exact set holds
    unsigned int has_min;   // INT64_MIN seen (kept beside the set)
};

// One pass: kept rows, min, max, and the distinct keys while few (the
// builder's `Distinct`, filter.rs:140-150), into an open-addressing set.
__global__ void __launch_bounds__(256) stats_kernel(const int64_t *keys, const uint8_t *valid, int64_t voff,
                                                    int64_t n, unsigned long long *set, uint64_t mask,
                                                    uint64_t max_distinct, Stats *st) {
    __shared__ unsigned long long s_rows;
    __shared__ long long s_lo, s_hi;
    if (threadIdx.x == 0) {
        s_rows = 0;
        s_lo = LLONG_MAX;
        s_hi = LLONG_MIN;
    }
    __syncthreads();
    unsigned long long rows = 0;
    long long lo = LLONG_MAX, hi = LLONG_MIN;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += stride) {
        if (!bit_get(valid, voff, i)) continue;
        const long long k = keys[i];
        rows++;
        lo = k < lo ? k : lo;
        hi = k > hi ? k : hi;
        if (*(volatile unsigned int *)&st->overflow) continue;
        if (k == kEmptyKey) {
            if (atomicExch(&st->has_min, 1u) == 0u) {
                if (atomicAdd(&st->distinct, 1ull) + 1 > max_distinct) atomicExch(&st->overflow, 1u);
            }
            continue;
        }
        uint64_t pos = hash_word((uint64_t)k) & mask;
        for (uint64_t p = 0; p <= mask; p++) {
            // Past the exact forms' capacity the set is abandoned: stop at once
            // (thousands of concurrent inserts may have filled it).
            if (*(volatile unsigned int *)&st->overflow) break;
            const unsigned long long s = __ldcg(set + pos);
            if (s == (unsigned long long)k) break;
            if (s == (unsigned long long)kEmptyKey) {
                const unsigned long long old = atomicCAS(set + pos, (unsigned long long)kEmptyKey, (unsigned long long)k);
                if (old == (unsigned long long)kEmptyKey) {
                    if (atomicAdd(&st->distinct, 1ull) + 1 > max_distinct) atomicExch(&st->overflow, 1u);
                    break;
                }
                if (old == (unsigned long long)k) break;
            }
            pos = (pos + 1) & mask;
            if (p == mask) atomicExch(&st->overflow, 1u);
        }
    }
    atomicAdd(&s_rows, rows);
    atomicMin(&s_lo, lo);
    atomicMax(&s_hi, hi);
    __syncthreads();
    if (threadIdx.x == 0) {
        atomicAdd(&st->rows, s_rows);
        atomicMin(&st->lo, s_lo);
        atomicMax(&st->hi, s_hi);
    }
}

__global__ void fill_u64_kernel(unsigned long long *p, uint64_t n, unsigned long long v) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        p[i] = v;
}

// RuntimeBloom::insert_hash (bloom.rs:136-148) for every kept key.
__global__ void __launch_bounds__(256) bloom_insert_kernel(const int64_t *keys, const uint8_t *valid, int64_t voff,
                                                           int64_t n, uint32_t *words, uint64_t nblocks) {
    // Eight lanes per key, lane w setting the key's bit in word w: a warp's
    // atomic instruction then touches 4 blocks (one 32-byte sector each)
    // instead of 32.
    const int w = (int)(threadIdx.x & 7u);
    const int64_t stride = ((int64_t)gridDim.x * blockDim.x) >> 3;
    for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 3; i < n; i += stride) {
        if (!bit_get(valid, voff, i)) continue;
        const uint64_t h = xxh64_u64((uint64_t)keys[i]);
        atomicOr(words + sbbf_block(h, nblocks) * 8 + w, sbbf_bit((uint32_t)h, w));
    }
}

}  // namespace

namespace {
// KeyFilter::evaluate_keys (filter.rs:776-798): the bit of row i is whether
// it may match; a NULL row passes only when the producer let NULLs pass.
__global__ void __launch_bounds__(256) evaluate_kernel(KeyFilterDev f, const int64_t *keys, const uint8_t *valid,
                                                       int64_t voff, int64_t n, uint32_t *out) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t base = blockIdx.x * (int64_t)blockDim.x; base < n; base += stride) {
        const int64_t i = base + threadIdx.x;
        bool pass = false;
        if (i < n) {
            const bool v = bit_get(valid, voff, i);
            pass = v ? filter_pass(f, keys[i]) : f.nulls_pass != 0;
        }
        const unsigned word = __ballot_sync(0xFFFFFFFFu, pass);
        if ((threadIdx.x & 31) == 0 && i < n) out[i >> 5] = word;
    }
}
}  // namespace

void finish_bloom(Runtime *rt, const krv_key_filter_options &opt, const DevCol &keys, KeyFilterImpl &f);

KeyFilterDev key_filter_dev(const KeyFilterImpl &f) {
    KeyFilterDev d{};
    d.form = f.info.form;
    d.has_range = f.info.has_range;
    d.lo = f.info.lo;
    d.hi = f.info.hi;
    d.bloom = f.bloom.as<uint32_t>();
    d.nblocks = (uint64_t)(f.info.bloom_bytes / kBlockBytes);
    d.exact = f.exact_slots.as<unsigned long long>();
    d.exact_mask = f.exact_mask;
    d.exact_has_min = f.exact_has_min;
    d.nulls_pass = f.info.nulls_pass;
    return d;
}

std::shared_ptr<KeyFilterImpl> build_key_filter(Runtime *rt, const krv_key_filter_options &opt,
                                                const DevCol &keys, const KeyStats *known) {
    if (keys.type.id != Type::I64) fail(KRV_UNSUPPORTED, "key filters over int64 keys only");
    DeviceGuard g(rt);
    auto f = std::make_shared<KeyFilterImpl>();
    f->rt = rt;
    f->opt = opt;
    const uint64_t distinct_max = (uint64_t)std::max<int64_t>(opt.max_values, opt.exact_max_values);
    if (known && (known->rows == 0 || (uint64_t)known->distinct > distinct_max)) {
        // A join build counted the rows, distinct keys and range: no exact form
        // can apply, so no pass over the keys is needed before the Bloom.
        krv_key_filter_info &info = f->info;
        info.keys = known->rows;
        info.nulls_pass = 0;
        if (known->rows == 0) {
            info.form = KRV_FILTER_EMPTY;
            return f;
        }
        info.has_range = 1;
        info.lo = known->lo;
        info.hi = known->hi;
        info.distinct = -1;
        finish_bloom(rt, opt, keys, *f);
        return f;
    }
    const uint64_t set_slots = std::max<uint64_t>(64, next_pow2(2 * (distinct_max + 1)));
    f->exact_slots = DBuf(rt, set_slots * 8);
    f->exact_mask = set_slots - 1;
    fill_u64_kernel<<<grid_for(rt, (int64_t)set_slots, 256), 256, 0, rt->stream>>>(
        f->exact_slots.as<unsigned long long>(), set_slots, (unsigned long long)kEmptyKey);
    rt->launches++;
    DBuf stats(rt, sizeof(Stats));
    Stats init{0, LLONG_MAX, LLONG_MIN, 0, 0, 0};
    KRV_CUDA(cudaMemcpyAsync(stats.get(), &init, sizeof(Stats), cudaMemcpyHostToDevice, rt->stream));
    const int64_t n = keys.length;
    if (n > 0) {
        stats_kernel<<<grid_for(rt, n, 256, 8), 256, 0, rt->stream>>>(
            static_cast<const int64_t *>(keys.data), keys.valid, keys.valid_off, n,
            f->exact_slots.as<unsigned long long>(), f->exact_mask, distinct_max, stats.as<Stats>());
        rt->launches++;
        check_launch("stats_kernel");
    }
    Stats st = read_scalar<Stats>(rt, stats.get());
    krv_key_filter_info &info = f->info;
    info.keys = (int64_t)st.rows;
    info.nulls_pass = 0;  // NULL `=` keys are never kept by a join build
    if (st.rows == 0) {
        info.form = KRV_FILTER_EMPTY;
        return f;
    }
    info.has_range = 1;
    info.lo = st.lo;
    info.hi = st.hi;
    f->exact_has_min = (int32_t)st.has_min;
    // finish_with (filter.rs:533-593)
    if (!st.overflow) {
        info.distinct = (int64_t)st.distinct;
        const __int128 span = (__int128)st.hi - (__int128)st.lo + 1;
        if (span == (__int128)st.distinct) {
            info.form = KRV_FILTER_RANGE;  // dense (filter.rs:595-604): the range is exact
        } else if ((int64_t)st.distinct <= opt.exact_max_values) {
            info.form = KRV_FILTER_EXACT;
        } else {
            info.form = KRV_FILTER_RANGE;
        }
        if (info.form != KRV_FILTER_EXACT) f->exact_slots.reset();
        if (info.form == KRV_FILTER_EXACT || info.form == KRV_FILTER_RANGE) return f;
    }
    f->exact_slots.reset();
    info.distinct = -1;  // more than the exact forms hold
    finish_bloom(rt, opt, keys, *f);
    return f;
}

// bloom() (filter.rs:606-621): a Bloom filter sized for every kept row
// (info.keys), capped, unless expected to pass too many false positives;
// else the range alone.
void finish_bloom(Runtime *rt, const krv_key_filter_options &opt, const DevCol &keys, KeyFilterImpl &f) {
    krv_key_filter_info &info = f.info;
    const uint64_t rows = (uint64_t)info.keys;
    if (!opt.bloom || rows > (uint64_t)opt.bloom_max_items) {
        info.form = KRV_FILTER_RANGE;
        return;
    }
    int64_t bytes = opt.bloom_bytes > 0 ? opt.bloom_bytes : bloom_bytes_for(rows, opt.bloom_fpp);
    bytes = std::min<int64_t>(bytes, opt.bloom_max_bytes);
    bytes = std::max<int64_t>(1, ceil_div(bytes, kBlockBytes)) * kBlockBytes;  // with_bytes (bloom.rs:115-121)
    if (bloom_expected_fpp(bytes, rows) > opt.bloom_max_fpp) {
        info.form = KRV_FILTER_RANGE;
        return;
    }
    f.bloom = DBuf(rt, (size_t)bytes);
    KRV_CUDA(cudaMemsetAsync(f.bloom.get(), 0, (size_t)bytes, rt->stream));
    const int64_t n = keys.length;
    if (n > 0) {
        bloom_insert_kernel<<<grid_for(rt, n * 8, 256, 8), 256, 0, rt->stream>>>(
            static_cast<const int64_t *>(keys.data), keys.valid, keys.valid_off, n, f.bloom.as<uint32_t>(),
            (uint64_t)(bytes / kBlockBytes));
        rt->launches++;
        check_launch("bloom_insert_kernel");
    }
    info.form = KRV_FILTER_BLOOM;
    info.bloom_bytes = bytes;
}

DevCol evaluate_key_filter(const KeyFilterImpl &f, const DevCol &keys) {
    if (keys.type.id != Type::I64) fail(KRV_UNSUPPORTED, "key filters over int64 keys only");
    Runtime *rt = f.rt;
    DeviceGuard g(rt);
    const int64_t n = keys.length;
    DevCol out = make_col(rt, DType{Type::Bool, 0, 0}, n, false, "pass");
    KRV_CUDA(cudaMemsetAsync(const_cast<void *>(out.data), 0, out.hold_data->bytes(), rt->stream));
    if (n > 0) {
        evaluate_kernel<<<grid_for(rt, n, 256, 8), 256, 0, rt->stream>>>(
            key_filter_dev(f), static_cast<const int64_t *>(keys.data), keys.valid, keys.valid_off, n,
            (uint32_t *)out.data);
        rt->launches++;
        check_launch("evaluate_kernel");
    }
    return out;
}

}  // namespace krv
