// krv_filter.cuh -- the device-side member test of a runtime key filter,
// shared by the filter's evaluate kernel and the fused pipelines.
#pragma once

#include "krv_device.cuh"
#include "ops.h"

namespace krv {

constexpr int64_t kFilterEmptyKey = (int64_t)0x8000000000000000ULL;

// Member test of one valid key (member.rs:423-560): range, then the form.
__device__ __forceinline__ bool filter_pass(const KeyFilterDev &f, int64_t k) {
    if (f.form == KRV_FILTER_EMPTY) return false;
    if (f.has_range && (k < f.lo || k > f.hi)) return false;
    if (f.form == KRV_FILTER_BLOOM) {
        const uint64_t h = xxh64_u64((uint64_t)k);
        return sbbf_check_words(f.bloom + sbbf_block(h, f.nblocks) * 8, (uint32_t)h);
    }
    if (f.form == KRV_FILTER_EXACT) {
        if (k == kFilterEmptyKey) return f.exact_has_min != 0;
        uint64_t pos = hash_word((uint64_t)k) & f.exact_mask;
        for (uint64_t p = 0; p <= f.exact_mask; p++) {
            const unsigned long long s = __ldg(f.exact + pos);
            if (s == (unsigned long long)k) return true;
            if (s == (unsigned long long)kFilterEmptyKey) return false;
            pos = (pos + 1) & f.exact_mask;
        }
        return false;
    }
    return true;
}

}  // namespace krv
