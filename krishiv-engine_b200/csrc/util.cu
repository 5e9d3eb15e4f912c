// util.cu -- small device utilities shared by the operators: bitmap append
// and fill at arbitrary bit offsets.
#include "krv_device.cuh"
#include "ops.h"

namespace krv {

namespace {

// Each thread builds one 32-bit destination word from the source bits that
// land in it and ORs it in: one atomic per 32 rows, any offsets.
__global__ void append_bits_kernel(const uint8_t *src, int64_t src_off, int64_t n, uint32_t *dst,
                                   int64_t dst_off) {
    const int64_t first_word = dst_off >> 5;
    const int64_t last_word = (dst_off + n - 1) >> 5;
    for (int64_t w = first_word + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; w <= last_word;
         w += (int64_t)gridDim.x * blockDim.x) {
        uint32_t word = 0;
        for (int b = 0; b < 32; b++) {
            const int64_t d = (w << 5) + b;  // destination bit
            const int64_t r = d - dst_off;   // source row
            if (r >= 0 && r < n && (src == nullptr || bit_get(src, src_off, r))) word |= 1u << b;
        }
        if (word) atomicOr(&dst[w], word);
    }
}

}  // namespace

void append_bits(Runtime *rt, const uint8_t *src, int64_t src_off, int64_t n, uint8_t *dst,
                 int64_t dst_off) {
    if (n <= 0) return;
    const int64_t words = ((dst_off + n - 1) >> 5) - (dst_off >> 5) + 1;
    append_bits_kernel<<<grid_for(rt, words, 256), 256, 0, rt->stream>>>(
        src, src_off, n, reinterpret_cast<uint32_t *>(dst), dst_off);
    rt->launches++;
    check_launch("append_bits_kernel");
}

void set_bits(Runtime *rt, uint8_t *dst, int64_t dst_off, int64_t n) {
    append_bits(rt, nullptr, 0, n, dst, dst_off);
}

}  // namespace krv
