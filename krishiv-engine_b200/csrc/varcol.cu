// varcol.cu -- variable-width (UTF-8 / binary) columns on the join path: the
// build arena's string columns (one byte heap, a start and a length per row)
// and the gather that makes an output string column from the source rows of
// the output rows (Arrow int32 offsets plus bytes).
//
// Reference: the row layout keeps strings as 16-byte views into a heap
// (crates/krishiv-exec/src/rows/layout.rs:24-31, 906-1030), and the probe
// decodes a build payload of the matched rows into Arrow columns
// (join/mod.rs:907-927, Shared::build_columns). Here the arena keeps the
// strings' bytes in one heap per column and the output is gathered by row.
#include <algorithm>
#include <string>

#include "krv_device.cuh"
#include "ops.h"

namespace krv {

namespace {

constexpr int kScanThreads = 1024;
constexpr int kScanPer = 4;
constexpr int kScanTile = kScanThreads * kScanPer;

// Arena rows [base, base + n) of a string column: start in the heap
// (heap_at + offs[r] - o0) and length.
__global__ void var_append_kernel(const int32_t *offs, int64_t n, int64_t base, long long heap_at, int32_t o0,
                                  long long *starts, int32_t *lens) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        starts[base + r] = heap_at + (long long)(offs[r] - o0);
        lens[base + r] = offs[r + 1] - offs[r];
    }
}

// The length of each output row's value (0 where the source row is absent,
// -1 in `idx`, or its value NULL); the output validity word of each 32 rows.
__global__ void var_len_kernel(VarSrc s, const long long *idx, int64_t m, int32_t *len, uint32_t *ovalid) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t base = blockIdx.x * (int64_t)blockDim.x; base < m; base += stride) {
        const int64_t j = base + threadIdx.x;
        bool v = false;
        int32_t l = 0;
        if (j < m) {
            const long long r = idx ? idx[j] : j;
            if (r >= 0 && bit_get(s.valid, s.voff, r)) {
                v = true;
                l = s.lens ? s.lens[r] : s.offs[r + 1] - s.offs[r];
            }
            len[j] = l;
        }
        if (ovalid) {
            const unsigned w = __ballot_sync(0xFFFFFFFFu, v);
            if ((threadIdx.x & 31) == 0 && j < m) ovalid[j >> 5] = w;
        }
    }
}

// Exclusive scan of int32 lengths into int64 offsets: per tile, then the
// tiles' totals (one block), then the totals added back.
__global__ void __launch_bounds__(kScanThreads) scan_tile_kernel(const int32_t *in, int64_t n, long long *out,
                                                                 long long *tile_sum) {
    __shared__ long long s_warp[kScanThreads / 32];
    const int64_t t0 = (int64_t)blockIdx.x * kScanTile;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    long long v[kScanPer], sum = 0;
#pragma unroll
    for (int k = 0; k < kScanPer; k++) {
        const int64_t i = t0 + (int64_t)threadIdx.x * kScanPer + k;
        v[k] = i < n ? in[i] : 0;
        sum += v[k];
    }
    long long incl = sum;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const long long y = __shfl_up_sync(0xFFFFFFFFu, incl, d);
        if (lane >= d) incl += y;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        long long w = lane < kScanThreads / 32 ? s_warp[lane] : 0;
        long long wi = w;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const long long y = __shfl_up_sync(0xFFFFFFFFu, wi, d);
            if (lane >= d) wi += y;
        }
        if (lane < kScanThreads / 32) s_warp[lane] = wi - w;
        if (lane == kScanThreads / 32 - 1) tile_sum[blockIdx.x] = wi;
    }
    __syncthreads();
    long long acc = s_warp[warp] + incl - sum;
#pragma unroll
    for (int k = 0; k < kScanPer; k++) {
        const int64_t i = t0 + (int64_t)threadIdx.x * kScanPer + k;
        if (i < n) out[i] = acc;
        acc += v[k];
    }
}

__global__ void __launch_bounds__(kScanThreads) scan_totals_kernel(long long *tile_sum, int64_t tiles,
                                                                   long long *total) {
    __shared__ long long s_warp[kScanThreads / 32];
    __shared__ long long s_carry;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    for (int64_t b = 0; b < tiles; b += kScanThreads) {
        const int64_t i = b + threadIdx.x;
        const long long v = i < tiles ? tile_sum[i] : 0;
        long long incl = v;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const long long y = __shfl_up_sync(0xFFFFFFFFu, incl, d);
            if (lane >= d) incl += y;
        }
        if (lane == 31) s_warp[warp] = incl;
        __syncthreads();
        long long before = s_carry;
        for (int w = 0; w < warp; w++) before += s_warp[w];
        if (i < tiles) tile_sum[i] = before + incl - v;
        __syncthreads();
        if (threadIdx.x == 0)
            for (int w = 0; w < kScanThreads / 32; w++) s_carry += s_warp[w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = s_carry;
}

// out (int32 offsets, m + 1 of them) = tile prefix + in-tile offset.
__global__ void scan_finish_kernel(const long long *part, const long long *tile_sum, int64_t m,
                                   const long long *total, int32_t *offs) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i <= m; i += (int64_t)gridDim.x * blockDim.x)
        offs[i] = i < m ? (int32_t)(tile_sum[i / kScanTile] + part[i]) : (int32_t)*total;
}

// The bytes of each output row, one warp per row (lanes copy strided bytes).
__global__ void var_copy_kernel(VarSrc s, const long long *idx, int64_t m, const int32_t *offs, uint8_t *out) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x / 32);
    for (int64_t j = (int64_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5); j < m; j += warps) {
        const int32_t len = offs[j + 1] - offs[j];
        if (len == 0) continue;
        const long long r = idx ? idx[j] : j;
        const uint8_t *src = s.bytes + (s.starts ? s.starts[r] : (long long)s.offs[r]);
        uint8_t *dst = out + offs[j];
        for (int32_t b = lane; b < len; b += 32) dst[b] = src[b];
    }
}

}  // namespace

void var_arena_append(Runtime *rt, VarArena &a, const DevCol &c, int64_t base_row, int64_t n) {
    if (n == 0) return;
    int32_t ends[2] = {0, 0};
    read_device(rt, c.data, 4, &ends[0]);
    read_device(rt, static_cast<const int32_t *>(c.data) + n, 4, &ends[1]);
    const int64_t nbytes = (int64_t)ends[1] - ends[0];
    if (nbytes < 0) fail(KRV_INVALID_ARGUMENT, "column '" + c.name + "' has decreasing offsets");
    if (a.heap_size + nbytes > a.heap_cap) {
        const int64_t cap = std::max<int64_t>({a.heap_size + nbytes, a.heap_cap * 2, 4096});
        auto nh = std::make_shared<DBuf>(rt, (size_t)cap);
        if (a.heap_size)
            KRV_CUDA(cudaMemcpyAsync(nh->get(), a.heap->get(), (size_t)a.heap_size, cudaMemcpyDeviceToDevice, rt->stream));
        a.heap = nh;
        a.heap_cap = cap;
    }
    if (nbytes)
        KRV_CUDA(cudaMemcpyAsync(a.heap->as<uint8_t>() + a.heap_size, static_cast<const uint8_t *>(c.bytes) + ends[0],
                                 (size_t)nbytes, cudaMemcpyDeviceToDevice, rt->stream));
    var_append_kernel<<<grid_for(rt, n, 256, 8), 256, 0, rt->stream>>>(
        static_cast<const int32_t *>(c.data), n, base_row, a.heap_size, ends[0], a.starts->as<long long>(),
        a.lens->as<int32_t>());
    rt->launches++;
    check_launch("var_append_kernel");
    a.heap_size += nbytes;
}

DevCol var_gather(Runtime *rt, const VarSrc &src, const long long *idx, int64_t m, DType type, bool nullable,
                  const std::string &name) {
    DevCol col;
    col.type = type;
    col.name = name;
    col.nullable = nullable;
    col.length = m;
    if (nullable) {
        col.hold_valid = std::make_shared<DBuf>(rt, (size_t)ceil_div(std::max<int64_t>(m, 1), 32) * 4 + 8);
        KRV_CUDA(cudaMemsetAsync(col.hold_valid->get(), 0, col.hold_valid->bytes(), rt->stream));
        col.valid = col.hold_valid->as<uint8_t>();
    }
    col.hold_data = std::make_shared<DBuf>(rt, (size_t)(m + 1) * 4);
    col.data = col.hold_data->get();
    if (m == 0) {
        KRV_CUDA(cudaMemsetAsync(col.hold_data->get(), 0, 4, rt->stream));
        col.hold_bytes = std::make_shared<DBuf>(rt, 8);
        col.bytes = col.hold_bytes->get();
        col.var_bytes = 0;
        return col;
    }
    DBuf len(rt, (size_t)m * 4), part(rt, (size_t)m * 8);
    const int64_t tiles = ceil_div(m, kScanTile);
    DBuf tile_sum(rt, (size_t)tiles * 8), total(rt, 8);
    var_len_kernel<<<grid_for(rt, m, 256, 8), 256, 0, rt->stream>>>(src, idx, m, len.as<int32_t>(),
                                                                    nullable ? col.hold_valid->as<uint32_t>() : nullptr);
    scan_tile_kernel<<<(int)tiles, kScanThreads, 0, rt->stream>>>(len.as<int32_t>(), m, part.as<long long>(),
                                                                  tile_sum.as<long long>());
    scan_totals_kernel<<<1, kScanThreads, 0, rt->stream>>>(tile_sum.as<long long>(), tiles, total.as<long long>());
    const long long bytes = read_scalar<long long>(rt, total.get());
    if (bytes > 0x7FFFFFFFll) fail(KRV_UNSUPPORTED, "a string output column of 2 GiB or more in one batch");
    scan_finish_kernel<<<grid_for(rt, m + 1, 256, 8), 256, 0, rt->stream>>>(
        part.as<long long>(), tile_sum.as<long long>(), m, total.as<long long>(), col.hold_data->as<int32_t>());
    col.hold_bytes = std::make_shared<DBuf>(rt, (size_t)std::max<long long>(bytes, 8));
    col.bytes = col.hold_bytes->get();
    col.var_bytes = bytes;
    if (bytes > 0)
        var_copy_kernel<<<grid_for(rt, m * 32, 256, 8), 256, 0, rt->stream>>>(src, idx, m, col.hold_data->as<int32_t>(),
                                                                           col.hold_bytes->as<uint8_t>());
    rt->launches += bytes > 0 ? 5 : 4;
    check_launch("var_gather");
    return col;
}

}  // namespace krv
