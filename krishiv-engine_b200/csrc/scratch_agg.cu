// scratch_agg.cu -- a grouped SUM/COUNT over one int64 key that allocates no
// memory: krv_agg_sum_i64_scratch (declared in krv_gpu.h).
//
// It is a variant of the global-table aggregate kernel (aggregate.cu) for
// callers that cannot allocate device memory at the point of the call: an
// engine that has handed all of HBM to its own pool and accounts every byte
// through it, or a loop where a cudaMalloc / cudaFree would stall the device
// (cudaFree waits for all work on it). Its hash table lives in a fixed
// file-scope device array, so the call only launches kernels on the caller's
// stream; the caller owns the inputs and the outputs.
//
// Limits and rules of use:
//  - at most KRV_SCRATCH_MAX_GROUPS distinct keys (the scratch holds a table
//    of twice that many slots); a larger max_groups is rejected on the host;
//  - the first call on a device (with that device current) looks up the
//    address of the scratch array for that device; the CUDA runtime places
//    the array when it loads this file's kernels there. Make that first call
//    before any stream capture;
//  - nothing has to start at zero: each call clears the scratch on its stream
//    before its first row, and writes every output it reports;
//  - calls on one device share one scratch array: two calls that overlap in
//    time on that device (different streams, or host threads) race and give
//    wrong answers. Calls issued one after another on one stream are safe.
//
// Results are those of HashAggregate (crates/krishiv-exec/src/aggregate/
// sink.rs:181) for GROUP BY key with SUM(value) and COUNT(*) over non-NULL
// int64 columns, with spark.sql.ansi.enabled off: a sum that leaves int64
// wraps (two's complement, as SumInt does) and is flagged in out_info[1].
#include <algorithm>
#include <mutex>
#include <string>

#include "krv_device.cuh"
#include "krv_internal.h"

namespace {

constexpr int64_t kMaxGroups = KRV_SCRATCH_MAX_GROUPS;
constexpr int64_t kSlots = 2 * kMaxGroups;  // table slots (power of two)
static_assert((kSlots & (kSlots - 1)) == 0, "slot count must be a power of two");
// The key that marks an empty slot; rows with this key go to slot kSlots.
constexpr unsigned long long kEmpty = 0x8000000000000000ull;
constexpr uint64_t kSeed = 0x53435241544348ull;
// Longest probe run a key may take. With at most kMaxGroups keys the table is
// at most half full and runs stay short; a key that finds no slot within the
// limit (more distinct keys than the table holds) voids the answer.
constexpr int kProbeLimit = 8192;

// Scratch layout, in 64-bit words:
//   keys[kSlots]        slot key (kEmpty: free)
//   cnt[kSlots + 1]     COUNT(*) per slot; slot kSlots holds key kEmpty
//   lo[kSlots + 1]      128-bit SUM per slot, low word
//   hi[kSlots + 1]      128-bit SUM per slot, high word
//   ctl[8]              [0] groups written, [1] a key found no slot, [2] a sum left int64,
//                       [3] slots claimed (distinct keys seen, the marker key aside)
constexpr int64_t kOffCnt = kSlots;
constexpr int64_t kOffLo = kOffCnt + kSlots + 1;
constexpr int64_t kOffHi = kOffLo + kSlots + 1;
constexpr int64_t kOffCtl = kOffHi + kSlots + 1;
constexpr int64_t kScratchWords = (kOffCtl + 8 + 31) / 32 * 32;  // 4 MiB + 128 B

static __device__ __align__(256) unsigned long long g_scratch[kScratchWords];

constexpr int kThreads = 256;
constexpr int kMaxDevices = 64;

struct DeviceScratch {
    unsigned long long *words = nullptr;  // device address of g_scratch
    int blocks = 0;                       // grid of the row kernel
};
std::mutex g_mu;
DeviceScratch g_dev[kMaxDevices];

__global__ void clear_kernel(unsigned long long *s) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < kScratchWords; i += stride)
        s[i] = i < kSlots ? kEmpty : 0ull;
}

// How often (in rows of one thread) the row loop looks at the void flags.
constexpr int kVoidCheckEvery = 8;

// One row: find or claim the key's slot, then add to its count and sum.
// Once the answer is void (a key found no slot, or more than max_groups keys
// claimed slots) the remaining rows are skipped: the kernel would otherwise
// keep walking long probe runs of a full table only to report -1.
__global__ void rows_kernel(unsigned long long *s, const int64_t *__restrict__ keys,
                            const int64_t *__restrict__ values, int64_t n, int64_t max_groups) {
    unsigned long long *slot_key = s;
    unsigned long long *cnt = s + kOffCnt;
    unsigned long long *lo = s + kOffLo;
    long long *hi = reinterpret_cast<long long *>(s + kOffHi);
    unsigned long long *ctl = s + kOffCtl;
    const volatile unsigned long long *vctl = ctl;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int since_check = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        if (++since_check == kVoidCheckEvery) {
            since_check = 0;
            if (vctl[1] != 0 || (int64_t)vctl[3] > max_groups) break;
        }
        const unsigned long long k = (unsigned long long)keys[i];
        const int64_t v = values[i];
        int64_t slot = -1;
        if (k == kEmpty) {
            slot = kSlots;
        } else {
            uint64_t p = krv::finalize(krv::hash_word(k), kSeed) & (uint64_t)(kSlots - 1);
            for (int t = 0; t < kProbeLimit; t++) {
                unsigned long long cur = slot_key[p];
                if (cur == kEmpty) {
                    cur = atomicCAS(&slot_key[p], kEmpty, k);
                    if (cur == kEmpty && (int64_t)atomicAdd(&ctl[3], 1ull) >= max_groups) {
                        // one key more than the caller's outputs hold
                        atomicOr(&ctl[1], 1ull);
                        break;
                    }
                }
                if (cur == kEmpty || cur == k) {
                    slot = (int64_t)p;
                    break;
                }
                p = (p + 1) & (uint64_t)(kSlots - 1);
            }
        }
        if (slot < 0) {  // no slot within the probe limit: the answer is void
            atomicOr(&ctl[1], 1ull);
            continue;
        }
        atomicAdd(&cnt[slot], 1ull);
        krv::atomic_add_i128_from_i64(&lo[slot], &hi[slot], v);
    }
}

// Writes each used slot as one output group (in no particular order).
__global__ void emit_kernel(unsigned long long *s, int64_t max_groups, int64_t *__restrict__ out_keys,
                            int64_t *__restrict__ out_sums, int64_t *__restrict__ out_counts) {
    const unsigned long long *slot_key = s;
    const unsigned long long *cnt = s + kOffCnt;
    const unsigned long long *lo = s + kOffLo;
    const long long *hi = reinterpret_cast<const long long *>(s + kOffHi);
    unsigned long long *ctl = s + kOffCtl;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= kSlots; i += stride) {
        const bool used = i < kSlots ? slot_key[i] != kEmpty : cnt[kSlots] != 0;
        if (!used) continue;
        const unsigned long long at = atomicAdd(&ctl[0], 1ull);
        if ((int64_t)at >= max_groups) continue;
        const unsigned long long l = lo[i];
        const long long h = hi[i];
        const bool fits64 = (h == 0 && !(l >> 63)) || (h == -1 && (l >> 63));
        if (!fits64) atomicOr(&ctl[2], 1ull);
        out_keys[at] = (int64_t)(i < kSlots ? slot_key[i] : kEmpty);
        out_sums[at] = (int64_t)l;
        out_counts[at] = (int64_t)cnt[i];
    }
}

__global__ void info_kernel(const unsigned long long *s, int64_t max_groups, int64_t *out_info) {
    const unsigned long long *ctl = s + kOffCtl;
    const bool void_answer = ctl[1] != 0 || (int64_t)ctl[0] > max_groups;
    out_info[0] = void_answer ? -1 : (int64_t)ctl[0];
    out_info[1] = void_answer ? 0 : (int64_t)(ctl[2] != 0);
}

krv_status error(krv_status code, const std::string &msg) {
    krv::set_last_error(code, msg, 0);
    return code;
}

krv_status cuda_error(const char *what, cudaError_t e) {
    return error(KRV_CUDA_ERROR, std::string(what) + ": " + cudaGetErrorString(e));
}

// The scratch of the current device, looked up on its first use.
krv_status scratch_of(int device, DeviceScratch &out) {
    std::lock_guard<std::mutex> lock(g_mu);
    DeviceScratch &d = g_dev[device];
    if (!d.words) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess) return cuda_error("cudaGetSymbolAddress(scratch)", e);
        int sms = 0;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        if (e != cudaSuccess) return cuda_error("cudaDeviceGetAttribute(multiProcessorCount)", e);
        d.blocks = sms * 8;
        d.words = static_cast<unsigned long long *>(p);
    }
    out = d;
    return KRV_OK;
}

}  // namespace

krv_status krv_agg_sum_i64_scratch(const int64_t *keys, const int64_t *values, int64_t n, int64_t max_groups,
                                   int64_t *out_keys, int64_t *out_sums, int64_t *out_counts, int64_t *out_info,
                                   void *stream) {
    krv::set_last_error(KRV_OK, "", 0);
    if (n < 0) return error(KRV_INVALID_ARGUMENT, "krv_agg_sum_i64_scratch: negative row count");
    if (max_groups < 0 || max_groups > kMaxGroups)
        return error(KRV_INVALID_ARGUMENT,
                     "krv_agg_sum_i64_scratch: max_groups " + std::to_string(max_groups) +
                         " is outside [0, " + std::to_string(kMaxGroups) +
                         "], the groups its fixed scratch table holds");
    if (n > 0 && (!keys || !values))
        return error(KRV_INVALID_ARGUMENT, "krv_agg_sum_i64_scratch: null keys or values");
    if (max_groups > 0 && (!out_keys || !out_sums || !out_counts))
        return error(KRV_INVALID_ARGUMENT, "krv_agg_sum_i64_scratch: null output column");
    if (!out_info) return error(KRV_INVALID_ARGUMENT, "krv_agg_sum_i64_scratch: null out_info");
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return cuda_error("cudaGetDevice", e);
    if (device < 0 || device >= kMaxDevices)
        return error(KRV_INVALID_ARGUMENT, "krv_agg_sum_i64_scratch: device ordinal out of range");
    DeviceScratch d;
    const krv_status st = scratch_of(device, d);
    if (st != KRV_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // Drops an error an earlier, unrelated runtime call left on this thread,
    // so that the check after the launches sees only theirs.
    (void)cudaGetLastError();
    const int slot_blocks = (int)((kScratchWords + kThreads - 1) / kThreads);
    clear_kernel<<<std::min(slot_blocks, d.blocks), kThreads, 0, s>>>(d.words);
    if (n > 0) {
        const int row_blocks = (int)std::min<int64_t>(d.blocks, (n + kThreads - 1) / kThreads);
        rows_kernel<<<row_blocks, kThreads, 0, s>>>(d.words, keys, values, n, max_groups);
    }
    emit_kernel<<<std::min(slot_blocks, d.blocks), kThreads, 0, s>>>(d.words, max_groups, out_keys, out_sums,
                                                                      out_counts);
    info_kernel<<<1, 1, 0, s>>>(d.words, max_groups, out_info);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_error("krv_agg_sum_i64_scratch launch", e);
    return KRV_OK;
}
