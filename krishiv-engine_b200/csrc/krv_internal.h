// krv_internal.h -- host-side internals shared by the operators: the
// runtime (device, stream, HBM budget), device buffers, column views and the
// Arrow C (Device) Data Interface import/export.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "krv_gpu.h"

namespace krv {

// An error crossing no ABI: thrown inside the library, caught at the C
// boundary and turned into a krv_status (no panics in library code, as the
// reference's clippy `panic = "deny"` rule asks).
struct Error {
    krv_status code;
    std::string msg;
    int64_t need_bytes = 0;
};

[[noreturn]] void fail(krv_status code, const std::string &msg);
void set_last_error(krv_status code, const std::string &msg, int64_t need = 0);

#define KRV_CUDA(expr)                                                                \
    do {                                                                              \
        cudaError_t e_ = (expr);                                                      \
        if (e_ != cudaSuccess)                                                        \
            ::krv::fail(KRV_CUDA_ERROR, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// After a launch: a launch error becomes KRV_CUDA_ERROR.
void check_launch(const char *what);

// The allocation bookkeeping of a runtime, shared with every buffer it
// handed out (an exported output may outlive the runtime).
struct Pool {
    std::atomic<int64_t> used{0};
    int64_t budget = 0;           // bytes; 0 = unlimited
    cudaStream_t stream = nullptr;
    int device = 0;
    std::atomic<bool> alive{true};
};

// Page-locked host blocks kept for reuse: the spill space of partitioned
// joins (the engine spills grace partitions to disk; a GPU spills them over
// the host link to host memory). Freed with the runtime.
class HostPool {
  public:
    static constexpr size_t kBlock = size_t(256) << 20;
    HostPool() = default;
    HostPool(const HostPool &) = delete;
    HostPool &operator=(const HostPool &) = delete;
    ~HostPool();
    // A block of at least `bytes` (kBlock, or exactly `bytes` when larger).
    uint8_t *take(size_t bytes);
    void give(uint8_t *p, size_t bytes);

  private:
    std::mutex mu_;
    std::vector<std::pair<uint8_t *, size_t>> free_, all_;
};

struct Runtime {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int64_t budget = 0;           // bytes; 0 = unlimited
    std::shared_ptr<Pool> pool;
    std::atomic<int64_t> launches{0};
    int sm_count = 148;
    int max_smem_optin = 227 * 1024;
    void *status_dev = nullptr;   // device status words (errors from kernels)
    void *status_host = nullptr;  // pinned mirror
    void *status_host_dev = nullptr;  // its device address
    // Work queued on the stream still reads the caller's host buffers
    // (copies from page-locked memory, or columns read in place).
    bool host_borrowed = false;
    std::shared_ptr<HostPool> host_pool = std::make_shared<HostPool>();
};

// Scope of a call that takes host batches: the caller owns its buffers again
// when the call returns, so the call waits for the work that reads them.
struct HostBorrow {
    Runtime *rt;
    explicit HostBorrow(Runtime *r) : rt(r) { rt->host_borrowed = false; }
    ~HostBorrow() {
        if (rt->host_borrowed) cudaStreamSynchronize(rt->stream);
        rt->host_borrowed = false;
    }
    HostBorrow(const HostBorrow &) = delete;
    HostBorrow &operator=(const HostBorrow &) = delete;
};

// Makes `rt`'s device current for the scope.
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(const Runtime *rt);
    ~DeviceGuard();
};

// Stream-ordered device allocation charged to the runtime's budget.
class DBuf {
  public:
    DBuf() = default;
    DBuf(Runtime *rt, size_t bytes);
    ~DBuf();
    DBuf(const DBuf &) = delete;
    DBuf &operator=(const DBuf &) = delete;
    DBuf(DBuf &&o) noexcept { swap(o); }
    DBuf &operator=(DBuf &&o) noexcept {
        DBuf t(std::move(o));
        swap(t);
        return *this;
    }
    void swap(DBuf &o) noexcept {
        std::swap(pool_, o.pool_);
        std::swap(p_, o.p_);
        std::swap(bytes_, o.bytes_);
    }
    void reset();
    void *get() const { return p_; }
    template <class T> T *as() const { return static_cast<T *>(p_); }
    size_t bytes() const { return bytes_; }

  private:
    std::shared_ptr<Pool> pool_;
    void *p_ = nullptr;
    size_t bytes_ = 0;
};

// Column types of the path (Arrow format strings in parentheses).
enum class Type : int32_t {
    Bool = 1,    // "b" (bit-packed)
    I32 = 2,     // "i"
    I64 = 3,     // "l"
    F64 = 4,     // "g"
    Dec64 = 5,   // "d:p,s,64"
    Dec128 = 6,  // "d:p,s" / "d:p,s,128"
    Date32 = 7,  // "tdD" (int32 days)
    U8 = 8,      // "C" (internal)
    Utf8 = 9,    // "u" (int32 offsets + bytes)
    Binary = 10, // "z" (int32 offsets + bytes)
};

struct DType {
    Type id = Type::I64;
    int32_t precision = 0;
    int32_t scale = 0;
    int width() const;  // bytes per value (Bool: 0, bit-packed; Utf8/Binary: 0, variable)
    bool var() const { return id == Type::Utf8 || id == Type::Binary; }
    std::string format() const;
    bool operator==(const DType &o) const {
        return id == o.id && precision == o.precision && scale == o.scale;
    }
    bool operator!=(const DType &o) const { return !(*this == o); }
};
DType parse_format(const char *fmt);

// A column in device memory. `data` points at element 0 of the column (the
// Arrow offset applied); `valid` is a bitmap whose bit `valid_off` is row 0.
struct DevCol {
    DType type;
    int64_t length = 0;
    const void *data = nullptr;  // values; Utf8/Binary: int32 offsets of rows 0..length
    const void *bytes = nullptr; // Utf8/Binary: value i is bytes[offsets[i] .. offsets[i + 1])
    int64_t var_bytes = -1;      // Utf8/Binary: offsets[length] when offsets[0] is 0 and it is known
    const void *host = nullptr;  // a column read in place: its host address
    const uint8_t *valid = nullptr;
    int64_t valid_off = 0;
    bool nullable = true;
    std::string name;
    std::shared_ptr<DBuf> hold_data;   // owned memory, if any
    std::shared_ptr<DBuf> hold_valid;
    std::shared_ptr<DBuf> hold_bytes;
};

struct DevBatch {
    std::vector<DevCol> cols;
    int64_t rows = 0;
};

// Import: host batch -> device (copies), device batch -> views (no copy).
// With HostRead::InPlace, columns in page-locked host memory (cudaHostAlloc,
// cudaHostRegister) become views that kernels read where they lie, over the
// host link, and only the bytes a kernel touches cross it; other columns are
// copied. Either way the calling entry point holds a HostBorrow.
// Utf8/Binary columns are taken only where `var` is Var::Allow (an
// aggregate's group keys, a join's keys); elsewhere they fail with
// KRV_UNSUPPORTED.
enum class HostRead { Copy, InPlace };
enum class Var { Reject, Allow };
DevBatch import_host(Runtime *rt, const ArrowArray *arr, const ArrowSchema *schema,
                     HostRead mode = HostRead::Copy, Var var = Var::Reject);
DevBatch import_device(Runtime *rt, const ArrowDeviceArray *arr, const ArrowSchema *schema, Var var = Var::Reject);
// Export: moves the batch's buffers to the caller.
void export_host(Runtime *rt, const DevBatch &b, ArrowArray *out, ArrowSchema *out_schema);
void export_device(Runtime *rt, const DevBatch &b, ArrowDeviceArray *out,
                   ArrowSchema *out_schema);
// A schema for a batch (names + types + nullability).
void export_schema(const DevBatch &b, ArrowSchema *out);

// A new owned device column of `n` values (validity bitmap if `nullable`).
DevCol make_col(Runtime *rt, DType t, int64_t n, bool nullable, const std::string &name);
// Slice rows [from, from + n) of a column as a view sharing its memory.
DevCol slice_col(const DevCol &c, int64_t from, int64_t n);

// Copy a small device value to the host (synchronizes the stream).
// Reads n (<= 4032) bytes of device memory after the work queued on the
// runtime's stream: a one-block kernel stores them into mapped page-locked
// memory, so the read does not queue behind bulk copies on the copy engines.
void read_device(Runtime *rt, const void *dev, size_t n, void *host);
template <class T> T read_scalar(Runtime *rt, const void *dev) {
    T v;
    read_device(rt, dev, sizeof(T), &v);
    return v;
}

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }
inline uint64_t next_pow2(uint64_t v) {
    uint64_t p = 1;
    while (p < v) p <<= 1;
    return p;
}

// Grid size for a streaming kernel: a multiple of the SM count.
int grid_for(const Runtime *rt, int64_t work_items, int threads, int per_sm = 4);

// Status words written by kernels (bounded waits that gave up, overflow,
// capacity). Reset with clear_status, read with take_status.
enum StatusBit : uint32_t {
    ST_TIMEOUT = 1u,
    ST_OVERFLOW = 2u,
    ST_CAPACITY = 4u,
    ST_TOO_MANY = 8u,
    ST_MISCOUNT = 16u,  // a pass wrote more rows than its counting pass gave it room for
};
uint32_t *status_word(Runtime *rt);
void clear_status(Runtime *rt);
uint32_t take_status(Runtime *rt);  // synchronizes

}  // namespace krv
