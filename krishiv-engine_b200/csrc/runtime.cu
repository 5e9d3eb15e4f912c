// runtime.cu -- the runtime (device, stream, HBM budget), device buffers,
// error plumbing and the Arrow C (Device) Data Interface import/export.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "krv_device.cuh"
#include "krv_internal.h"

namespace krv {

static thread_local std::string g_last_error;
static thread_local int64_t g_last_need = 0;

void set_last_error(krv_status code, const std::string &msg, int64_t need) {
    (void)code;
    g_last_error = msg;
    g_last_need = need;
}

[[noreturn]] void fail(krv_status code, const std::string &msg) { throw Error{code, msg, 0}; }

}  // namespace krv

extern "C" const char *krv_last_error(void) { return krv::g_last_error.c_str(); }
extern "C" int64_t krv_last_need_bytes(void) { return krv::g_last_need; }

namespace krv {

void check_launch(const char *what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) fail(KRV_CUDA_ERROR, std::string(what) + ": " + cudaGetErrorString(e));
}

DeviceGuard::DeviceGuard(const Runtime *rt) {
    cudaGetDevice(&prev);
    if (prev != rt->device) cudaSetDevice(rt->device);
}
DeviceGuard::~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
}

DBuf::DBuf(Runtime *rt, size_t bytes) : pool_(rt->pool), bytes_(bytes) {
    if (bytes == 0) return;
    const size_t rounded = (bytes + 255) & ~size_t(255);
    const int64_t before = pool_->used.fetch_add((int64_t)rounded);
    if (pool_->budget > 0 && before + (int64_t)rounded > pool_->budget) {
        pool_->used.fetch_sub((int64_t)rounded);
        Error e{KRV_NEED_MEMORY,
                "device allocation of " + std::to_string(bytes) + " bytes exceeds the HBM budget (" +
                    std::to_string(before) + " of " + std::to_string(pool_->budget) + " in use)",
                (int64_t)bytes};
        throw e;
    }
    cudaError_t err = cudaMallocAsync(&p_, rounded, rt->stream);
    if (err != cudaSuccess) {
        pool_->used.fetch_sub((int64_t)rounded);
        p_ = nullptr;
        Error e{KRV_NEED_MEMORY,
                std::string("cudaMallocAsync(") + std::to_string(bytes) + "): " + cudaGetErrorString(err),
                (int64_t)bytes};
        cudaGetLastError();
        throw e;
    }
    bytes_ = rounded;
}

void DBuf::reset() {
    if (p_) {
        if (pool_->alive.load()) cudaFreeAsync(p_, pool_->stream);
        else {
            int cur = -1;
            cudaGetDevice(&cur);
            if (cur != pool_->device) cudaSetDevice(pool_->device);
            cudaFree(p_);
            if (cur >= 0 && cur != pool_->device) cudaSetDevice(cur);
        }
        pool_->used.fetch_sub((int64_t)bytes_);
    }
    p_ = nullptr;
    bytes_ = 0;
}
DBuf::~DBuf() { reset(); }

int DType::width() const {
    switch (id) {
    case Type::Bool: return 0;
    case Type::I32: return 4;
    case Type::I64: return 8;
    case Type::F64: return 8;
    case Type::Dec64: return 8;
    case Type::Dec128: return 16;
    case Type::Date32: return 4;
    case Type::U8: return 1;
    case Type::Utf8: return 0;
    case Type::Binary: return 0;
    }
    return 0;
}

std::string DType::format() const {
    switch (id) {
    case Type::Bool: return "b";
    case Type::I32: return "i";
    case Type::I64: return "l";
    case Type::F64: return "g";
    case Type::Dec64:
        return "d:" + std::to_string(precision) + "," + std::to_string(scale) + ",64";
    case Type::Dec128: return "d:" + std::to_string(precision) + "," + std::to_string(scale);
    case Type::Date32: return "tdD";
    case Type::U8: return "C";
    case Type::Utf8: return "u";
    case Type::Binary: return "z";
    }
    return "l";
}

DType parse_format(const char *fmt) {
    if (!fmt) fail(KRV_INVALID_ARGUMENT, "column without a format");
    std::string f(fmt);
    DType t;
    if (f == "b") t.id = Type::Bool;
    else if (f == "i") t.id = Type::I32;
    else if (f == "l") t.id = Type::I64;
    else if (f == "g") t.id = Type::F64;
    else if (f == "tdD") t.id = Type::Date32;
    else if (f == "C") t.id = Type::U8;
    else if (f == "u") t.id = Type::Utf8;
    else if (f == "z") t.id = Type::Binary;
    else if (f.rfind("d:", 0) == 0) {
        int p = 0, s = 0, bits = 128;
        const int n = std::sscanf(f.c_str() + 2, "%d,%d,%d", &p, &s, &bits);
        if (n < 2) fail(KRV_INVALID_ARGUMENT, "bad decimal format " + f);
        if (bits == 64) t.id = Type::Dec64;
        else if (bits == 128) t.id = Type::Dec128;
        else fail(KRV_UNSUPPORTED, "decimal of " + std::to_string(bits) + " bits");
        t.precision = p;
        t.scale = s;
    } else {
        fail(KRV_UNSUPPORTED, "column type with Arrow format '" + f + "'");
    }
    return t;
}

HostPool::~HostPool() {
    for (auto &b : all_) cudaFreeHost(b.first);
}

uint8_t *HostPool::take(size_t bytes) {
    const size_t want = bytes > kBlock ? bytes : kBlock;
    {
        std::lock_guard<std::mutex> lock(mu_);
        for (size_t i = 0; i < free_.size(); i++)
            if (free_[i].second == want) {
                uint8_t *p = free_[i].first;
                free_.erase(free_.begin() + (long)i);
                return p;
            }
    }
    void *p = nullptr;
    const cudaError_t e = cudaHostAlloc(&p, want, cudaHostAllocDefault);
    if (e != cudaSuccess) {
        cudaGetLastError();
        fail(KRV_NEED_MEMORY, std::string("page-locked host spill space: ") + cudaGetErrorString(e));
    }
    std::lock_guard<std::mutex> lock(mu_);
    all_.push_back({static_cast<uint8_t *>(p), want});
    return static_cast<uint8_t *>(p);
}

void HostPool::give(uint8_t *p, size_t bytes) {
    const size_t want = bytes > kBlock ? bytes : kBlock;
    std::lock_guard<std::mutex> lock(mu_);
    free_.push_back({p, want});
}

int grid_for(const Runtime *rt, int64_t work_items, int threads, int per_sm) {
    const int64_t need = ceil_div(work_items > 0 ? work_items : 1, threads);
    const int64_t cap = (int64_t)rt->sm_count * per_sm;
    return (int)(need < cap ? need : cap);
}

uint32_t *status_word(Runtime *rt) { return static_cast<uint32_t *>(rt->status_dev); }
void clear_status(Runtime *rt) {
    KRV_CUDA(cudaMemsetAsync(rt->status_dev, 0, sizeof(uint32_t) * 4, rt->stream));
}
namespace {
__global__ void readback_kernel(const uint8_t *src, size_t n, volatile uint8_t *dst) {
    for (size_t i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
}
}  // namespace

void read_device(Runtime *rt, const void *dev, size_t n, void *host) {
    if (n == 0) return;
    if (n > 4032) fail(KRV_INTERNAL, "read_device: more than 4032 bytes");
    volatile uint8_t *area = static_cast<volatile uint8_t *>(rt->status_host) + 64;
    readback_kernel<<<1, 128, 0, rt->stream>>>(static_cast<const uint8_t *>(dev), n,
                                               static_cast<volatile uint8_t *>(rt->status_host_dev) + 64);
    check_launch("readback_kernel");
    KRV_CUDA(cudaStreamSynchronize(rt->stream));
    for (size_t i = 0; i < n; i++) static_cast<uint8_t *>(host)[i] = area[i];
}

uint32_t take_status(Runtime *rt) {
    uint32_t v = 0;
    read_device(rt, rt->status_dev, sizeof(uint32_t), &v);
    return v;
}

DevCol make_col(Runtime *rt, DType t, int64_t n, bool nullable, const std::string &name) {
    DevCol c;
    c.type = t;
    c.length = n;
    c.name = name;
    c.nullable = nullable;
    const size_t bytes = t.id == Type::Bool ? (size_t)ceil_div(n, 8) : (size_t)n * (size_t)t.width();
    c.hold_data = std::make_shared<DBuf>(rt, bytes > 0 ? bytes : 8);
    c.data = c.hold_data->get();
    if (nullable) {
        c.hold_valid = std::make_shared<DBuf>(rt, (size_t)ceil_div(n > 0 ? n : 1, 8) + 8);
        c.valid = static_cast<const uint8_t *>(c.hold_valid->get());
    }
    return c;
}

DevCol slice_col(const DevCol &c, int64_t from, int64_t n) {
    DevCol s = c;
    s.length = n;
    if (c.type.id == Type::Bool) {
        // Bit-packed data: keep byte alignment requirements simple.
        if (from % 8) fail(KRV_INTERNAL, "unaligned boolean slice");
        s.data = static_cast<const uint8_t *>(c.data) + from / 8;
    } else if (c.type.var()) {
        s.data = static_cast<const int32_t *>(c.data) + from;  // offsets stay absolute into `bytes`
        s.var_bytes = -1;
    } else {
        s.data = static_cast<const uint8_t *>(c.data) + from * c.type.width();
    }
    s.valid_off = c.valid_off + from;
    return s;
}

// ---------------------------------------------------------------------------------
// Arrow import

static void check_struct(const ArrowArray *arr, const ArrowSchema *schema) {
    if (!arr || !schema) fail(KRV_INVALID_ARGUMENT, "null ArrowArray or ArrowSchema");
    if (!schema->format || std::string(schema->format) != "+s")
        fail(KRV_INVALID_ARGUMENT, "a record batch must be a struct array ('+s')");
    if (arr->n_children != schema->n_children)
        fail(KRV_INVALID_ARGUMENT, "array and schema disagree on the column count");
    if (arr->release == nullptr) fail(KRV_INVALID_ARGUMENT, "released ArrowArray");
}

// The device address of host range [p, p + bytes) when all of it is
// page-locked host memory mapped for the device, else nullptr.
static const uint8_t *mapped_host(const uint8_t *p, size_t bytes) {
    if (!p || bytes == 0) return nullptr;
    cudaPointerAttributes a0{}, a1{};
    if (cudaPointerGetAttributes(&a0, p) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    if (a0.type != cudaMemoryTypeHost || !a0.devicePointer) return nullptr;
    const uint8_t *last = p + bytes - 1;
    if (cudaPointerGetAttributes(&a1, last) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    if (a1.type != cudaMemoryTypeHost || !a1.devicePointer) return nullptr;
    const uint8_t *d0 = static_cast<const uint8_t *>(a0.devicePointer);
    if (static_cast<const uint8_t *>(a1.devicePointer) != d0 + (bytes - 1)) return nullptr;
    return d0;
}

// Whether host pointer p is page-locked (a copy from it runs asynchronously).
static bool page_locked(const void *p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// A Utf8/Binary column's offsets and bytes. A device column is viewed where
// it lies; a host column is copied with its offsets rebased to start at 0.
static void import_var(Runtime *rt, bool device, const ArrowArray *c, int64_t off, int64_t rows, DevCol &col) {
    const int32_t *offs = static_cast<const int32_t *>(c->buffers[1]) + off;
    const uint8_t *bytes = static_cast<const uint8_t *>(c->buffers[2]);
    if (device) {
        col.data = offs;
        col.bytes = bytes;
        return;
    }
    const int32_t o0 = rows > 0 ? offs[0] : 0, on = rows > 0 ? offs[rows] : 0;
    if (on < o0) fail(KRV_INVALID_ARGUMENT, "column '" + col.name + "' has decreasing offsets");
    col.hold_data = std::make_shared<DBuf>(rt, (size_t)(rows + 1) * 4);
    std::vector<int32_t> rebased((size_t)rows + 1);
    for (int64_t i = 0; i <= rows; i++) rebased[(size_t)i] = rows > 0 ? offs[i] - o0 : 0;
    KRV_CUDA(cudaMemcpyAsync(col.hold_data->get(), rebased.data(), rebased.size() * 4, cudaMemcpyHostToDevice,
                             rt->stream));
    const size_t nb = (size_t)(on - o0);
    col.hold_bytes = std::make_shared<DBuf>(rt, nb > 0 ? nb : 8);
    if (nb) {
        KRV_CUDA(cudaMemcpyAsync(col.hold_bytes->get(), bytes + o0, nb, cudaMemcpyHostToDevice, rt->stream));
        if (page_locked(bytes + o0)) rt->host_borrowed = true;
    }
    KRV_CUDA(cudaStreamSynchronize(rt->stream));  // `rebased` is read by the copy
    col.data = col.hold_data->get();
    col.bytes = col.hold_bytes->get();
    col.var_bytes = (int64_t)nb;
}

template <bool Device>
static DevBatch import_impl(Runtime *rt, const ArrowArray *arr, const ArrowSchema *schema,
                            HostRead mode = HostRead::Copy, Var var = Var::Reject) {
    check_struct(arr, schema);
    DevBatch b;
    b.rows = arr->length;
    for (int64_t i = 0; i < arr->n_children; i++) {
        const ArrowArray *c = arr->children[i];
        const ArrowSchema *cs = schema->children[i];
        DevCol col;
        col.type = parse_format(cs->format);
        col.name = cs->name ? cs->name : "";
        col.nullable = (cs->flags & ARROW_FLAG_NULLABLE) != 0;
        col.length = b.rows;
        if (c->length < arr->offset + b.rows)
            fail(KRV_INVALID_ARGUMENT, "column '" + col.name + "' is shorter than its batch");
        if (c->n_buffers < 2) fail(KRV_INVALID_ARGUMENT, "column '" + col.name + "' has no data buffer");
        const int64_t off = arr->offset + c->offset;
        const uint8_t *data = static_cast<const uint8_t *>(c->buffers[1]);
        const uint8_t *valid = c->null_count == 0 ? nullptr : static_cast<const uint8_t *>(c->buffers[0]);
        const int w = col.type.width();
        if (col.type.var()) {
            if (var != Var::Allow)
                fail(KRV_UNSUPPORTED, "column '" + col.name + "': string and binary columns are taken as aggregate "
                                      "group keys and join keys only");
            if (c->n_buffers < 3) fail(KRV_INVALID_ARGUMENT, "column '" + col.name + "' has no value bytes buffer");
            import_var(rt, Device, c, off, b.rows, col);
        }
        if (Device) {
            if (col.type.var()) {
                col.valid = valid;
                col.valid_off = off;
            } else if (col.type.id == Type::Bool) {
                if (off % 8) fail(KRV_UNSUPPORTED, "boolean device column at an unaligned offset");
                col.data = data + off / 8;
                col.valid = valid;
                col.valid_off = off;
            } else {
                col.data = data + off * w;
                col.valid = valid;
                col.valid_off = off;
            }
        } else {
            size_t bytes = 0;
            const uint8_t *src = nullptr;
            if (col.type.var()) {
                // imported above
            } else if (col.type.id == Type::Bool) {
                if (off % 8) fail(KRV_UNSUPPORTED, "boolean column at an unaligned offset");
                bytes = (size_t)ceil_div(b.rows, 8);
                src = data + off / 8;
            } else {
                bytes = (size_t)b.rows * (size_t)w;
                src = data + off * w;
            }
            const uint8_t *in_place = mode == HostRead::InPlace && src ? mapped_host(src, bytes) : nullptr;
            if (col.type.var()) {
                // offsets and bytes copied by import_var
            } else if (in_place) {
                col.data = in_place;
                col.host = src;
                rt->host_borrowed = true;
            } else {
                col.hold_data = std::make_shared<DBuf>(rt, bytes > 0 ? bytes : 8);
                if (bytes) {
                    KRV_CUDA(cudaMemcpyAsync(col.hold_data->get(), src, bytes, cudaMemcpyHostToDevice, rt->stream));
                    if (page_locked(src)) rt->host_borrowed = true;
                }
                col.data = col.hold_data->get();
            }
            if (valid) {
                const int64_t first = off / 8, last = (off + b.rows + 7) / 8;
                const size_t vb = (size_t)(last - first);
                col.hold_valid = std::make_shared<DBuf>(rt, vb > 0 ? vb : 8);
                if (vb) {
                    KRV_CUDA(cudaMemcpyAsync(col.hold_valid->get(), valid + first, vb, cudaMemcpyHostToDevice,
                                             rt->stream));
                    if (page_locked(valid + first)) rt->host_borrowed = true;
                }
                col.valid = static_cast<const uint8_t *>(col.hold_valid->get());
                col.valid_off = off % 8;
            }
        }
        b.cols.push_back(std::move(col));
    }
    return b;
}

DevBatch import_host(Runtime *rt, const ArrowArray *arr, const ArrowSchema *schema, HostRead mode, Var var) {
    return import_impl<false>(rt, arr, schema, mode, var);
}

DevBatch import_device(Runtime *rt, const ArrowDeviceArray *arr, const ArrowSchema *schema, Var var) {
    if (!arr) fail(KRV_INVALID_ARGUMENT, "null ArrowDeviceArray");
    if (arr->device_type != ARROW_DEVICE_CUDA)
        fail(KRV_INVALID_ARGUMENT, "device batch is not ARROW_DEVICE_CUDA");
    if (arr->device_id != rt->device)
        fail(KRV_INVALID_ARGUMENT, "device batch lives on device " + std::to_string(arr->device_id) +
                                       ", the runtime on " + std::to_string(rt->device));
    if (arr->sync_event) {
        cudaEvent_t ev = *static_cast<cudaEvent_t *>(arr->sync_event);
        KRV_CUDA(cudaStreamWaitEvent(rt->stream, ev, 0));
    }
    return import_impl<true>(rt, &arr->array, schema, HostRead::Copy, var);
}

// ---------------------------------------------------------------------------------
// Arrow export

namespace {

__global__ void realign_bits_kernel(const uint8_t *src, int64_t off, int64_t n, uint8_t *dst) {
    const int64_t nbytes = (n + 7) / 8;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nbytes;
         i += (int64_t)gridDim.x * blockDim.x) {
        uint8_t v = 0;
        for (int k = 0; k < 8; k++) {
            const int64_t r = i * 8 + k;
            if (r < n && bit_get(src, off, r)) v |= (uint8_t)(1u << k);
        }
        dst[i] = v;
    }
}

struct SchemaPriv {
    std::vector<std::string> formats, names;
    std::vector<ArrowSchema> child_storage;
    std::vector<ArrowSchema *> children;
};

void release_schema(ArrowSchema *s) {
    if (!s || !s->release) return;
    delete static_cast<SchemaPriv *>(s->private_data);
    s->release = nullptr;
}
void release_child_schema(ArrowSchema *s) { s->release = nullptr; }

struct HostArrayPriv {
    std::vector<std::vector<uint8_t>> bufs;
    std::vector<std::vector<const void *>> child_bufs;
    std::vector<ArrowArray> child_storage;
    std::vector<ArrowArray *> children;
    std::vector<const void *> top_bufs;
};
void release_host_array(ArrowArray *a) {
    if (!a || !a->release) return;
    delete static_cast<HostArrayPriv *>(a->private_data);
    a->release = nullptr;
}
void release_child_array(ArrowArray *a) { a->release = nullptr; }

struct DevArrayPriv {
    std::vector<std::shared_ptr<DBuf>> hold;
    std::vector<std::vector<const void *>> child_bufs;
    std::vector<ArrowArray> child_storage;
    std::vector<ArrowArray *> children;
    std::vector<const void *> top_bufs;
};
void release_dev_array(ArrowArray *a) {
    if (!a || !a->release) return;
    delete static_cast<DevArrayPriv *>(a->private_data);
    a->release = nullptr;
}

}  // namespace

void export_schema(const DevBatch &b, ArrowSchema *out) {
    auto *p = new SchemaPriv();
    const size_t n = b.cols.size();
    p->formats.reserve(n);
    p->names.reserve(n + 1);
    p->child_storage.resize(n);
    p->children.resize(n);
    for (size_t i = 0; i < n; i++) {
        p->formats.push_back(b.cols[i].type.format());
        p->names.push_back(b.cols[i].name);
    }
    for (size_t i = 0; i < n; i++) {
        ArrowSchema &c = p->child_storage[i];
        std::memset(&c, 0, sizeof(c));
        c.format = p->formats[i].c_str();
        c.name = p->names[i].c_str();
        c.flags = b.cols[i].nullable ? ARROW_FLAG_NULLABLE : 0;
        c.release = release_child_schema;
        p->children[i] = &c;
    }
    std::memset(out, 0, sizeof(*out));
    out->format = "+s";
    out->name = "";
    out->n_children = (int64_t)n;
    out->children = n ? p->children.data() : nullptr;
    out->release = release_schema;
    out->private_data = p;
}

// A column's validity as a bitmap starting at bit 0 (copied if needed), or
// null when the column has no NULLs bitmap.
static std::shared_ptr<DBuf> aligned_validity(Runtime *rt, const DevCol &c) {
    if (!c.valid) return nullptr;
    if (c.valid_off == 0 && c.hold_valid) return c.hold_valid;
    auto buf = std::make_shared<DBuf>(rt, (size_t)ceil_div(c.length > 0 ? c.length : 1, 8) + 8);
    realign_bits_kernel<<<grid_for(rt, ceil_div(c.length, 8), 256), 256, 0, rt->stream>>>(
        c.valid, c.valid_off, c.length, buf->as<uint8_t>());
    rt->launches++;
    check_launch("realign_bits_kernel");
    return buf;
}

void export_host(Runtime *rt, const DevBatch &b, ArrowArray *out, ArrowSchema *out_schema) {
    const size_t n = b.cols.size();
    auto *p = new HostArrayPriv();
    p->bufs.reserve(2 * n);
    p->child_bufs.resize(n);
    p->child_storage.resize(n);
    p->children.resize(n);
    std::vector<std::shared_ptr<DBuf>> keep;
    for (size_t i = 0; i < n; i++) {
        const DevCol &c = b.cols[i];
        const size_t bytes = c.type.id == Type::Bool ? (size_t)ceil_div(b.rows, 8)
                             : c.type.var()          ? (size_t)(b.rows + 1) * 4
                                                     : (size_t)b.rows * c.type.width();
        p->bufs.emplace_back(bytes + 64);
        std::vector<uint8_t> &data = p->bufs.back();
        if (bytes) KRV_CUDA(cudaMemcpyAsync(data.data(), c.data, bytes, cudaMemcpyDeviceToHost, rt->stream));
        const uint8_t *bptr = nullptr;
        if (c.type.var()) {
            // the offsets first: they say which bytes to copy; rebased to 0
            KRV_CUDA(cudaStreamSynchronize(rt->stream));
            int32_t *offs = reinterpret_cast<int32_t *>(data.data());
            const int32_t o0 = offs[0], on = offs[b.rows];
            for (int64_t r = 0; r <= b.rows; r++) offs[r] -= o0;
            p->bufs.emplace_back((size_t)(on - o0) + 64);
            if (on > o0)
                KRV_CUDA(cudaMemcpyAsync(p->bufs.back().data(), static_cast<const uint8_t *>(c.bytes) + o0,
                                         (size_t)(on - o0), cudaMemcpyDeviceToHost, rt->stream));
            bptr = p->bufs.back().data();
        }
        const uint8_t *vptr = nullptr;
        auto v = aligned_validity(rt, c);
        if (v) {
            keep.push_back(v);
            const size_t vb = (size_t)ceil_div(b.rows, 8);
            p->bufs.emplace_back(vb + 64);
            if (vb) KRV_CUDA(cudaMemcpyAsync(p->bufs.back().data(), v->get(), vb, cudaMemcpyDeviceToHost, rt->stream));
            vptr = p->bufs.back().data();
        }
        p->child_bufs[i] = {vptr, data.data()};
        if (c.type.var()) p->child_bufs[i].push_back(bptr);
    }
    KRV_CUDA(cudaStreamSynchronize(rt->stream));
    for (size_t i = 0; i < n; i++) {
        ArrowArray &a = p->child_storage[i];
        std::memset(&a, 0, sizeof(a));
        a.length = b.rows;
        // With a bitmap the count is left to the consumer (-1: unknown).
        a.null_count = p->child_bufs[i][0] ? -1 : 0;
        a.n_buffers = (int64_t)p->child_bufs[i].size();
        a.buffers = p->child_bufs[i].data();
        a.release = release_child_array;
        p->children[i] = &a;
    }
    p->top_bufs = {nullptr};
    std::memset(out, 0, sizeof(*out));
    out->length = b.rows;
    out->n_buffers = 1;
    out->buffers = p->top_bufs.data();
    out->n_children = (int64_t)n;
    out->children = n ? p->children.data() : nullptr;
    out->release = release_host_array;
    out->private_data = p;
    if (out_schema) export_schema(b, out_schema);
}

void export_device(Runtime *rt, const DevBatch &b, ArrowDeviceArray *out, ArrowSchema *out_schema) {
    const size_t n = b.cols.size();
    auto *p = new DevArrayPriv();
    p->child_bufs.resize(n);
    p->child_storage.resize(n);
    p->children.resize(n);
    for (size_t i = 0; i < n; i++) {
        const DevCol &c = b.cols[i];
        if (c.hold_data) p->hold.push_back(c.hold_data);
        if (c.hold_bytes) p->hold.push_back(c.hold_bytes);
        auto v = aligned_validity(rt, c);
        if (v) p->hold.push_back(v);
        p->child_bufs[i] = {v ? v->get() : nullptr, c.data};
        if (c.type.var()) p->child_bufs[i].push_back(c.bytes);
    }
    for (size_t i = 0; i < n; i++) {
        ArrowArray &a = p->child_storage[i];
        std::memset(&a, 0, sizeof(a));
        a.length = b.rows;
        a.null_count = p->child_bufs[i][0] ? -1 : 0;  // unknown without a device pass
        a.n_buffers = (int64_t)p->child_bufs[i].size();
        a.buffers = p->child_bufs[i].data();
        a.release = release_child_array;
        p->children[i] = &a;
    }
    p->top_bufs = {nullptr};
    std::memset(out, 0, sizeof(*out));
    out->array.length = b.rows;
    out->array.n_buffers = 1;
    out->array.buffers = p->top_bufs.data();
    out->array.n_children = (int64_t)n;
    out->array.children = n ? p->children.data() : nullptr;
    out->array.release = release_dev_array;
    out->array.private_data = p;
    out->device_id = rt->device;
    out->device_type = ARROW_DEVICE_CUDA;
    out->sync_event = nullptr;
    // The buffers are complete once the runtime's stream reaches this point;
    // a consumer on another stream synchronizes with the runtime first.
    if (out_schema) export_schema(b, out_schema);
}

}  // namespace krv
