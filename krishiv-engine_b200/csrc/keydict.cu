// keydict.cu -- dense codes for composite group keys.
//
// Reference: a grouped aggregate keys its row tables by the row hash g of
// all group-by columns and compares the encoded key rows
// (crates/krishiv-exec/src/aggregate/rowtable.rs:816-1185, rowtable/probe.rs:8-214;
// key rows from rows/layout.rs:487-555, strings as 16-byte views plus a heap,
// :24-31, :906-1030). Here: a group key of up to eight columns (int32/int64/
// date32/decimal/float64 values, UTF-8 strings and binary) is mapped to a
// dense int64 code by one open-addressing table in HBM, and the aggregate
// runs on that code with its single-key kernels (a join with string or
// binary keys likewise: the build side inserts, the probe side looks up). The table keeps each code's
// key (fixed-width values by column, strings in a byte heap) and 64-bit
// hash. NULL is a key value of its own (GROUP BY puts NULLs in one group);
// float keys compare after normalisation (-0.0 is 0.0, one NaN), as the
// reference's key encoder does (rows/layout.rs:1147-1153). Which codes the
// groups get does not change any result: codes only name groups.
#include <algorithm>
#include <string>
#include <vector>

#include "krv_device.cuh"
#include "ops.h"

namespace krv {

namespace {

constexpr uint32_t kDictPending = 0xFFFFFFFFu;  // slot claimed, code not yet published
constexpr uint32_t kDictDead = 0xFFFFFFFEu;     // claimed past the code capacity (never read as a code)

struct DictKeyIn {
    const void *data;      // values, or int32 offsets (strings)
    const uint8_t *bytes;  // strings: value bytes
    const uint8_t *valid;
    int64_t voff;
    int32_t width;  // 4, 8 or 16; 0: string
    int32_t is_float;
};
struct DictStore {
    void *vals;         // fixed width: width bytes per code
    uint8_t *valid;     // 1 byte per code
    long long *str_off; // strings: heap offset per code
    int32_t *str_len;   // strings: length per code
};
struct DictDev {
    DictKeyIn in[KRV_MAX_GROUP_KEYS];
    DictStore st[KRV_MAX_GROUP_KEYS];
    int32_t n;
    unsigned long long *slots;
    uint64_t mask;
    unsigned long long *hashes;  // per code
    unsigned long long *ncodes;
    unsigned long long code_cap;
    uint8_t *heap;
    unsigned long long *heap_used;
    unsigned long long heap_cap;
    uint32_t *status;
};

__device__ __forceinline__ uint64_t load_le(const uint8_t *p, int n) {
    uint64_t w = 0;
    for (int k = 0; k < n; k++) w |= (uint64_t)p[k] << (8 * k);
    return w;
}

__device__ __forceinline__ void fixed_words(const DictKeyIn &c, int64_t i, uint64_t &w0, uint64_t &w1) {
    w1 = 0;
    if (c.width == 4) {
        w0 = static_cast<const uint32_t *>(c.data)[i];
    } else if (c.width == 8) {
        w0 = static_cast<const uint64_t *>(c.data)[i];
        if (c.is_float) w0 = normalize_f64_bits(w0);
    } else {
        const uint64_t *p = static_cast<const uint64_t *>(c.data) + 2 * i;
        w0 = p[0];
        w1 = p[1];
    }
}

// The composite key's hash: each column's words mixed in turn (a NULL mixes
// a constant, a string its length and then its bytes 8 at a time).
__device__ uint64_t dict_hash(const DictDev &D, int64_t i) {
    uint64_t h = 0;
    for (int c = 0; c < D.n; c++) {
        const DictKeyIn &K = D.in[c];
        if (!bit_get(K.valid, K.voff, i)) {
            h = mix(h, kNullHash);
            continue;
        }
        if (K.width == 0) {
            const int32_t *offs = static_cast<const int32_t *>(K.data);
            const int32_t o = offs[i], len = offs[i + 1] - o;
            h = mix(h, (uint64_t)(uint32_t)len);
            for (int32_t k = 0; k < len; k += 8) h = mix(h, load_le(K.bytes + o + k, min(8, len - k)));
        } else {
            uint64_t w0, w1;
            fixed_words(K, i, w0, w1);
            h = mix(h, w0);
            if (K.width == 16) h = mix(h, w1);
        }
    }
    return fold(h, kFinish);
}

// Row i's key equals code `code`'s stored key. The stored keys are read
// through L2 (ld.global.cg): they were written by another thread after this
// SM may have cached their neighbours.
__device__ bool dict_eq(const DictDev &D, int64_t i, uint64_t code) {
    for (int c = 0; c < D.n; c++) {
        const DictKeyIn &K = D.in[c];
        const DictStore &S = D.st[c];
        const bool v = bit_get(K.valid, K.voff, i);
        if (v != (__ldcg(S.valid + code) != 0)) return false;
        if (!v) continue;
        if (K.width == 0) {
            const int32_t *offs = static_cast<const int32_t *>(K.data);
            const int32_t o = offs[i], len = offs[i + 1] - o;
            if (len != __ldcg(S.str_len + code)) return false;
            const uint8_t *a = K.bytes + o;
            const uint8_t *b = D.heap + __ldcg(S.str_off + code);
            for (int32_t k = 0; k < len; k++)
                if (a[k] != __ldcg(b + k)) return false;
        } else {
            uint64_t w0, w1, s0, s1 = 0;
            fixed_words(K, i, w0, w1);
            if (K.width == 4) {
                s0 = __ldcg(static_cast<const uint32_t *>(S.vals) + code);
            } else if (K.width == 8) {
                s0 = __ldcg(static_cast<const unsigned long long *>(S.vals) + code);
            } else {
                s0 = __ldcg(static_cast<const unsigned long long *>(S.vals) + 2 * code);
                s1 = __ldcg(static_cast<const unsigned long long *>(S.vals) + 2 * code + 1);
            }
            if (w0 != s0 || w1 != s1) return false;
        }
    }
    return true;
}

__device__ void dict_store(const DictDev &D, int64_t i, uint64_t code) {
    for (int c = 0; c < D.n; c++) {
        const DictKeyIn &K = D.in[c];
        const DictStore &S = D.st[c];
        const bool v = bit_get(K.valid, K.voff, i);
        S.valid[code] = v ? 1 : 0;
        if (K.width == 0) {
            int32_t len = 0;
            unsigned long long at = 0;
            if (v) {
                const int32_t *offs = static_cast<const int32_t *>(K.data);
                const int32_t o = offs[i];
                len = offs[i + 1] - o;
                at = atomicAdd(D.heap_used, (unsigned long long)len);
                if (at + (unsigned long long)len <= D.heap_cap) {
                    for (int32_t k = 0; k < len; k++) D.heap[at + k] = K.bytes[o + k];
                } else {
                    atomicOr(D.status, ST_CAPACITY);
                    len = 0;
                    at = 0;
                }
            }
            S.str_off[code] = (long long)at;
            S.str_len[code] = len;
        } else {
            uint64_t w0 = 0, w1 = 0;
            if (v) fixed_words(K, i, w0, w1);
            if (K.width == 4) {
                static_cast<uint32_t *>(S.vals)[code] = (uint32_t)w0;
            } else if (K.width == 8) {
                static_cast<unsigned long long *>(S.vals)[code] = w0;
            } else {
                static_cast<unsigned long long *>(S.vals)[2 * code] = w0;
                static_cast<unsigned long long *>(S.vals)[2 * code + 1] = w1;
            }
        }
    }
}

// The code of every row's key: found, or (insert) claimed in the table and
// given the next dense code; -1 for a key not in the table (lookup only) or
// past the capacities the host sized (status bits say which).
__global__ void __launch_bounds__(256) dict_encode_kernel(DictDev D, int64_t n, int insert, long long *codes) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t h = dict_hash(D, i);
        const unsigned long long tag = h >> 32;
        uint64_t pos = h & D.mask;
        long long code = -1;
        for (uint64_t probes = 0; probes <= D.mask; probes++) {
            unsigned long long s = *reinterpret_cast<volatile unsigned long long *>(D.slots + pos);
            if (s == 0) {
                if (!insert) break;
                const unsigned long long mine = (tag << 32) | kDictPending;
                const unsigned long long old = atomicCAS(D.slots + pos, 0ull, mine);
                if (old == 0) {
                    const unsigned long long c = atomicAdd(D.ncodes, 1ull);
                    if (c >= D.code_cap) {
                        atomicOr(D.status, ST_CAPACITY);
                        atomicExch(D.slots + pos, (tag << 32) | kDictDead);
                        break;
                    }
                    dict_store(D, i, c);
                    D.hashes[c] = h;
                    __threadfence();
                    atomicExch(D.slots + pos, (tag << 32) | (c + 1));
                    code = (long long)c;
                    break;
                }
                s = old;
            }
            if ((s >> 32) == tag) {
                uint32_t lo = (uint32_t)s;
                if (lo == kDictPending) {
                    int it = 0;
                    for (; it < (1 << 22) && lo == kDictPending; it++) {
                        __nanosleep(32);
                        lo = (uint32_t)*reinterpret_cast<volatile unsigned long long *>(D.slots + pos);
                    }
                    if (lo == kDictPending) {
                        atomicOr(D.status, ST_TIMEOUT);
                        break;
                    }
                    __threadfence();
                }
                if (lo != kDictDead && dict_eq(D, i, lo - 1)) {
                    code = (long long)(lo - 1);
                    break;
                }
            }
            pos = (pos + 1) & D.mask;
        }
        codes[i] = code;
    }
}

// Re-inserts codes [0, n) into an empty table by their stored hashes.
__global__ void dict_rehash_kernel(const unsigned long long *hashes, uint64_t n, unsigned long long *slots,
                                   uint64_t mask) {
    for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < n; c += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t h = hashes[c];
        uint64_t pos = h & mask;
        for (uint64_t probes = 0; probes <= mask; probes++) {
            if (atomicCAS(slots + pos, 0ull, ((h >> 32) << 32) | (c + 1)) == 0) break;
            pos = (pos + 1) & mask;
        }
    }
}

// Output column k for codes[0, n): fixed-width values and validity bits.
__global__ void dict_gather_fixed_kernel(const long long *codes, int64_t n, const void *vals, const uint8_t *valid,
                                         int width, void *out, uint32_t *out_valid) {
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
        const long long c = codes[j];
        if (width == 4) static_cast<uint32_t *>(out)[j] = static_cast<const uint32_t *>(vals)[c];
        else if (width == 8) static_cast<unsigned long long *>(out)[j] = static_cast<const unsigned long long *>(vals)[c];
        else static_cast<uint4 *>(out)[j] = static_cast<const uint4 *>(vals)[c];
        if (out_valid && valid[c]) atomicOr(out_valid + (j >> 5), 1u << (j & 31));
    }
}

__global__ void dict_gather_len_kernel(const long long *codes, int64_t n, const int32_t *lens, const uint8_t *valid,
                                       int32_t *out_len, uint32_t *out_valid) {
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
        const long long c = codes[j];
        out_len[j] = valid[c] ? lens[c] : 0;
        if (out_valid && valid[c]) atomicOr(out_valid + (j >> 5), 1u << (j & 31));
    }
}

// One warp per output string: its bytes from the heap.
__global__ void dict_gather_bytes_kernel(const long long *codes, int64_t n, const long long *str_off,
                                         const int32_t *offsets, const uint8_t *heap, uint8_t *out) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x / 32);
    for (int64_t j = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / 32; j < n; j += warps) {
        const int32_t o = offsets[j], len = offsets[j + 1] - o;
        const uint8_t *src = heap + str_off[codes[j]];
        for (int32_t k = lane; k < len; k += 32) out[o + k] = src[k];
    }
}

}  // namespace

// ---- the dictionary ----------------------------------------------------------------
class KeyDict {
  public:
    KeyDict(Runtime *rt, const std::vector<DevCol> &meta) : rt_(rt), meta_(meta) {
        if (meta_.empty() || meta_.size() > (size_t)KRV_MAX_GROUP_KEYS)
            fail(KRV_INVALID_ARGUMENT, "group keys: 1 to 8 columns");
        for (const DevCol &m : meta_) {
            const Type t = m.type.id;
            if (!(t == Type::I32 || t == Type::I64 || t == Type::Date32 || t == Type::Dec64 || t == Type::Dec128 ||
                  t == Type::F64 || t == Type::Utf8 || t == Type::Binary))
                fail(KRV_UNSUPPORTED, "group key of type " + m.type.format());
        }
        store_.resize(meta_.size());
        ncodes_ = DBuf(rt_, 8);
        heap_used_ = DBuf(rt_, 8);
        KRV_CUDA(cudaMemsetAsync(ncodes_.get(), 0, 8, rt_->stream));
        KRV_CUDA(cudaMemsetAsync(heap_used_.get(), 0, 8, rt_->stream));
    }

    int64_t size() const { return count_; }
    // Device views of column 0's stored strings (valid until the next encode).
    void strings(const long long **off, const int32_t **len, const uint8_t **heap) const {
        *off = store_[0].str_off.as<long long>();
        *len = store_[0].str_len.as<int32_t>();
        *heap = heap_.as<uint8_t>();
    }

    // The int64 code of each row's key (columns `cols` of b); unseen keys get
    // new codes (insert) or -1 (lookup only).
    DBuf encode(const DevBatch &b, const std::vector<int> &cols, bool insert = true) {
        const int64_t n = b.rows;
        if (cols.size() != meta_.size()) fail(KRV_INTERNAL, "key dictionary: column count");
        for (size_t k = 0; k < cols.size(); k++)
            if (b.cols[cols[k]].type != meta_[k].type) fail(KRV_INVALID_ARGUMENT, "key columns differ in types");
        DBuf codes(rt_, (size_t)std::max<int64_t>(n, 1) * 8);
        if (n == 0) return codes;
        if (!insert) {
            if (slot_count_ == 0) {
                KRV_CUDA(cudaMemsetAsync(codes.get(), 0xFF, (size_t)n * 8, rt_->stream));
                return codes;
            }
            DictDev D = dev(b, cols);
            clear_status(rt_);
            dict_encode_kernel<<<grid_for(rt_, n, 256, 8), 256, 0, rt_->stream>>>(D, n, 0, codes.as<long long>());
            rt_->launches++;
            check_launch("dict_encode_kernel");
            if (take_status(rt_) & ST_TIMEOUT) fail(KRV_TIMEOUT, "group keys: a wait for a code gave up");
            return codes;
        }
        int64_t heap_need = 0;
        for (int c : cols) {
            const DevCol &col = b.cols[c];
            if (!col.type.var()) continue;
            if (col.var_bytes >= 0) {
                heap_need += col.var_bytes;
            } else {
                int32_t ends[2];
                read_device(rt_, col.data, 4, &ends[0]);
                read_device(rt_, static_cast<const int32_t *>(col.data) + n, 4, &ends[1]);
                heap_need += std::max<int32_t>(0, ends[1] - ends[0]);
            }
        }
        reserve(count_ + n, heap_used_host_ + heap_need);
        DictDev D = dev(b, cols);
        clear_status(rt_);
        dict_encode_kernel<<<grid_for(rt_, n, 256, 8), 256, 0, rt_->stream>>>(D, n, 1, codes.as<long long>());
        rt_->launches++;
        check_launch("dict_encode_kernel");
        unsigned long long got[2];
        read_device(rt_, ncodes_.get(), 8, &got[0]);
        read_device(rt_, heap_used_.get(), 8, &got[1]);
        const uint32_t st = take_status(rt_);
        if (st & ST_TIMEOUT) fail(KRV_TIMEOUT, "group keys: a wait for a code gave up");
        if (st & ST_CAPACITY) fail(KRV_INTERNAL, "group keys: capacity exceeded");
        count_ = (int64_t)got[0];
        heap_used_host_ = (int64_t)got[1];
        return codes;
    }

    // The key columns of codes[0, n) (device int64 codes), named and typed as
    // the group-by columns.
    std::vector<DevCol> decode(const long long *codes, int64_t n) {
        std::vector<DevCol> out;
        for (size_t k = 0; k < meta_.size(); k++) {
            const DevCol &m = meta_[k];
            const Store &S = store_[k];
            DevCol col;
            col.type = m.type;
            col.name = m.name;
            col.nullable = m.nullable;
            col.length = n;
            if (m.nullable) {
                col.hold_valid = std::make_shared<DBuf>(rt_, (size_t)ceil_div(std::max<int64_t>(n, 1), 32) * 4 + 8);
                KRV_CUDA(cudaMemsetAsync(col.hold_valid->get(), 0, col.hold_valid->bytes(), rt_->stream));
                col.valid = col.hold_valid->as<uint8_t>();
            }
            uint32_t *ov = m.nullable ? col.hold_valid->as<uint32_t>() : nullptr;
            if (!m.type.var()) {
                const int w = m.type.width();
                col.hold_data = std::make_shared<DBuf>(rt_, (size_t)std::max<int64_t>(n, 1) * w);
                col.data = col.hold_data->get();
                if (n > 0) {
                    dict_gather_fixed_kernel<<<grid_for(rt_, n, 256, 8), 256, 0, rt_->stream>>>(
                        codes, n, S.vals.get(), S.valid.as<uint8_t>(), w, col.hold_data->get(), ov);
                    rt_->launches++;
                    check_launch("dict_gather_fixed_kernel");
                }
            } else {
                // lengths on the device, offsets by a scan on the host, then the bytes
                DBuf lens(rt_, (size_t)std::max<int64_t>(n, 1) * 4);
                if (n > 0) {
                    dict_gather_len_kernel<<<grid_for(rt_, n, 256, 8), 256, 0, rt_->stream>>>(
                        codes, n, S.str_len.as<int32_t>(), S.valid.as<uint8_t>(), lens.as<int32_t>(), ov);
                    rt_->launches++;
                    check_launch("dict_gather_len_kernel");
                }
                std::vector<int32_t> hl((size_t)n), ho((size_t)n + 1);
                if (n > 0) {
                    KRV_CUDA(cudaMemcpyAsync(hl.data(), lens.get(), (size_t)n * 4, cudaMemcpyDeviceToHost, rt_->stream));
                    KRV_CUDA(cudaStreamSynchronize(rt_->stream));
                }
                int64_t acc = 0;
                for (int64_t j = 0; j < n; j++) {
                    ho[(size_t)j] = (int32_t)acc;
                    acc += hl[(size_t)j];
                    if (acc > 0x7FFFFFFFll) fail(KRV_UNSUPPORTED, "group key strings of 2 GiB or more in one output");
                }
                ho[(size_t)n] = (int32_t)acc;
                col.hold_data = std::make_shared<DBuf>(rt_, ho.size() * 4);
                KRV_CUDA(cudaMemcpyAsync(col.hold_data->get(), ho.data(), ho.size() * 4, cudaMemcpyHostToDevice,
                                         rt_->stream));
                col.hold_bytes = std::make_shared<DBuf>(rt_, (size_t)std::max<int64_t>(acc, 1));
                if (acc > 0) {
                    dict_gather_bytes_kernel<<<grid_for(rt_, n * 32, 256, 8), 256, 0, rt_->stream>>>(
                        codes, n, S.str_off.as<long long>(), col.hold_data->as<int32_t>(), heap_.as<uint8_t>(),
                        col.hold_bytes->as<uint8_t>());
                    rt_->launches++;
                    check_launch("dict_gather_bytes_kernel");
                }
                KRV_CUDA(cudaStreamSynchronize(rt_->stream));  // `ho` is read by the copy
                col.data = col.hold_data->get();
                col.bytes = col.hold_bytes->get();
                col.var_bytes = acc;
            }
            out.push_back(std::move(col));
        }
        return out;
    }

  private:
    struct Store {
        DBuf vals, valid, str_off, str_len;
    };

    DictDev dev(const DevBatch &b, const std::vector<int> &cols) {
        DictDev D{};
        D.n = (int32_t)meta_.size();
        for (size_t k = 0; k < meta_.size(); k++) {
            const DevCol &c = b.cols[cols[k]];
            DictKeyIn &K = D.in[k];
            K.data = c.data;
            K.bytes = static_cast<const uint8_t *>(c.bytes);
            K.valid = c.valid;
            K.voff = c.valid_off;
            K.width = c.type.var() ? 0 : c.type.width();
            K.is_float = c.type.id == Type::F64;
            const Store &S = store_[k];
            D.st[k] = DictStore{S.vals.get(), S.valid.as<uint8_t>(), S.str_off.as<long long>(), S.str_len.as<int32_t>()};
        }
        D.slots = slots_.as<unsigned long long>();
        D.mask = slot_count_ - 1;
        D.hashes = hashes_.as<unsigned long long>();
        D.ncodes = ncodes_.as<unsigned long long>();
        D.code_cap = (unsigned long long)code_cap_;
        D.heap = heap_.as<uint8_t>();
        D.heap_used = heap_used_.as<unsigned long long>();
        D.heap_cap = (unsigned long long)heap_cap_;
        D.status = status_word(rt_);
        return D;
    }

    // Room for `codes` codes (the table at most half full) and `heap` bytes of
    // strings; what is kept moves to the larger buffers.
    void reserve(int64_t codes, int64_t heap) {
        if (codes > code_cap_) {
            const int64_t cap = std::max<int64_t>({codes, code_cap_ * 2, 1024});
            for (size_t k = 0; k < meta_.size(); k++) {
                Store &S = store_[k];
                const DType t = meta_[k].type;
                Store N;
                N.valid = DBuf(rt_, (size_t)cap);
                if (t.var()) {
                    N.str_off = DBuf(rt_, (size_t)cap * 8);
                    N.str_len = DBuf(rt_, (size_t)cap * 4);
                } else {
                    N.vals = DBuf(rt_, (size_t)cap * t.width());
                }
                if (count_ > 0) {
                    copy(N.valid, S.valid, (size_t)count_);
                    if (t.var()) {
                        copy(N.str_off, S.str_off, (size_t)count_ * 8);
                        copy(N.str_len, S.str_len, (size_t)count_ * 4);
                    } else {
                        copy(N.vals, S.vals, (size_t)count_ * t.width());
                    }
                }
                S = std::move(N);
            }
            DBuf h(rt_, (size_t)cap * 8);
            if (count_ > 0) copy(h, hashes_, (size_t)count_ * 8);
            hashes_ = std::move(h);
            code_cap_ = cap;
        }
        if ((uint64_t)codes * 2 > slot_count_) {
            uint64_t slots = 1024;
            while (slots < (uint64_t)codes * 2) slots <<= 1;
            slots_ = DBuf(rt_, slots * 8);
            KRV_CUDA(cudaMemsetAsync(slots_.get(), 0, slots * 8, rt_->stream));
            slot_count_ = slots;
            if (count_ > 0) {
                dict_rehash_kernel<<<grid_for(rt_, count_, 256, 8), 256, 0, rt_->stream>>>(
                    hashes_.as<unsigned long long>(), (uint64_t)count_, slots_.as<unsigned long long>(), slots - 1);
                rt_->launches++;
                check_launch("dict_rehash_kernel");
            }
        }
        if (heap > heap_cap_) {
            const int64_t cap = std::max<int64_t>({heap, heap_cap_ * 2, 4096});
            DBuf nh(rt_, (size_t)cap);
            if (heap_used_host_ > 0) copy(nh, heap_, (size_t)heap_used_host_);
            heap_ = std::move(nh);
            heap_cap_ = cap;
        }
        if (!heap_.get()) {
            heap_ = DBuf(rt_, 4096);
            heap_cap_ = 4096;
        }
    }

    void copy(DBuf &dst, const DBuf &src, size_t bytes) {
        if (bytes) KRV_CUDA(cudaMemcpyAsync(dst.get(), src.get(), bytes, cudaMemcpyDeviceToDevice, rt_->stream));
    }

    Runtime *rt_;
    std::vector<DevCol> meta_;
    std::vector<Store> store_;
    DBuf slots_, hashes_, ncodes_, heap_, heap_used_;
    uint64_t slot_count_ = 0;
    int64_t code_cap_ = 0, heap_cap_ = 0;
    int64_t count_ = 0, heap_used_host_ = 0;
};

KeyDict *make_key_dict(Runtime *rt, const std::vector<DevCol> &meta) { return new KeyDict(rt, meta); }
void key_dict_destroy(KeyDict *d) { delete d; }
DBuf key_dict_encode(KeyDict *d, const DevBatch &b, const std::vector<int> &cols, bool insert) {
    return d->encode(b, cols, insert);
}
std::vector<DevCol> key_dict_decode(KeyDict *d, const long long *codes, int64_t n) { return d->decode(codes, n); }
int64_t key_dict_size(const KeyDict *d) { return d->size(); }
void key_dict_strings(const KeyDict *d, const long long **off, const int32_t **len, const uint8_t **heap) {
    d->strings(off, len, heap);
}

}  // namespace krv
