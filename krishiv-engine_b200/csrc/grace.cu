// grace.cu -- the partitioned ("grace") hash join: inner and left outer joins
// on one int64 key whose build side, with its hash tables, does not fit the
// device memory budget.
//
// Reference: the engine's grace join (crates/krishiv-exec/src/join/grace.rs:
// step :828, split :1397, scatter :1481) partitions both sides by the key
// hash, spills partitions to disk and joins them one at a time, splitting a
// partition that is still too large with the next level of hash bits. Here:
//  - a radix partition pass (histogram, then a scatter staged in shared
//    memory so that each partition's rows leave a tile as one contiguous,
//    coalesced run) splits every batch into 2^radix partitions by the top
//    `radix` bits of the row hash h (level 0, join/keys.rs:118-128); a split
//    of a partition uses bits [48-3d, 51-3d) of g = fin(h ^ seed) (level d,
//    hash.rs:139-148), 8 ways;
//  - hybrid residency: partitions are joined in HBM while the build's
//    estimated footprint (rows, table and chains) fits half of the runtime's
//    HBM budget; the others spill to page-locked host memory;
//  - every partition is joined by a HashJoin (the same table, probe and
//    output code as the unpartitioned join), so the output rows are exactly
//    those of the unpartitioned join, in another order;
//  - NULL probe keys never match: their rows are padded at once (left outer)
//    or dropped (inner); NULL build keys are dropped in the partition pass.
// Spilled partitions are joined after the last probe batch, one output batch
// per call, so the output never has to fit the budget.
#include <algorithm>
#include <deque>
#include <memory>
#include <string>
#include <vector>

#include "krv_device.cuh"
#include "ops.h"

namespace krv {

namespace {

constexpr int kPartThreads = 512;
constexpr int kPartTile = 2048;  // rows staged per tile
constexpr int kMaxParts = 64;    // 2^6: the reference clamps radix to 3..6
constexpr int kMaxCols = 8;
constexpr int kMaxLevel = 6;

struct PartCol {
    const void *src;
    void *dst;
    int width;  // 4 or 8
};
struct PartArgs {
    const long long *key;
    const uint8_t *kvalid;
    int64_t kvoff;
    int64_t n;
    int level, bits;
    uint64_t seed;
    int nparts;      // partitions; bucket `nparts` holds NULL keys, `nparts + 1` filtered rows
    int keep_nulls;  // write the NULL bucket (probe side) or drop it (build side)
    int keep_filtered;  // write the filtered bucket (left outer) or drop it (inner)
    int filter_mode;    // kFilterNone, kFilterInsert (build side) or kFilterTest (probe side)
    uint32_t *bloom;    // blocked Bloom filter over h: 8 words (one 32-byte block) per key
    uint64_t bloom_blocks;
    uint8_t *bucket;    // with kFilterTest: each row's bucket, written by the histogram pass for the scatter
    PartCol c[kMaxCols];
    int ncols;
};
constexpr int kFilterNone = 0, kFilterInsert = 1, kFilterTest = 2;

// The partition of row r and its key hash h. With kFilterTest, a row whose
// key the build side's Bloom filter rules out goes to bucket nparts + 1.
__device__ __forceinline__ int part_of(const PartArgs &A, int64_t r, uint64_t &h) {
    h = 0;
    if (A.kvalid && !bit_get(A.kvalid, A.kvoff, r)) return A.nparts;
    h = hash_word((uint64_t)A.key[r]);
    if (A.filter_mode == kFilterTest &&
        !sbbf_check_words(A.bloom + 8 * sbbf_block(h, A.bloom_blocks), (uint32_t)h))
        return A.nparts + 1;
    if (A.level == 0) return (int)(h >> (64 - A.bits));
    return (int)((finalize(h, A.seed) >> (48 - 3 * A.level)) & 7u);
}

__global__ void __launch_bounds__(256) part_hist_kernel(PartArgs A, unsigned long long *hist) {
    __shared__ unsigned int s_hist[kMaxParts + 2];
    for (int p = threadIdx.x; p <= A.nparts + 1; p += blockDim.x) s_hist[p] = 0;
    __syncthreads();
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < A.n; r += (int64_t)gridDim.x * blockDim.x) {
        uint64_t h;
        const int p = part_of(A, r, h);
        atomicAdd(&s_hist[p], 1u);
        if (A.bucket) A.bucket[r] = (uint8_t)p;  // the scatter reads it: no second hash or filter lookup
    }
    __syncthreads();
    for (int p = threadIdx.x; p <= A.nparts + 1; p += blockDim.x)
        if (s_hist[p]) atomicAdd(hist + p, (unsigned long long)s_hist[p]);
}

// Tiles of kPartTile rows: rank every row within its partition in shared
// memory, claim each partition's run of the output with one atomic per tile,
// then write the tile column by column in partition order (coalesced runs).
//
// With kFilterInsert every non-NULL key also goes into the Bloom filter (one
// 32-byte block per key: 8 lanes of a warp set one word each), so that the
// filter is complete when the build side's partition passes end.
__global__ void __launch_bounds__(kPartThreads) part_scatter_kernel(PartArgs A, unsigned long long *cursor) {
    __shared__ unsigned int s_cnt[kMaxParts + 2], s_off[kMaxParts + 3];
    __shared__ unsigned long long s_base[kMaxParts + 2];
    __shared__ uint8_t s_part[kPartTile];
    __shared__ __align__(16) unsigned long long s_val[kPartTile];
    constexpr int U = kPartTile / kPartThreads;
    const int64_t ntiles = (A.n + kPartTile - 1) / kPartTile;
    for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int64_t row0 = t * kPartTile;
        for (int p = threadIdx.x; p <= A.nparts + 1; p += kPartThreads) s_cnt[p] = 0;
        __syncthreads();
        int part[U];
        unsigned rank[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int i = u * kPartThreads + threadIdx.x;
            const int64_t r = row0 + i;
            uint64_t h = 0;
            part[u] = r >= A.n ? -1 : A.bucket ? (int)A.bucket[r] : part_of(A, r, h);
            if (A.filter_mode == kFilterInsert) {
                // four keys per round, each key's 8 words set by 8 lanes
                unsigned todo = __ballot_sync(0xFFFFFFFFu, part[u] >= 0 && part[u] < A.nparts);
                const int w = (int)(lane_id() & 7u), q = (int)(lane_id() >> 3);
                while (todo) {
                    unsigned m = todo;
                    for (int j = 0; j < q; j++) m &= m - 1;  // drop the q lowest keys of the round
                    const int src = m ? __ffs(m) - 1 : 0;
                    const uint64_t hs = __shfl_sync(0xFFFFFFFFu, h, src);
                    if (m) atomicOr(A.bloom + 8 * sbbf_block(hs, A.bloom_blocks) + w, sbbf_bit((uint32_t)hs, w));
                    for (int j = 0; j < 4 && todo; j++) todo &= todo - 1;
                }
            }
            if (part[u] == A.nparts && !A.keep_nulls) part[u] = -1;
            if (part[u] == A.nparts + 1 && !A.keep_filtered) part[u] = -1;
            rank[u] = part[u] >= 0 ? atomicAdd(&s_cnt[part[u]], 1u) : 0u;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned acc = 0;
            for (int p = 0; p <= A.nparts + 1; p++) {
                s_off[p] = acc;
                acc += s_cnt[p];
            }
            s_off[A.nparts + 2] = acc;
        }
        for (int p = threadIdx.x; p <= A.nparts + 1; p += kPartThreads)
            s_base[p] = s_cnt[p] ? atomicAdd(cursor + p, (unsigned long long)s_cnt[p]) : 0ull;
        __syncthreads();
#pragma unroll
        for (int u = 0; u < U; u++)
            if (part[u] >= 0) s_part[s_off[part[u]] + rank[u]] = (uint8_t)part[u];
        const unsigned total = s_off[A.nparts + 2];
        for (int c = 0; c < A.ncols; c++) {
            const PartCol C = A.c[c];
#pragma unroll
            for (int u = 0; u < U; u++) {
                if (part[u] < 0) continue;
                const int64_t r = row0 + u * kPartThreads + threadIdx.x;
                const unsigned slot = s_off[part[u]] + rank[u];
                s_val[slot] = C.width == 8 ? static_cast<const unsigned long long *>(C.src)[r]
                                           : (unsigned long long)static_cast<const uint32_t *>(C.src)[r];
            }
            __syncthreads();
            for (unsigned j = threadIdx.x; j < total; j += kPartThreads) {
                const int p = s_part[j];
                const unsigned long long at = s_base[p] + (j - s_off[p]);
                if (C.width == 8) static_cast<unsigned long long *>(C.dst)[at] = s_val[j];
                else static_cast<uint32_t *>(C.dst)[at] = (uint32_t)s_val[j];
            }
            __syncthreads();
        }
    }
}

// ---- the fallback for a partition that splitting cannot shrink ------------------
// Probe row ids of a chunk: base, base + 1, ...
__global__ void iota_kernel(long long *out, int64_t n, long long base) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = base + i;
}
// The probe rows that matched some build row (their ids in an output batch).
__global__ void mark_matched_kernel(const long long *ids, int64_t n, uint8_t *matched) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        matched[ids[i]] = 1;
}
// The rows of a chunk (ids base..) that matched nothing, compacted (any order).
__global__ void compact_unmatched_kernel(PartArgs A, const uint8_t *matched, long long base,
                                         unsigned long long *count) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t b0 = blockIdx.x * (int64_t)blockDim.x; b0 < A.n; b0 += stride) {
        const int64_t r = b0 + threadIdx.x;
        const bool keep = r < A.n && !matched[base + r];
        const unsigned long long at = warp_alloc(count, keep, 0xFFFFFFFFu);
        if (!keep) continue;
        for (int c = 0; c < A.ncols; c++) {
            if (A.c[c].width == 4)
                static_cast<uint32_t *>(A.c[c].dst)[at] = static_cast<const uint32_t *>(A.c[c].src)[r];
            else
                static_cast<uint64_t *>(A.c[c].dst)[at] = static_cast<const uint64_t *>(A.c[c].src)[r];
        }
    }
}

// ---- the resident partitions' probe: one launch per input slice ------------------
// Every resident partition's rows of the slice are probed against that
// partition's table in one launch (tiles of 256 rows, each tile within one
// partition), and all their output rows go to one output batch: no launch,
// output count read or output copy per partition. The table lookups, chain
// walks and output rounds are those of the unpartitioned join's probe
// (pairs: newest build row first, left outer pads unmatched rows). Tiles of
// 64 rows, each within one partition, are taken one per warp, two rows per
// lane with their first lookups in flight together.
constexpr int kGProbeThreads = 256;
constexpr int kGRows = 2;  // probe rows per lane
constexpr int kGMaxOut = 16;
constexpr uint32_t kGNone = 0xFFFFFFFFu;
struct GPartDev {
    const unsigned long long *slots;
    uint64_t mask;
    const uint32_t *next;
    const long long *bkey;
    const void *bcol[kMaxCols];  // the partition's build columns
    int64_t prow0, rows;         // its rows of the partitioned slice
    int64_t tile0;               // its first tile (of 32 x kGRows rows)
};
struct GOutCol {
    void *dst;
    uint32_t *dst_valid;  // zeroed bitmap words, or null
    int32_t width;
    int32_t side;  // 0: probe column `col`, 1: build column `col`
    int32_t col;
};
struct GOutDev {
    GOutCol c[kGMaxOut];
    int32_t n;
    const void *pcol[kMaxCols];  // the partitioned slice's columns
    const long long *pkey;
};

__device__ __forceinline__ void gcopy(void *dst, const void *src, unsigned long long di, int64_t si, int w) {
    if (w == 8) static_cast<unsigned long long *>(dst)[di] = static_cast<const unsigned long long *>(src)[si];
    else static_cast<uint32_t *>(dst)[di] = static_cast<const uint32_t *>(src)[si];
}

__global__ void __launch_bounds__(kGProbeThreads) grace_probe_kernel(const GPartDev *parts, int nparts, int64_t tiles,
                                                                     uint64_t seed, GOutDev out, unsigned long long cap,
                                                                     unsigned long long *count, int pad,
                                                                     int single_match, uint32_t *status) {
    const unsigned lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1u;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    // Tiles of 32 x kGRows rows, one warp each: no block-wide synchronization.
    for (int64_t t = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < tiles; t += nwarps) {
        // the tile's partition: the last one whose first tile is at most t
        int p = 0;
        for (int base = 0; base < nparts; base += 32) {
            const int q = base + (int)lane;
            const unsigned m = __ballot_sync(0xFFFFFFFFu, q < nparts && parts[q].tile0 <= t);
            if (m) p = base + 31 - __clz(m);
        }
        const GPartDev *sp = parts + p;
        const unsigned long long *slots = sp->slots;
        const uint64_t mask = sp->mask;
        const long long *bkey = sp->bkey;
        // kGRows rows per lane: their first slot loads, then their first
        // candidates' key loads, are in flight together
        bool live[kGRows];
        int64_t prow[kGRows];
        long long key[kGRows], bk[kGRows];
        unsigned long long tag[kGRows], sl[kGRows];
        uint64_t pos[kGRows];
        uint32_t cand[kGRows], cur[kGRows];
#pragma unroll
        for (int u = 0; u < kGRows; u++) {
            const int64_t local = (t - sp->tile0) * (32 * kGRows) + u * 32 + lane;
            live[u] = local < sp->rows;
            prow[u] = sp->prow0 + local;
            key[u] = live[u] ? out.pkey[prow[u]] : 0;
            const uint64_t g = finalize(hash_word((uint64_t)key[u]), seed);
            tag[u] = g >> 32;
            pos[u] = g & mask;
        }
#pragma unroll
        for (int u = 0; u < kGRows; u++) sl[u] = live[u] ? __ldg(slots + pos[u]) : 0ull;
#pragma unroll
        for (int u = 0; u < kGRows; u++) {
            cand[u] = (sl[u] != 0 && (sl[u] >> 32) == tag[u]) ? (uint32_t)(sl[u] & 0xFFFFFFFFull) - 1u : kGNone;
            bk[u] = cand[u] != kGNone ? __ldg(bkey + cand[u]) : 0;
        }
#pragma unroll
        for (int u = 0; u < kGRows; u++) {
            cur[u] = kGNone;
            if (!live[u] || sl[u] == 0) continue;  // an empty first slot: no match
            if (cand[u] != kGNone && bk[u] == key[u]) {
                cur[u] = cand[u];
                continue;
            }
            // the rest of the probe sequence, a slot at a time
            uint64_t q = (pos[u] + 1) & mask;
            for (uint64_t probes = 1; probes <= mask; probes++) {
                const unsigned long long s2 = __ldg(slots + q);
                if (s2 == 0) break;
                if ((s2 >> 32) == tag[u]) {
                    const uint32_t o = (uint32_t)(s2 & 0xFFFFFFFFull) - 1u;
                    if (__ldg(bkey + o) == key[u]) {
                        cur[u] = o;
                        break;
                    }
                }
                q = (q + 1) & mask;
            }
        }
        const uint32_t *next = sp->next;
#pragma unroll
        for (int u = 0; u < kGRows; u++) {
            const int64_t pr = prow[u];
            uint32_t c0 = cur[u];
            bool padrow = live[u] && c0 == kGNone && pad;
            unsigned chain = 0;
            while (__any_sync(0xFFFFFFFFu, c0 != kGNone || padrow)) {
                const bool want = c0 != kGNone || padrow;
                const unsigned ballot = __ballot_sync(0xFFFFFFFFu, want);
                unsigned long long first = 0;
                if (lane == 0) first = atomicAdd(count, (unsigned long long)__popc(ballot));
                first = __shfl_sync(0xFFFFFFFFu, first, 0);
                const unsigned rank = __popc(ballot & below);
                const unsigned long long at = first + rank;
                for (int c = 0; c < out.n; c++) {
                    const GOutCol C = out.c[c];
                    bool v = false;
                    if (want && at < cap) {
                        if (C.side == 0) {
                            gcopy(C.dst, out.pcol[C.col], at, pr, C.width);
                            v = true;
                        } else if (c0 != kGNone) {
                            gcopy(C.dst, sp->bcol[C.col], at, c0, C.width);
                            v = true;
                        } else if (C.width == 8) {
                            static_cast<unsigned long long *>(C.dst)[at] = 0ull;
                        } else {
                            static_cast<uint32_t *>(C.dst)[at] = 0u;
                        }
                    }
                    if (C.dst_valid) {
                        // this round's bits in output order, OR-ed in with at most two atomics
                        const unsigned m = __reduce_or_sync(0xFFFFFFFFu, v ? (1u << rank) : 0u);
                        if (lane == 0 && m) {
                            const unsigned long long w = first >> 5;
                            const unsigned sh = (unsigned)(first & 31);
                            const unsigned long long capw = (cap + 31) >> 5;
                            if (w < capw) atomicOr(C.dst_valid + w, m << sh);
                            if (sh && w + 1 < capw && (m >> (32 - sh))) atomicOr(C.dst_valid + w + 1, m >> (32 - sh));
                        }
                    }
                }
                if (c0 != kGNone) {
                    chain++;
                    c0 = next[c0];
                } else {
                    padrow = false;
                }
            }
            if (single_match && chain > 1) atomicOr(status, ST_TOO_MANY);
        }
    }
}

int radix_for(int64_t build_rows, int64_t row_bytes, int64_t budget) {
    // 2^radix partitions of at most a sixteenth of the budget each (3..6 bits).
    if (budget <= 0 || build_rows <= 0) return 3;
    const double total = (double)build_rows * (double)(row_bytes + 40);
    int bits = 3;
    while (bits < 6 && total / (double)(1 << bits) > (double)budget / 16.0) bits++;
    return bits;
}

}  // namespace

// ---- the operator ------------------------------------------------------------------
class GraceJoin {
    // One partition's rows of a partitioned slice (views of its buffers).
    struct Segment {
        DevBatch batch;
        int64_t rows = 0;
    };

  public:
    GraceJoin(Runtime *rt, const krv_join_spec &spec, const krv_grace_options &opt) : rt_(rt), spec_(spec), opt_(opt) {
        if (spec.join_type != KRV_JOIN_INNER && spec.join_type != KRV_JOIN_LEFT_OUTER)
            fail(KRV_UNSUPPORTED, "partitioned joins are inner or left outer");
        if (spec.n_keys != 1 || spec.null_safe[0])
            fail(KRV_UNSUPPORTED, "partitioned joins have one `=` key");
        if (spec.has_residual_filter)
            fail(KRV_UNSUPPORTED, "KRISHIV_UNSUPPORTED_FEATURE: residual join filters on the GPU join");
        spec_.runtime_filter = 0;
        if (spec_.seed == 0) spec_.seed = 0x4B52565F4A4F494EULL;
        budget_ = opt_.device_budget_bytes > 0 ? opt_.device_budget_bytes : rt_->budget;
        if (budget_ <= 0) {
            size_t free_b = 0, total_b = 0;
            KRV_CUDA(cudaMemGetInfo(&free_b, &total_b));
            budget_ = (int64_t)(free_b / 2);
        }
        KRV_CUDA(cudaStreamCreateWithFlags(&cs_, cudaStreamNonBlocking));
    }
    ~GraceJoin() {
        cudaStreamSynchronize(cs_);  // copies into or out of the spill space
        cudaStreamSynchronize(rt_->stream);
        for (auto &f : inflight_) cudaEventDestroy(f.done);
        inflight_.clear();
        if (prefetch_.ready) cudaEventDestroy(prefetch_.ready);
        cudaStreamDestroy(cs_);
        for (auto &b : host_blocks_) rt_->host_pool->give(b.first, b.second);
    }

    void build_push(const DevBatch &in) {
        if (built_) fail(KRV_INVALID_ARGUMENT, "build_push after build_finish");
        DeviceGuard g(rt_);
        if (!schema_) init_schema(in);
        check_shape(in, build_types_, spec_.build_keys[0], "build");
        counters_.build_rows += in.rows;
        for (int64_t from = 0; from < in.rows; from += slice_rows()) build_slice(slice(in, from));
    }

    void build_slice(const DevBatch &b) {
        std::vector<Segment> segs = partition(b, spec_.build_keys[0], 0, parts_bits_, false, bloom_ ? kFilterInsert : kFilterNone);
        for (int p = 0; p < nparts_; p++) {
            Segment &s = segs[p];
            if (s.rows == 0) continue;
            Part &P = parts_[p];
            if (P.spilled) {
                P.build_host.push_back(spill(s));
            } else {
                P.join->build_push(s.batch);
                P.build_rows += s.rows;
            }
        }
        enforce_residency();
    }

    void build_finish() {
        if (built_) fail(KRV_INVALID_ARGUMENT, "build_finish called twice");
        DeviceGuard g(rt_);
        if (!schema_) fail(KRV_INVALID_ARGUMENT, "a partitioned join needs the build side's schema: push a build batch");
        for (auto &P : parts_)
            if (!P.spilled) {
                P.join->build_finish();
                counters_.build_keys += P.join->counters().build_keys;
                counters_.table_slots += P.join->counters().table_slots;
            }
        // A join over no build rows pads the NULL-key probe rows (left outer).
        null_join_.reset(new HashJoin(rt_, spec_));
        null_join_->build_push(empty_like(build_types_));
        null_join_->build_finish();
        built_ = true;
    }

    // The output of one probe batch that is ready now: its rows with NULL keys
    // (left outer) and its rows of resident partitions. Rows of spilled
    // partitions wait for finish.
    std::vector<DevBatch> probe(const DevBatch &in) {
        if (!built_) fail(KRV_INVALID_ARGUMENT, "probe before build_finish");
        DeviceGuard g(rt_);
        if (probe_types_.empty()) {
            for (const DevCol &c : in.cols) probe_types_.push_back(c);
            check_cols(in, spec_.probe_keys[0], "probe");
        }
        check_shape(in, probe_types_, spec_.probe_keys[0], "probe");
        counters_.probe_rows += in.rows;
        std::vector<DevBatch> out;
        int64_t out_rows = 0;
        // The batches go out as they are, one per call of krv_join_probe: one
        // batch would cost a copy of them all (and its allocation).
        for (int64_t from = 0; from < in.rows; from += slice_rows()) probe_slice(slice(in, from), out, out_rows);
        return out;
    }

    // One slice: NULL-key rows padded now (left outer); rows of resident
    // partitions joined now while this call's output stays under a quarter
    // of the budget, else deferred to host memory like those of spilled
    // partitions (and joined at finish by the same resident tables).
    void probe_slice(const DevBatch &in, std::vector<DevBatch> &out, int64_t &out_rows) {
        std::vector<Segment> segs = partition(in, spec_.probe_keys[0], 0, parts_bits_, true, bloom_ ? kFilterTest : kFilterNone);
        Segment &nulls = segs[nparts_];
        if (nulls.rows > 0 && spec_.join_type == KRV_JOIN_LEFT_OUTER) {
            out_rows += nulls.rows;
            keep(out, null_join_->probe(with_null_keys(nulls)));
        }
        // Rows whose key the build side's Bloom filter rules out match no
        // build row: padded now (left outer), never partitioned or spilled.
        Segment &ruled_out = segs[nparts_ + 1];
        counters_filtered_ += last_filtered_;
        const int64_t out_cap = budget_ / 8 / out_row_bytes();
        if (ruled_out.rows > 0 && spec_.join_type == KRV_JOIN_LEFT_OUTER) {
            if (out_rows + ruled_out.rows > out_cap) {
                pad_later_.push_back(spill(ruled_out));  // past this call's output share: padded at finish
            } else {
                out_rows += ruled_out.rows;
                keep(out, null_join_->probe(ruled_out.batch));
            }
        }
        const double ratio = out_ratio();
        std::vector<int> now;  // resident partitions joined by this slice's launch
        double expect = 0;
        for (int p = 0; p < nparts_; p++) {
            Segment &s = segs[p];
            if (s.rows == 0) continue;
            Part &P = parts_[p];
            if (P.spilled) {
                P.probe_host.push_back(spill(s));
            } else if ((double)out_rows + expect >= (double)out_cap) {
                P.deferred.push_back(spill(s));
            } else {
                now.push_back(p);
                expect += (double)s.rows * ratio;
            }
        }
        if (!now.empty()) {
            DevBatch o = probe_resident(segs, now, ratio);
            out_rows += o.rows;
            keep(out, std::move(o));
        }
    }

    // Output rows per probe row of the resident partitions: as observed so
    // far, else the build's mean rows per key (at least 1 for left outer).
    double out_ratio() const {
        if (res_probe_rows_ > 0) return (double)res_out_rows_ / (double)res_probe_rows_;
        int64_t rows = 0, keys = 0;
        for (const Part &P : parts_)
            if (!P.spilled && P.join) {
                rows += P.join->indexed_rows();
                keys += P.join->counters().build_keys;
            }
        double r = keys > 0 ? (double)rows / (double)keys : 1.0;
        if (spec_.join_type == KRV_JOIN_LEFT_OUTER) r = std::max(r, 1.0);
        return r;
    }

    static std::vector<int> projection(int n, const int32_t *cols, int ncols) {
        std::vector<int> v;
        if (n < 0) {
            for (int i = 0; i < ncols; i++) v.push_back(i);
        } else {
            for (int i = 0; i < n; i++) {
                if (cols[i] < 0 || cols[i] >= ncols) fail(KRV_INVALID_ARGUMENT, "projection column out of range");
                v.push_back(cols[i]);
            }
        }
        return v;
    }

    // The segments `now` of one partitioned slice, each probed against its
    // resident partition's table, in one launch and one output batch.
    DevBatch probe_resident(const std::vector<Segment> &segs, const std::vector<int> &now, double ratio) {
        const int key = spec_.probe_keys[0];
        const std::vector<int> pcols = projection(spec_.n_probe_out, spec_.probe_out, (int)probe_types_.size());
        const std::vector<int> bcols = projection(spec_.n_build_out, spec_.build_out, (int)build_types_.size());
        if (pcols.size() + bcols.size() > (size_t)kGMaxOut) fail(KRV_UNSUPPORTED, "more than 16 output columns");
        const DevBatch &first = segs[now[0]].batch;
        GOutDev od{};
        for (size_t c = 0; c < first.cols.size(); c++) od.pcol[c] = first.cols[c].hold_data->get();
        od.pkey = static_cast<const long long *>(od.pcol[key]);
        std::vector<GPartDev> hp;
        int64_t tiles = 0, rows = 0;
        for (int p : now) {
            const Segment &s = segs[p];
            const HashJoin &J = *parts_[p].join;
            const HashJoin::TableDev tv = J.table_dev();
            GPartDev d{};
            d.slots = tv.slots;
            d.mask = tv.mask;
            d.next = tv.next;
            const DevBatch &arena = J.arena();
            d.bkey = arena.cols.empty() ? nullptr : static_cast<const long long *>(arena.cols[spec_.build_keys[0]].data);
            for (size_t c = 0; c < arena.cols.size() && c < (size_t)kMaxCols; c++) d.bcol[c] = arena.cols[c].data;
            d.prow0 = (static_cast<const uint8_t *>(s.batch.cols[key].data) - static_cast<const uint8_t *>(od.pcol[key])) / 8;
            d.rows = s.rows;
            d.tile0 = tiles;
            tiles += ceil_div(s.rows, (int64_t)(32 * kGRows));
            rows += s.rows;
            hp.push_back(d);
        }
        DBuf dparts(rt_, hp.size() * sizeof(GPartDev));
        KRV_CUDA(cudaMemcpyAsync(dparts.get(), hp.data(), hp.size() * sizeof(GPartDev), cudaMemcpyHostToDevice,
                                 rt_->stream));
        const bool left = spec_.join_type == KRV_JOIN_LEFT_OUTER;
        unsigned long long cap = std::max<unsigned long long>(1, (unsigned long long)((double)rows * ratio * 1.05) + 1024);
        DBuf cnt(rt_, 8);
        for (int attempt = 0; attempt < 3; attempt++) {
            DevBatch o;
            od.n = 0;
            for (int pc : pcols) {
                const DevCol &m = probe_types_[pc];
                DevCol d = make_col(rt_, m.type, (int64_t)cap, m.nullable, m.name);
                if (d.valid) KRV_CUDA(cudaMemsetAsync(const_cast<uint8_t *>(d.valid), 0, d.hold_valid->bytes(), rt_->stream));
                od.c[od.n++] = GOutCol{const_cast<void *>(d.data), (uint32_t *)d.valid, m.type.width(), 0, pc};
                o.cols.push_back(d);
            }
            for (int bc : bcols) {
                const DevCol &m = build_types_[bc];
                DevCol d = make_col(rt_, m.type, (int64_t)cap, m.nullable || left, m.name);
                if (d.valid) KRV_CUDA(cudaMemsetAsync(const_cast<uint8_t *>(d.valid), 0, d.hold_valid->bytes(), rt_->stream));
                od.c[od.n++] = GOutCol{const_cast<void *>(d.data), (uint32_t *)d.valid, m.type.width(), 1, bc};
                o.cols.push_back(d);
            }
            KRV_CUDA(cudaMemsetAsync(cnt.get(), 0, 8, rt_->stream));
            clear_status(rt_);
            const int grid = (int)std::min<int64_t>(ceil_div(tiles, (int64_t)kGProbeThreads / 32), (int64_t)rt_->sm_count * 8);
            grace_probe_kernel<<<grid, kGProbeThreads, 0, rt_->stream>>>(
                dparts.as<GPartDev>(), (int)hp.size(), tiles, spec_.seed, od, cap, cnt.as<unsigned long long>(),
                left ? 1 : 0, spec_.single_match, status_word(rt_));
            rt_->launches++;
            check_launch("grace_probe_kernel");
            const unsigned long long got = read_scalar<unsigned long long>(rt_, cnt.get());
            if (take_status(rt_) & ST_TOO_MANY)
                fail(KRV_TOO_MANY_ROWS, "SCALAR_SUBQUERY_TOO_MANY_ROWS: a probe row matched more than one build row");
            if (got <= cap) {
                o.rows = (int64_t)got;
                for (DevCol &c : o.cols) c.length = o.rows;
                res_probe_rows_ += rows;
                res_out_rows_ += o.rows;
                return o;
            }
            cap = got;  // more output than expected: again, with room for all of it
        }
        fail(KRV_INTERNAL, "partitioned probe output did not converge");
    }

    // Bytes of one output row: every column of both sides.
    int64_t out_row_bytes() const {
        int64_t b = 0;
        for (const DevCol &c : build_types_) b += c.type.width();
        for (const DevCol &c : probe_types_) b += c.type.width();
        return std::max<int64_t>(b, 8);
    }

    // Input batches are taken in slices whose partitioned copy and output
    // stay within a sixteenth of the budget (a multiple of 64 rows, so that
    // every slice starts on a byte of the validity bitmaps).
    int64_t slice_rows() const {
        const int64_t per = std::max<int64_t>(row_bytes_, 16) * 4;
        return std::max<int64_t>(1 << 16, budget_ / 16 / per / 64 * 64);
    }
    DevBatch slice(const DevBatch &b, int64_t from) const {
        if (from == 0 && b.rows <= slice_rows()) return b;
        DevBatch s;
        s.rows = std::min(slice_rows(), b.rows - from);
        for (const DevCol &c : b.cols) s.cols.push_back(slice_col(c, from, s.rows));
        return s;
    }

    // After the last probe batch: the next output batch of the spilled
    // partitions; false when none is left.
    bool finish_next(DevBatch &out) {
        if (!built_) fail(KRV_INVALID_ARGUMENT, "finish before build_finish");
        DeviceGuard g(rt_);
        if (!finishing_) {
            finishing_ = true;
            reap(true);  // every spill has landed in host memory
            for (int p = 0; p < nparts_; p++)
                if (parts_[p].spilled) tasks_.push_back(Task{0, std::move(parts_[p].build_host), std::move(parts_[p].probe_host)});
        }
        // Ruled-out rows that did not fit their call's output: padded now.
        while (pad_chunk_ < pad_later_.size()) {
            DevBatch o = null_join_->probe(load_group(pad_later_, pad_chunk_));
            counters_.output_rows += o.rows;
            if (o.rows > 0) {
                out = o;
                return true;
            }
        }
        // Deferred rows of resident partitions, by their resident tables.
        for (; deferred_part_ < nparts_; deferred_part_++, deferred_chunk_ = 0) {
            Part &P = parts_[deferred_part_];
            while (!P.spilled && deferred_chunk_ < P.deferred.size()) {
                DevBatch o = P.join->probe(load_group(P.deferred, deferred_chunk_));
                counters_.output_rows += o.rows;
                if (o.rows > 0) {
                    out = o;
                    return true;
                }
            }
            P.join.reset();  // this resident table is done
        }
        for (;;) {
            if (fb_.active) {
                if (fallback_next(out)) return true;
                continue;
            }
            if (cur_join_) {
                if (prefetch_.pending || cur_probe_ < cur_.probe_host.size()) {
                    DevBatch pb = prefetch_.pending ? take_prefetch() : load_group(cur_.probe_host, cur_probe_);
                    // the next group crosses the host link while this one is probed
                    if (cur_probe_ < cur_.probe_host.size()) start_prefetch(cur_.probe_host, cur_probe_);
                    DevBatch o = cur_join_->probe(pb);
                    counters_.output_rows += o.rows;
                    if (o.rows == 0) continue;
                    out = o;
                    return true;
                }
                cur_join_.reset();
                cur_ = Task{};
            }
            if (tasks_.empty()) return false;
            Task t = std::move(tasks_.front());
            tasks_.pop_front();
            int64_t rows = 0;
            for (const HostChunk &c : t.build_host) rows += c.rows;
            if (t.probe_host.empty()) continue;  // no probe rows: nothing to emit
            if (est_part_bytes(rows) > resident_cap() && t.level < kMaxLevel && !no_shrink(t, rows)) {
                split(t);
                continue;
            }
            if (est_part_bytes(rows) > resident_cap()) {
                // Splitting cannot shrink it (one heavy key): the fallback.
                start_fallback(std::move(t));
                continue;
            }
            krv_join_spec js = spec_;
            js.build_rows_hint = rows;
            cur_join_.reset(new HashJoin(rt_, js));
            if (rows == 0) cur_join_->build_push(empty_like(build_types_));
            else cur_join_->build_adopt(load_all(t.build_host, build_types_));
            cur_join_->build_finish();
            counters_.build_keys += cur_join_->counters().build_keys;
            counters_.table_slots += cur_join_->counters().table_slots;
            cur_ = std::move(t);
            cur_probe_ = 0;
        }
    }

    bool done() const {
        return finishing_ && pad_chunk_ >= pad_later_.size() && deferred_part_ >= nparts_ && !cur_join_ &&
               tasks_.empty() && !fb_.active;
    }
    // A zero-row batch of the output's shape.
    DevBatch empty_output() {
        if (!built_ || probe_types_.empty()) return DevBatch{};
        return null_join_->probe(empty_like(probe_types_));
    }
    const krv_join_spec &spec() const { return spec_; }
    krv_join_counters counters() const {
        krv_join_counters c = counters_;
        c.partitions = nparts_ + splits_;
        return c;
    }
    int64_t filtered_probe_rows() const { return counters_filtered_; }
    int64_t spilled_partitions() const {
        int64_t n = 0;
        for (const auto &P : parts_) n += P.spilled;
        return n;
    }

  private:
    struct HostChunk {
        std::vector<uint8_t *> cols;
        int64_t rows = 0;
    };
    struct Part {
        std::unique_ptr<HashJoin> join;  // resident: the partition's join
        bool spilled = false;
        int64_t build_rows = 0;
        std::vector<HostChunk> build_host, probe_host;
        std::vector<HostChunk> deferred;  // probe rows for the resident table, joined at finish
    };
    struct Task {
        int level = 0;
        std::vector<HostChunk> build_host, probe_host;
    };

    void check_cols(const DevBatch &b, int key, const char *side) {
        if (key < 0 || key >= (int)b.cols.size()) fail(KRV_INVALID_ARGUMENT, std::string(side) + " key column out of range");
        if (b.cols[key].type.id != Type::I64) fail(KRV_UNSUPPORTED, "partitioned joins have an int64 key");
        if ((int)b.cols.size() > kMaxCols) fail(KRV_UNSUPPORTED, "partitioned joins take at most 8 columns per side");
        for (int i = 0; i < (int)b.cols.size(); i++) {
            const int w = b.cols[i].type.width();
            if (b.cols[i].type.id == Type::Bool || (w != 4 && w != 8))
                fail(KRV_UNSUPPORTED, "partitioned joins take 4- and 8-byte columns");
        }
    }
    void init_schema(const DevBatch &b) {
        check_cols(b, spec_.build_keys[0], "build");
        for (const DevCol &c : b.cols) build_types_.push_back(c);
        int64_t row_bytes = 0;
        for (const DevCol &c : b.cols) row_bytes += c.type.width();
        row_bytes_ = row_bytes;
        parts_bits_ = spec_.radix_bits >= 3 ? std::min(spec_.radix_bits, 6)
                                            : radix_for(spec_.build_rows_hint, row_bytes_, budget_);
        nparts_ = 1 << parts_bits_;
        parts_.resize(nparts_);
        if (opt_.probe_filter_bits > 0) {
            // the Bloom filter the build side's partition passes fill
            const int64_t want = spec_.build_rows_hint > 0 ? spec_.build_rows_hint * opt_.probe_filter_bits / 8
                                                           : std::min<int64_t>(budget_ / 32, 64 << 20);
            bloom_bytes_ = std::max<int64_t>(32, std::min<int64_t>(want, budget_ / 16)) / 32 * 32;
            bloom_blocks_ = (uint64_t)bloom_bytes_ / 32;
            bloom_.reset(new DBuf(rt_, (size_t)bloom_bytes_));
            KRV_CUDA(cudaMemsetAsync(bloom_->get(), 0, (size_t)bloom_bytes_, rt_->stream));
        }
        // With a size hint the spilled partitions are known up front; without
        // one, partitions spill as the resident footprint passes its share.
        int resident = nparts_;
        if (spec_.build_rows_hint > 0) {
            const int64_t per = std::max<int64_t>(est_part_bytes(spec_.build_rows_hint / nparts_ * 21 / 20), 1);
            resident = (int)std::min<int64_t>(nparts_, resident_cap() / per);
        }
        for (int p = 0; p < nparts_; p++) {
            parts_[p].spilled = p >= resident;
            if (!parts_[p].spilled) {
                krv_join_spec js = spec_;
                js.build_rows_hint = spec_.build_rows_hint > 0 ? spec_.build_rows_hint / nparts_ * 9 / 8 + 1024 : 0;
                parts_[p].join.reset(new HashJoin(rt_, js));
                // the build schema, even for a partition that gets no rows
                parts_[p].join->build_push(empty_like(build_types_));
            }
        }
        schema_ = true;
    }
    void check_shape(const DevBatch &b, const std::vector<DevCol> &types, int key_col, const char *side) const {
        if (b.cols.size() != types.size()) fail(KRV_INVALID_ARGUMENT, std::string(side) + " batches differ in columns");
        for (size_t i = 0; i < types.size(); i++) {
            if (b.cols[i].type != types[i].type) fail(KRV_INVALID_ARGUMENT, std::string(side) + " batches differ in types");
            const bool key = (int)i == key_col;
            if (!key && b.cols[i].valid)
                fail(KRV_UNSUPPORTED, "partitioned joins take NULLs in the key column only");
        }
    }
    // Device bytes of a partition's table over `rows` build rows: the rows
    // (with their arena's headroom and validity bits), the chain links and the
    // slots (a power of two of at least rows / 0.5).
    int64_t est_part_bytes(int64_t rows) const {
        uint64_t slots = 1;
        while (slots < (uint64_t)(2 * rows)) slots <<= 1;
        return rows * (row_bytes_ * 9 / 8 + 4 + 1) + (int64_t)slots * 8;
    }
    // The share of the budget that resident tables may take; the rest holds
    // a slice's partitioned copy and a call's output.
    int64_t resident_cap() const { return (budget_ - bloom_bytes_) / 10 * 6; }
    int64_t resident_bytes() const {
        int64_t b = 0;
        for (const auto &P : parts_)
            if (!P.spilled) b += est_part_bytes(P.build_rows);
        return b;
    }

    void enforce_residency() {
        while (resident_bytes() > resident_cap()) {
            int victim = -1;
            for (int p = 0; p < nparts_; p++)
                if (!parts_[p].spilled && (victim < 0 || parts_[p].build_rows > parts_[victim].build_rows)) victim = p;
            if (victim < 0) break;
            Part &P = parts_[victim];
            if (P.build_rows > 0) {
                Segment s;
                s.batch = P.join->staged();
                s.rows = P.build_rows;
                P.build_host.push_back(spill(s));
            }
            P.join.reset();
            P.spilled = true;
        }
    }

    // Partitions batch `b` by its key column at `level`: one segment (a
    // device batch of the partition's rows) per partition, plus the NULL-key
    // bucket at index nparts (kept when keep_nulls).
    std::vector<Segment> partition(const DevBatch &b, int key, int level, int bits, bool keep_nulls,
                                   int filter_mode = kFilterNone) {
        const int nparts = level == 0 ? (1 << bits) : 8;
        PartArgs A{};
        A.key = static_cast<const long long *>(b.cols[key].data);
        A.kvalid = b.cols[key].valid;
        A.kvoff = b.cols[key].valid_off;
        A.n = b.rows;
        A.level = level;
        A.bits = bits;
        A.seed = spec_.seed;
        A.nparts = nparts;
        A.keep_nulls = keep_nulls ? 1 : 0;
        A.filter_mode = filter_mode;
        A.keep_filtered = spec_.join_type == KRV_JOIN_LEFT_OUTER ? 1 : 0;
        A.bloom = bloom_ ? bloom_->as<uint32_t>() : nullptr;
        A.bloom_blocks = bloom_blocks_;
        A.ncols = (int)b.cols.size();
        const int nb = nparts + 2;  // partitions, the NULL bucket, the filtered bucket
        DBuf ctr(rt_, (size_t)nb * 8 * 2);
        DBuf bucket;
        if (filter_mode == kFilterTest && b.rows > 0) {
            bucket = DBuf(rt_, (size_t)b.rows);
            A.bucket = bucket.as<uint8_t>();
        }
        unsigned long long *hist = ctr.as<unsigned long long>(), *cursor = hist + nb;
        KRV_CUDA(cudaMemsetAsync(hist, 0, (size_t)nb * 8, rt_->stream));
        part_hist_kernel<<<grid_for(rt_, b.rows, 256, 8), 256, 0, rt_->stream>>>(A, hist);
        rt_->launches++;
        check_launch("part_hist_kernel");
        std::vector<unsigned long long> h(nb);
        KRV_CUDA(cudaMemcpyAsync(h.data(), hist, nb * 8, cudaMemcpyDeviceToHost, rt_->stream));
        KRV_CUDA(cudaStreamSynchronize(rt_->stream));
        last_filtered_ = (int64_t)h[nparts + 1];  // counted whether the bucket is kept or dropped
        std::vector<unsigned long long> start(nb);
        std::vector<bool> kept_bucket(nb, true);
        kept_bucket[nparts] = keep_nulls;
        kept_bucket[nparts + 1] = A.keep_filtered != 0;
        unsigned long long acc = 0;
        for (int p = 0; p < nb; p++) {
            start[p] = acc;
            if (kept_bucket[p]) acc += h[p];
        }
        KRV_CUDA(cudaMemcpyAsync(cursor, start.data(), nb * 8, cudaMemcpyHostToDevice, rt_->stream));
        const int64_t kept = (int64_t)acc;
        std::vector<std::shared_ptr<DBuf>> outs;
        for (int c = 0; c < A.ncols; c++) {
            const int w = b.cols[c].type.width();
            outs.push_back(std::make_shared<DBuf>(rt_, (size_t)std::max<int64_t>(kept, 1) * w));
            A.c[c] = PartCol{b.cols[c].data, outs.back()->get(), w};
        }
        if (kept > 0) {
            part_scatter_kernel<<<grid_for(rt_, ceil_div(b.rows, kPartTile), 1, 4), kPartThreads, 0, rt_->stream>>>(
                A, cursor);
            rt_->launches++;
            check_launch("part_scatter_kernel");
        }
        std::vector<Segment> segs(nb);
        for (int p = 0; p < nb; p++) {
            Segment &s = segs[p];
            s.rows = kept_bucket[p] ? (int64_t)h[p] : 0;
            s.batch.rows = s.rows;
            for (int c = 0; c < A.ncols; c++) {
                DevCol col;
                col.type = b.cols[c].type;
                col.name = b.cols[c].name;
                col.nullable = b.cols[c].nullable;
                col.length = s.rows;
                col.hold_data = outs[c];
                col.data = outs[c]->as<uint8_t>() + start[p] * (size_t)b.cols[c].type.width();
                s.batch.cols.push_back(col);
            }
        }
        return segs;
    }

    // The NULL bucket's rows with their key column marked NULL.
    DevBatch with_null_keys(const Segment &s) {
        DevBatch b = s.batch;
        const int key = spec_.probe_keys[0];
        auto bits = std::make_shared<DBuf>(rt_, (size_t)ceil_div(s.rows, 8) + 8);
        KRV_CUDA(cudaMemsetAsync(bits->get(), 0, bits->bytes(), rt_->stream));
        b.cols[key].hold_valid = bits;
        b.cols[key].valid = bits->as<uint8_t>();
        b.cols[key].valid_off = 0;
        b.cols[key].nullable = true;
        return b;
    }

    DevBatch empty_like(const std::vector<DevCol> &types) {
        DevBatch b;
        for (const DevCol &t : types) b.cols.push_back(make_col(rt_, t.type, 0, t.nullable, t.name));
        return b;
    }

    void keep(std::vector<DevBatch> &out, DevBatch b) {
        counters_.output_rows += b.rows;
        if (b.rows > 0) out.push_back(std::move(b));
    }

    uint8_t *host_alloc(size_t bytes) {
        bytes = (bytes + 255) / 256 * 256;
        if (bytes > HostPool::kBlock) {
            uint8_t *p = rt_->host_pool->take(bytes);
            host_blocks_.push_back({p, bytes});
            return p;
        }
        if (host_blocks_.empty() || cur_block_used_ + bytes > HostPool::kBlock || cur_block_ == nullptr) {
            cur_block_ = rt_->host_pool->take(HostPool::kBlock);
            host_blocks_.push_back({cur_block_, HostPool::kBlock});
            cur_block_used_ = 0;
        }
        uint8_t *p = cur_block_ + cur_block_used_;
        cur_block_used_ += bytes;
        return p;
    }

    // Copies a segment to the spill space (asynchronously, stream-ordered).
    // Copies a segment to the spill space on the copy stream, so that the
    // transfer overlaps the next slice's kernels; the segment's device
    // buffers stay alive until the copy has landed.
    HostChunk spill(const Segment &s) {
        HostChunk h;
        h.rows = s.rows;
        cudaEvent_t ready;
        KRV_CUDA(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
        KRV_CUDA(cudaEventRecord(ready, rt_->stream));
        KRV_CUDA(cudaStreamWaitEvent(cs_, ready, 0));
        KRV_CUDA(cudaEventDestroy(ready));
        InFlight f;
        for (const DevCol &c : s.batch.cols) {
            const size_t bytes = (size_t)s.rows * c.type.width();
            uint8_t *p = host_alloc(bytes);
            KRV_CUDA(cudaMemcpyAsync(p, c.data, bytes, cudaMemcpyDeviceToHost, cs_));
            h.cols.push_back(p);
            f.hold.push_back(c.hold_data);
            f.bytes += bytes;
        }
        KRV_CUDA(cudaEventCreateWithFlags(&f.done, cudaEventDisableTiming));
        KRV_CUDA(cudaEventRecord(f.done, cs_));
        inflight_bytes_ += f.bytes;
        inflight_.push_back(std::move(f));
        spilled_bytes_ += (int64_t)s.rows * row_bytes_;
        reap(false);
        // A short queue of spills: other small transfers share the copy engines.
        while (inflight_bytes_ > std::min<size_t>((size_t)(budget_ / 8), (size_t)1 << 30) && !inflight_.empty())
            reap_one();
        return h;
    }

    // Releases the buffers of spills that have landed (all of them: wait).
    void reap(bool all) {
        while (!inflight_.empty()) {
            if (all) {
                reap_one();
                continue;
            }
            const cudaError_t q = cudaEventQuery(inflight_.front().done);
            if (q == cudaErrorNotReady) return;
            if (q != cudaSuccess) fail(KRV_CUDA_ERROR, std::string("spill copy: ") + cudaGetErrorString(q));
            reap_one();
        }
    }
    void reap_one() {
        InFlight &f = inflight_.front();
        KRV_CUDA(cudaEventSynchronize(f.done));
        KRV_CUDA(cudaEventDestroy(f.done));
        inflight_bytes_ -= f.bytes;
        inflight_.pop_front();
    }

    // The probe chunks from `at` on that fit one slice, copied to the device on
    // the copy stream; take_prefetch orders the join's stream after them.
    void start_prefetch(const std::vector<HostChunk> &hs, size_t &at) {
        std::vector<HostChunk> group;
        int64_t rows = 0;
        while (at < hs.size() && (group.empty() || rows + hs[at].rows <= slice_rows())) {
            rows += hs[at].rows;
            group.push_back(hs[at++]);
        }
        prefetch_.batch = alloc_like(probe_types_, rows);  // allocated in the join's stream order
        cudaEvent_t ready;
        KRV_CUDA(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
        KRV_CUDA(cudaEventRecord(ready, rt_->stream));
        KRV_CUDA(cudaStreamWaitEvent(cs_, ready, 0));
        KRV_CUDA(cudaEventDestroy(ready));
        copy_in(group, prefetch_.batch, cs_);
        if (!prefetch_.ready) KRV_CUDA(cudaEventCreateWithFlags(&prefetch_.ready, cudaEventDisableTiming));
        KRV_CUDA(cudaEventRecord(prefetch_.ready, cs_));
        prefetch_.pending = true;
    }
    DevBatch take_prefetch() {
        KRV_CUDA(cudaStreamWaitEvent(rt_->stream, prefetch_.ready, 0));
        prefetch_.pending = false;
        DevBatch b = std::move(prefetch_.batch);
        prefetch_.batch = DevBatch{};
        return b;
    }
    DevBatch alloc_like(const std::vector<DevCol> &types, int64_t rows) {
        DevBatch b;
        b.rows = rows;
        for (const DevCol &t : types) {
            DevCol col;
            col.type = t.type;
            col.name = t.name;
            col.nullable = t.nullable;
            col.length = rows;
            col.hold_data = std::make_shared<DBuf>(rt_, (size_t)std::max<int64_t>(rows, 1) * t.type.width());
            col.data = col.hold_data->get();
            b.cols.push_back(col);
        }
        return b;
    }
    void copy_in(const std::vector<HostChunk> &hs, DevBatch &b, cudaStream_t st) {
        for (size_t c = 0; c < b.cols.size(); c++) {
            const int w = b.cols[c].type.width();
            int64_t at = 0;
            for (const HostChunk &h : hs) {
                if (h.rows)
                    KRV_CUDA(cudaMemcpyAsync(b.cols[c].hold_data->as<uint8_t>() + at * w, h.cols[c], (size_t)h.rows * w,
                                             cudaMemcpyHostToDevice, st));
                at += h.rows;
            }
        }
    }

    // Probe chunks from `at` on, as many as fit one slice, loaded as one
    // device batch; `at` moves past them.
    DevBatch load_group(const std::vector<HostChunk> &hs, size_t &at) {
        std::vector<HostChunk> group;
        int64_t rows = 0;
        while (at < hs.size() && (group.empty() || rows + hs[at].rows <= slice_rows())) {
            rows += hs[at].rows;
            group.push_back(hs[at++]);
        }
        return load_all(group, probe_types_);
    }

    DevBatch load(const HostChunk &h, const std::vector<DevCol> &types) {
        std::vector<HostChunk> one{h};
        return load_all(one, types);
    }
    // The rows of chunks `hs`, back on the device as owned columns (after
    // the spills still on their way to host memory, which they may be).
    DevBatch load_all(const std::vector<HostChunk> &hs, const std::vector<DevCol> &types) {
        int64_t rows = 0;
        for (const HostChunk &h : hs) rows += h.rows;
        if (!inflight_.empty()) KRV_CUDA(cudaStreamWaitEvent(rt_->stream, inflight_.back().done, 0));
        DevBatch b = alloc_like(types, rows);
        copy_in(hs, b, rt_->stream);
        return b;
    }

    // ---- the fallback (join/fallback.rs: a partition that splitting
    // cannot shrink joins by sort-merge, started at join/grace.rs:1006-1013)
    // Here the same rows come from the build side in groups of chunks that
    // each fit the resident share of the budget: every group's table joins
    // every probe chunk (inner pairs, each probe row carrying its id), the
    // ids of matched probe rows are marked, and for a left outer join the
    // probe rows no group matched are padded at the end.
    struct Fallback {
        bool active = false;
        std::vector<std::vector<HostChunk>> groups;
        size_t group = 0;
        std::unique_ptr<HashJoin> join;
        std::vector<HostChunk> probe_host;
        std::vector<long long> probe_base;  // id of each probe chunk's first row
        size_t probe_at = 0;
        DBuf matched;                        // a byte per probe row: matched by some group
        bool padding = false;
    } fb_;
    int64_t fallbacks_ = 0;

    // Whether the task's build side would not shrink: its rows all share one key.
    bool no_shrink(const Task &t, int64_t rows) {
        if (rows < 2) return true;
        reap(true);  // the chunks' spill copies have landed
        long long first = 0;
        bool have = false;
        for (const HostChunk &c : t.build_host)
            if (c.rows) {
                first = reinterpret_cast<const long long *>(c.cols[spec_.build_keys[0]])[0];
                have = true;
                break;
            }
        if (!have) return true;
        for (const HostChunk &c : t.build_host) {
            const long long *k = reinterpret_cast<const long long *>(c.cols[spec_.build_keys[0]]);
            for (int64_t i = 0; i < c.rows; i++)
                if (k[i] != first) return false;
        }
        return true;
    }

    void start_fallback(Task t) {
        fallbacks_++;
        fb_ = Fallback{};
        fb_.active = true;
        std::vector<HostChunk> g;
        int64_t grows = 0;
        for (HostChunk &c : t.build_host) {
            if (!g.empty() && est_part_bytes(grows + c.rows) > resident_cap()) {
                fb_.groups.push_back(std::move(g));
                g.clear();
                grows = 0;
            }
            grows += c.rows;
            g.push_back(c);
        }
        if (!g.empty()) fb_.groups.push_back(std::move(g));
        long long base = 0;
        for (const HostChunk &c : t.probe_host) {
            fb_.probe_base.push_back(base);
            base += c.rows;
        }
        fb_.probe_host = std::move(t.probe_host);
        if (spec_.join_type == KRV_JOIN_LEFT_OUTER) {
            fb_.matched = DBuf(rt_, (size_t)std::max<long long>(base, 1));
            KRV_CUDA(cudaMemsetAsync(fb_.matched.get(), 0, fb_.matched.bytes(), rt_->stream));
        }
    }

    // The probe chunk at `at` with its row ids as a last column.
    DevBatch load_with_ids(size_t at) {
        DevBatch b = load(fb_.probe_host[at], probe_types_);
        DevCol id;
        id.type = DType{Type::I64, 0, 0};
        id.name = "#row";
        id.nullable = false;
        id.length = b.rows;
        id.hold_data = std::make_shared<DBuf>(rt_, (size_t)std::max<int64_t>(b.rows, 1) * 8);
        id.data = id.hold_data->get();
        if (b.rows) {
            iota_kernel<<<grid_for(rt_, b.rows, 256, 4), 256, 0, rt_->stream>>>(id.hold_data->as<long long>(), b.rows,
                                                                                fb_.probe_base[at]);
            rt_->launches++;
            check_launch("iota_kernel");
        }
        b.cols.push_back(id);
        return b;
    }

    // The next output batch of the fallback; false when it produced none
    // this step (the caller calls again until it is no longer active).
    bool fallback_next(DevBatch &out) {
        if (!fb_.padding) {
            if (!fb_.join) {
                if (fb_.group == fb_.groups.size()) {
                    fb_.padding = spec_.join_type == KRV_JOIN_LEFT_OUTER;
                    fb_.probe_at = 0;
                    if (!fb_.padding) fb_ = Fallback{};
                    return false;
                }
                // inner pairs of this group; the probe rows keep their id
                krv_join_spec js = spec_;
                js.join_type = KRV_JOIN_INNER;
                js.runtime_filter = 0;
                const int np = (int)probe_types_.size();
                if (spec_.n_probe_out < 0) {
                    js.n_probe_out = np + 1;
                    for (int c = 0; c <= np; c++) js.probe_out[c] = c;
                } else {
                    js.probe_out[js.n_probe_out++] = np;
                }
                int64_t rows = 0;
                for (const HostChunk &c : fb_.groups[fb_.group]) rows += c.rows;
                js.build_rows_hint = rows;
                fb_.join.reset(new HashJoin(rt_, js));
                fb_.join->build_adopt(load_all(fb_.groups[fb_.group], build_types_));
                fb_.join->build_finish();
                fb_.probe_at = 0;
            }
            if (fb_.probe_at == fb_.probe_host.size()) {
                fb_.join.reset();
                fb_.group++;
                return false;
            }
            const size_t at = fb_.probe_at++;
            DevBatch o = fb_.join->probe(load_with_ids(at));
            // the id column follows the probe columns
            const int idc = spec_.n_probe_out < 0 ? (int)probe_types_.size() : spec_.n_probe_out;
            if (fb_.matched.get() && o.rows) {
                mark_matched_kernel<<<grid_for(rt_, o.rows, 256, 4), 256, 0, rt_->stream>>>(
                    static_cast<const long long *>(o.cols[idc].data), o.rows, fb_.matched.as<uint8_t>());
                rt_->launches++;
                check_launch("mark_matched_kernel");
            }
            o.cols.erase(o.cols.begin() + idc);
            counters_.output_rows += o.rows;
            if (o.rows == 0) return false;
            out = o;
            return true;
        }
        // left outer: the probe rows no group matched, the build side NULL
        if (fb_.probe_at == fb_.probe_host.size()) {
            fb_ = Fallback{};
            return false;
        }
        const size_t at = fb_.probe_at++;
        DevBatch b = load(fb_.probe_host[at], probe_types_);
        DevBatch keep = alloc_like(probe_types_, b.rows);
        PartArgs A{};
        A.n = b.rows;
        A.ncols = (int)b.cols.size();
        for (int c = 0; c < A.ncols; c++) A.c[c] = PartCol{b.cols[c].data, keep.cols[c].hold_data->get(), b.cols[c].type.width()};
        DBuf cnt(rt_, 8);
        KRV_CUDA(cudaMemsetAsync(cnt.get(), 0, 8, rt_->stream));
        if (b.rows) {
            compact_unmatched_kernel<<<grid_for(rt_, b.rows, 256, 4), 256, 0, rt_->stream>>>(
                A, fb_.matched.as<uint8_t>(), fb_.probe_base[at], cnt.as<unsigned long long>());
            rt_->launches++;
            check_launch("compact_unmatched_kernel");
        }
        keep.rows = (int64_t)read_scalar<unsigned long long>(rt_, cnt.get());
        for (DevCol &c : keep.cols) c.length = keep.rows;
        if (keep.rows == 0) return false;
        DevBatch o = null_join_->probe(keep);
        counters_.output_rows += o.rows;
        out = o;
        return true;
    }

    // Splits task `t` 8 ways with the next level of hash bits, chunk by chunk.
    void split(Task &t) {
        const int level = t.level + 1;
        std::vector<Task> sub(8);
        for (auto &s : sub) s.level = level;
        for (const HostChunk &h : t.build_host) {
            std::vector<Segment> segs = partition(load(h, build_types_), spec_.build_keys[0], level, 3, false);
            for (int p = 0; p < 8; p++)
                if (segs[p].rows) sub[p].build_host.push_back(spill(segs[p]));
        }
        for (const HostChunk &h : t.probe_host) {
            std::vector<Segment> segs = partition(load(h, probe_types_), spec_.probe_keys[0], level, 3, false);
            for (int p = 0; p < 8; p++)
                if (segs[p].rows) sub[p].probe_host.push_back(spill(segs[p]));
        }
        splits_ += 8;
        for (auto &s : sub) tasks_.push_front(std::move(s));
    }

    Runtime *rt_;
    krv_join_spec spec_;
    krv_grace_options opt_;
    int64_t budget_ = 0;
    std::unique_ptr<DBuf> bloom_;  // the probe-side filter over the build keys (none: no filter)
    int64_t bloom_bytes_ = 0;
    uint64_t bloom_blocks_ = 0;
    int64_t counters_filtered_ = 0;
    int64_t last_filtered_ = 0;  // rows the last partition pass's filter ruled out
    std::vector<HostChunk> pad_later_;  // ruled-out probe rows past a call's output share (left outer)
    size_t pad_chunk_ = 0;
    bool schema_ = false, built_ = false, finishing_ = false;
    std::vector<DevCol> build_types_, probe_types_;
    int64_t row_bytes_ = 0;
    int parts_bits_ = 3, nparts_ = 0;
    int64_t splits_ = 0;
    std::vector<Part> parts_;
    int64_t spilled_bytes_ = 0;
    std::unique_ptr<HashJoin> null_join_;
    std::deque<Task> tasks_;
    Task cur_;
    size_t cur_probe_ = 0;
    int deferred_part_ = 0;
    size_t deferred_chunk_ = 0;
    std::unique_ptr<HashJoin> cur_join_;
    std::vector<std::pair<uint8_t *, size_t>> host_blocks_;
    cudaStream_t cs_ = nullptr;  // copies to and from the spill space
    int64_t res_probe_rows_ = 0, res_out_rows_ = 0;  // the resident partitions' probes so far
    struct InFlight {
        cudaEvent_t done = nullptr;
        std::vector<std::shared_ptr<DBuf>> hold;
        size_t bytes = 0;
    };
    std::deque<InFlight> inflight_;
    size_t inflight_bytes_ = 0;
    struct Prefetch {
        DevBatch batch;
        cudaEvent_t ready = nullptr;
        bool pending = false;
    } prefetch_;
    uint8_t *cur_block_ = nullptr;
    size_t cur_block_used_ = 0;
    krv_join_counters counters_{};
};

GraceJoin *make_grace(Runtime *rt, const krv_join_spec &spec, const krv_grace_options &opt) {
    return new GraceJoin(rt, spec, opt);
}
void grace_destroy(GraceJoin *g) { delete g; }
void grace_build_push(GraceJoin *g, const DevBatch &b) { g->build_push(b); }
void grace_build_finish(GraceJoin *g) { g->build_finish(); }
std::vector<DevBatch> grace_probe(GraceJoin *g, const DevBatch &b) { return g->probe(b); }
bool grace_finish_next(GraceJoin *g, DevBatch &out) { return g->finish_next(out); }
bool grace_done(const GraceJoin *g) { return g->done(); }
DevBatch grace_empty_output(GraceJoin *g) { return g->empty_output(); }
const krv_join_spec &grace_spec(const GraceJoin *g) { return g->spec(); }
krv_join_counters grace_counters(const GraceJoin *g) { return g->counters(); }
int64_t grace_spilled_partitions(const GraceJoin *g) { return g->spilled_partitions(); }
int64_t grace_filtered_probe_rows(const GraceJoin *g) { return g->filtered_probe_rows(); }

}  // namespace krv
