// serve.cu -- a request server for join + grouped aggregate queries:
//   SELECT t.g, SUM(p.x), COUNT(*) FROM probe p JOIN table t ON p.k = t.k GROUP BY t.g
// over build tables kept resident on the device, with requests admitted by an
// HBM budget and run in ticks.
//
// Batched mode. A tick is one CUDA graph of three kernels over descriptors
// uploaded before it: clear the accumulators of newly admitted requests; one
// probe + aggregate launch over a device work queue of (request, row range)
// items from every running request, CTAs taking items off an atomic cursor;
// and compaction of the groups of the requests that end in the tick. A tick
// takes at most `tick_rows` probe rows, so a large request spans several
// ticks while requests that arrive meanwhile join the next one and finish
// early (continuous batching). Two ticks may be queued at once: the host
// forms and uploads the next while the device runs the current one.
// Aggregation runs in shared memory for requests with few groups (per-CTA
// 128-bit partial sums merged once per item) and in global memory otherwise.
// An online autotuner tries the candidate kernel shapes (block size, item
// rows, shared-memory group limit) on the first ticks and keeps the fastest.
//
// Plain mode runs each request through the operators one launch at a time:
// HashJoin probe (materialized (x, g) pairs), then HashAggregate.
//
// Reference semantics: HashJoin inner join (crates/krishiv-exec/src/join/
// mod.rs:1014) and HashAggregate SUM(int64) -> int64 with ANSI overflow,
// COUNT(*) (crates/krishiv-exec/src/aggregate/sink.rs:181); the operator
// protocol's NeedMemory for admission (crates/krishiv-exec/src/operator.rs:
// 314-330).
#include <algorithm>
#include <chrono>
#include <deque>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "krv_device.cuh"
#include "ops.h"

namespace krv {

namespace {

constexpr uint32_t kNoRow = 0xFFFFFFFFu;
constexpr int kMaxTickRequests = 512;
constexpr int kMaxTickItems = 16384;
constexpr int kSmemGroupsMax = 2048;  // shared-memory aggregation limit (48 KiB)
constexpr unsigned long long kGroupEmpty = 0x8000000000000000ull;

// How a resident table answers key -> group id:
//  - kDirect: unique keys over a span of at most 4 x rows: gid at key - lo;
//  - kRecords: unique keys: (key, gid) records at the join table's slot
//    positions, probed in the same order, one 16-byte read per step;
//  - kChains: duplicate keys: the join table's slots and newest-first chains.
enum Layout : int32_t { kDirect = 0, kRecords = 1, kChains = 2 };

struct Record {
    long long key;
    int32_t gid;   // -1: empty slot
    int32_t pad;
};

struct TableView {
    const unsigned long long *slots;
    uint64_t mask;
    const uint32_t *next;
    uint64_t seed;
    const long long *keys;
    const int32_t *gid;
    const Record *rec;       // kRecords
    const int32_t *direct;   // kDirect
    long long lo;            // kDirect: smallest key
    unsigned long long span; // kDirect: largest key - lo
    int32_t layout;
    int32_t pad;
};

// One running request, as the tick kernels see it.
struct ReqDev {
    const long long *k;
    const uint8_t *kvalid;
    int64_t kvoff;
    const long long *x;
    TableView t;
    unsigned long long *lo;  // per group: 128-bit SUM (lo, hi) and COUNT(*)
    long long *hi;
    unsigned long long *cnt;
    const long long *gkeys;  // group value of each dense group id
    long long *out_g, *out_sum, *out_cnt;
    int32_t ngroups;
    int32_t use_smem;
};
struct Item {
    int32_t req;
    int32_t pad;
    int64_t row0;
    int64_t rows;
};
struct TickHeader {
    unsigned long long cursor;  // work queue cursor
    int32_t n_items, n_init, n_final, pad;
};
struct Report {
    unsigned long long groups;
    unsigned int overflow;
    unsigned int pad;
};

// Device descriptor area of one tick slot.
struct TickDev {
    TickHeader *hdr;
    ReqDev *reqs;
    Item *items;
    int32_t *init;   // requests whose accumulators start at zero in this tick
    int32_t *final;  // requests that end in this tick
    Report *report;  // one per entry of `final`
};

__device__ __forceinline__ uint32_t table_head(const TableView &t, long long k) {
    const uint64_t g = finalize(hash_word((uint64_t)k), t.seed);
    const unsigned long long tag = g >> 32;
    uint64_t pos = g & t.mask;
    for (uint64_t p = 0; p <= t.mask; p++) {
        const unsigned long long s = __ldg(t.slots + pos);
        if (s == 0) return kNoRow;
        if ((s >> 32) == tag) {
            const uint32_t o = (uint32_t)(s & 0xFFFFFFFFull) - 1u;
            if (__ldg(t.keys + o) == k) return o;
        }
        pos = (pos + 1) & t.mask;
    }
    return kNoRow;
}

__device__ __forceinline__ int record_gid(const TableView &t, long long k) {
    const uint64_t g = finalize(hash_word((uint64_t)k), t.seed);
    uint64_t pos = g & t.mask;
    for (uint64_t p = 0; p <= t.mask; p++) {
        const longlong2 r = __ldg(reinterpret_cast<const longlong2 *>(t.rec + pos));
        const int gid = (int)(int32_t)(r.y & 0xFFFFFFFFll);
        if (gid < 0) return -1;
        if (r.x == k) return gid;
        pos = (pos + 1) & t.mask;
    }
    return -1;
}

__device__ __forceinline__ int direct_gid(const TableView &t, long long k) {
    const unsigned long long off = (unsigned long long)(k - t.lo);
    return off <= t.span ? __ldg(t.direct + off) : -1;
}

// Fills the records of a table with unique keys from its join slots.
__global__ void records_kernel(const unsigned long long *slots, uint64_t n, const long long *keys,
                               const int32_t *gid, Record *rec) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const unsigned long long s = slots[i];
        Record r{0, -1, 0};
        if (s) {
            const uint32_t row = (uint32_t)(s & 0xFFFFFFFFull) - 1u;
            r.key = keys[row];
            r.gid = gid[row];
        }
        rec[i] = r;
    }
}

__global__ void direct_kernel(const long long *keys, const int32_t *gid, int64_t n, long long lo, int32_t *direct) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        direct[(unsigned long long)(keys[i] - lo)] = gid[i];
}

__global__ void tick_init_kernel(TickDev d) {
    const TickHeader h = *d.hdr;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (int i = 0; i < h.n_init; i++) {
        const ReqDev &r = d.reqs[d.init[i]];
        for (int64_t gi = tid; gi < r.ngroups; gi += stride) {
            r.lo[gi] = 0;
            r.hi[gi] = 0;
            r.cnt[gi] = 0;
        }
    }
    for (int64_t i = tid; i < h.n_final; i += stride) d.report[i] = Report{0, 0, 0};
}

template <int THREADS>
__global__ void __launch_bounds__(THREADS) tick_probe_kernel(TickDev d) {
    extern __shared__ __align__(16) uint8_t smem[];
    unsigned long long *s_lo = reinterpret_cast<unsigned long long *>(smem);
    long long *s_hi = reinterpret_cast<long long *>(s_lo + kSmemGroupsMax);
    unsigned long long *s_cnt = reinterpret_cast<unsigned long long *>(s_hi + kSmemGroupsMax);
    __shared__ int s_item;
    const int n_items = d.hdr->n_items;
    constexpr int U = 4;  // rows per thread in flight
    for (;;) {
        if (threadIdx.x == 0) s_item = (int)atomicAdd(&d.hdr->cursor, 1ull);
        __syncthreads();
        const int item = s_item;
        __syncthreads();
        if (item >= n_items) break;
        const Item it = d.items[item];
        const ReqDev R = d.reqs[it.req];
        const bool sm = R.use_smem != 0;
        if (sm) {
            for (int gi = threadIdx.x; gi < R.ngroups; gi += THREADS) {
                s_lo[gi] = 0;
                s_hi[gi] = 0;
                s_cnt[gi] = 0;
            }
            __syncthreads();
        }
        const int64_t end = it.row0 + it.rows;
        for (int64_t base = it.row0; base < end; base += (int64_t)THREADS * U) {
            long long k[U], x[U];
            bool has[U];
            uint32_t row[U];
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int64_t r = base + (int64_t)u * THREADS + threadIdx.x;
                has[u] = r < end && (!R.kvalid || bit_get(R.kvalid, R.kvoff, r));
                k[u] = has[u] ? __ldcs(R.k + r) : 0;
                x[u] = has[u] ? __ldcs(R.x + r) : 0;
            }
            if (R.t.layout != kChains) {
                int g[U];
#pragma unroll
                for (int u = 0; u < U; u++)
                    g[u] = !has[u] ? -1 : R.t.layout == kDirect ? direct_gid(R.t, k[u]) : record_gid(R.t, k[u]);
#pragma unroll
                for (int u = 0; u < U; u++) {
                    if (g[u] < 0) continue;
                    if (sm) {
                        atomic_add_i128_from_i64(s_lo + g[u], s_hi + g[u], x[u]);
                        atomicAdd(s_cnt + g[u], 1ull);
                    } else {
                        atomic_add_i128_from_i64(R.lo + g[u], R.hi + g[u], x[u]);
                        atomicAdd(R.cnt + g[u], 1ull);
                    }
                }
                continue;
            }
#pragma unroll
            for (int u = 0; u < U; u++) row[u] = has[u] ? table_head(R.t, k[u]) : kNoRow;
#pragma unroll
            for (int u = 0; u < U; u++) {
                // every build row with this key (duplicates chain newest-first)
                for (uint32_t b = row[u]; b != kNoRow; b = __ldg(R.t.next + b)) {
                    const int g = __ldg(R.t.gid + b);
                    if (sm) {
                        atomic_add_i128_from_i64(s_lo + g, s_hi + g, x[u]);
                        atomicAdd(s_cnt + g, 1ull);
                    } else {
                        atomic_add_i128_from_i64(R.lo + g, R.hi + g, x[u]);
                        atomicAdd(R.cnt + g, 1ull);
                    }
                }
            }
        }
        if (sm) {
            __syncthreads();
            for (int gi = threadIdx.x; gi < R.ngroups; gi += THREADS) {
                const unsigned long long c = s_cnt[gi];
                if (!c) continue;
                atomic_add_i128(R.lo + gi, R.hi + gi, (int64_t)s_lo[gi], s_hi[gi]);
                atomicAdd(R.cnt + gi, c);
            }
        }
    }
}

// The groups of each request that ends in this tick, compacted.
__global__ void tick_final_kernel(TickDev d) {
    const TickHeader h = *d.hdr;
    const unsigned active = 0xFFFFFFFFu;
    for (int i = 0; i < h.n_final; i++) {
        const ReqDev &r = d.reqs[d.final[i]];
        const int64_t ng = r.ngroups;
        const int64_t stride = (int64_t)gridDim.x * blockDim.x;
        const int64_t span = (ng + 31) / 32 * 32;  // whole warps
        for (int64_t gi = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; gi < span; gi += stride) {
            const bool in = gi < ng && r.cnt[gi] != 0;
            const unsigned long long pos = warp_alloc(&d.report[i].groups, in, active);
            if (!in) continue;
            const unsigned long long l = r.lo[gi];
            const long long hh = r.hi[gi];
            const bool fits64 = (hh == 0 && !(l >> 63)) || (hh == -1 && (l >> 63));
            if (!fits64) atomicOr(&d.report[i].overflow, 1u);
            r.out_g[pos] = r.gkeys[gi];
            r.out_sum[pos] = (long long)l;
            r.out_cnt[pos] = (long long)r.cnt[gi];
        }
    }
}

// ---- the group directory of a resident table ------------------------------------
// Dense ids for the distinct group values of a build table, with no waits:
// keys are claimed by compare-and-swap, ids handed to occupied slots, then
// every row reads its id.
__global__ void gdir_insert_kernel(const long long *g, int64_t n, unsigned long long *keys, uint64_t mask,
                                   unsigned int *has_marker) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const unsigned long long v = (unsigned long long)g[i];
        if (v == kGroupEmpty) {
            *has_marker = 1;
            continue;
        }
        uint64_t p = finalize(hash_word(v), 0x6772) & mask;
        for (uint64_t t = 0; t <= mask; t++) {
            unsigned long long cur = keys[p];
            if (cur == kGroupEmpty) cur = atomicCAS(&keys[p], kGroupEmpty, v);
            if (cur == kGroupEmpty || cur == v) break;
            p = (p + 1) & mask;
        }
    }
}

__global__ void gdir_assign_kernel(const unsigned long long *keys, uint64_t slots, const unsigned int *has_marker,
                                   int32_t *slot_gid, long long *gkeys, unsigned long long *count) {
    const int64_t span = ((int64_t)slots + 1 + 31) / 32 * 32;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < span; i += (int64_t)gridDim.x * blockDim.x) {
        const bool used = i < (int64_t)slots ? keys[i] != kGroupEmpty : (i == (int64_t)slots && *has_marker != 0);
        const unsigned long long id = warp_alloc(count, used, 0xFFFFFFFFu);
        if (!used) continue;
        slot_gid[i] = (int32_t)id;
        gkeys[id] = i < (int64_t)slots ? (long long)keys[i] : (long long)kGroupEmpty;
    }
}

__global__ void gdir_lookup_kernel(const long long *g, int64_t n, const unsigned long long *keys, uint64_t mask,
                                   const int32_t *slot_gid, int32_t *gid) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const unsigned long long v = (unsigned long long)g[i];
        int32_t id = -1;
        if (v == kGroupEmpty) {
            id = slot_gid[mask + 1];
        } else {
            uint64_t p = finalize(hash_word(v), 0x6772) & mask;
            for (uint64_t t = 0; t <= mask; t++) {
                if (keys[p] == v) {
                    id = slot_gid[p];
                    break;
                }
                p = (p + 1) & mask;
            }
        }
        gid[i] = id;
    }
}

uint64_t pow2_at_least(uint64_t v) {
    uint64_t p = 1;
    while (p < v) p <<= 1;
    return p;
}

}  // namespace

// ---- resident tables --------------------------------------------------------------
struct ResidentTable {
    std::unique_ptr<HashJoin> join;  // inner join on key; arena (key, group)
    DBuf gid;                        // dense group id per build row
    DBuf gkeys;                      // group value per dense id
    DBuf rec;                        // kRecords: (key, gid) per join slot
    DBuf direct;                     // kDirect: gid per key - lo
    int32_t layout = kChains;
    long long lo = 0;
    unsigned long long span = 0;
    int64_t rows = 0;
    int64_t ngroups = 0;
};

// ---- the server -------------------------------------------------------------------------
class Server {
  public:
    Server(Runtime *rt, const krv_server_options &o) : rt_(rt), opt_(o) {
        if (opt_.mode != KRV_SERVE_BATCHED && opt_.mode != KRV_SERVE_PLAIN)
            fail(KRV_INVALID_ARGUMENT, "server mode must be KRV_SERVE_BATCHED or KRV_SERVE_PLAIN");
        if (opt_.tick_rows <= 0) opt_.tick_rows = 64ll << 20;
        if (opt_.max_tick_requests <= 0 || opt_.max_tick_requests > kMaxTickRequests)
            opt_.max_tick_requests = kMaxTickRequests;
        DeviceGuard g(rt_);
        for (int s = 0; s < 2; s++) {
            Slot &sl = slots_[s];
            sl.bytes = layout(nullptr);
            sl.dev = DBuf(rt_, sl.bytes);
            KRV_CUDA(cudaHostAlloc(&sl.host, sl.bytes, cudaHostAllocDefault));
            KRV_CUDA(cudaHostAlloc(&sl.report_host, sizeof(Report) * kMaxTickRequests, cudaHostAllocDefault));
            KRV_CUDA(cudaEventCreateWithFlags(&sl.start, cudaEventDefault));
            KRV_CUDA(cudaEventCreateWithFlags(&sl.done, cudaEventDefault));
        }
        build_candidates();
    }
    ~Server() {
        DeviceGuard g(rt_);
        cudaStreamSynchronize(rt_->stream);
        for (auto &kv : graphs_) cudaGraphExecDestroy(kv.second);
        for (auto &sl : slots_) {
            cudaFreeHost(sl.host);
            cudaFreeHost(sl.report_host);
            cudaEventDestroy(sl.start);
            cudaEventDestroy(sl.done);
        }
    }

    int64_t add_table(const DevBatch &b, int key_col, int group_col) {
        DeviceGuard g(rt_);
        const int nc = (int)b.cols.size();
        if (key_col < 0 || key_col >= nc || group_col < 0 || group_col >= nc)
            fail(KRV_INVALID_ARGUMENT, "table column out of range");
        const DevCol &kc = b.cols[key_col], &gc = b.cols[group_col];
        if (kc.type.id != Type::I64 || gc.type.id != Type::I64)
            fail(KRV_UNSUPPORTED, "server tables are (int64 key, int64 group)");
        if (gc.valid) fail(KRV_UNSUPPORTED, "server table groups without NULLs");
        if (b.rows >= (int64_t)0x7FFFFFFF) fail(KRV_UNSUPPORTED, "server tables below 2^31 rows");
        auto t = std::make_shared<ResidentTable>();
        krv_join_spec js;
        krv_join_spec_init(&js);
        js.join_type = KRV_JOIN_INNER;
        js.n_keys = 1;
        js.probe_keys[0] = 0;
        js.build_keys[0] = 0;
        js.runtime_filter = 0;
        js.build_rows_hint = b.rows;
        t->join.reset(new HashJoin(rt_, js));
        DevBatch kb;
        kb.rows = b.rows;
        kb.cols = {kc, gc};
        t->join->build_push(kb);
        t->join->build_finish();
        t->rows = b.rows;
        // group directory
        const int64_t n = b.rows;
        const DevCol &ag = t->join->arena().cols[1];
        const uint64_t cap = pow2_at_least((uint64_t)std::max<int64_t>(2 * n, 16));
        DBuf keys(rt_, cap * 8), slot_gid(rt_, (cap + 1) * 4), marker(rt_, 8), count(rt_, 8);
        fill_empty(keys.as<unsigned long long>(), cap);
        KRV_CUDA(cudaMemsetAsync(marker.get(), 0, 8, rt_->stream));
        KRV_CUDA(cudaMemsetAsync(count.get(), 0, 8, rt_->stream));
        t->gid = DBuf(rt_, (size_t)std::max<int64_t>(n, 1) * 4);
        if (n > 0) {
            gdir_insert_kernel<<<grid_for(rt_, n, 256, 8), 256, 0, rt_->stream>>>(
                static_cast<const long long *>(ag.data), n, keys.as<unsigned long long>(), cap - 1,
                marker.as<unsigned int>());
            rt_->launches++;
            check_launch("gdir_insert_kernel");
        }
        t->gkeys = DBuf(rt_, (size_t)std::max<int64_t>(n, 1) * 8);
        gdir_assign_kernel<<<grid_for(rt_, (int64_t)cap + 1, 256, 8), 256, 0, rt_->stream>>>(
            keys.as<unsigned long long>(), cap, marker.as<unsigned int>(), slot_gid.as<int32_t>(),
            t->gkeys.as<long long>(), count.as<unsigned long long>());
        rt_->launches++;
        check_launch("gdir_assign_kernel");
        if (n > 0) {
            gdir_lookup_kernel<<<grid_for(rt_, n, 256, 8), 256, 0, rt_->stream>>>(
                static_cast<const long long *>(ag.data), n, keys.as<unsigned long long>(), cap - 1,
                slot_gid.as<int32_t>(), t->gid.as<int32_t>());
            rt_->launches++;
            check_launch("gdir_lookup_kernel");
        }
        t->ngroups = (int64_t)read_scalar<unsigned long long>(rt_, count.get());
        choose_layout(*t);
        const int64_t id = next_table_++;
        tables_[id] = t;
        return id;
    }

    // Unique non-NULL keys get a one-read lookup: a direct array when the keys
    // are dense (span at most 4 x rows), else records at the slot positions.
    void choose_layout(ResidentTable &t) {
        HashJoin &j = *t.join;
        const int64_t rows = t.rows;
        const auto c = j.counters();
        t.layout = kChains;
        if (rows <= 0 || j.indexed_rows() != rows || c.build_keys != rows) return;
        const __int128 span = (__int128)j.key_hi() - (__int128)j.key_lo();
        const long long *keys = static_cast<const long long *>(j.arena().cols[0].data);
        if (span >= 0 && span < (__int128)4 * rows && span < ((__int128)1 << 31)) {
            t.lo = j.key_lo();
            t.span = (unsigned long long)span;
            t.direct = DBuf(rt_, ((size_t)span + 1) * 4);
            KRV_CUDA(cudaMemsetAsync(t.direct.get(), 0xFF, ((size_t)span + 1) * 4, rt_->stream));
            direct_kernel<<<grid_for(rt_, rows, 256, 8), 256, 0, rt_->stream>>>(keys, t.gid.as<int32_t>(), rows, t.lo,
                                                                               t.direct.as<int32_t>());
            rt_->launches++;
            check_launch("direct_kernel");
            t.layout = kDirect;
            return;
        }
        const auto tv = j.table_dev();
        const uint64_t n = tv.mask + 1;
        t.rec = DBuf(rt_, n * sizeof(Record));
        records_kernel<<<grid_for(rt_, (int64_t)n, 256, 8), 256, 0, rt_->stream>>>(tv.slots, n, keys,
                                                                                  t.gid.as<int32_t>(), t.rec.as<Record>());
        rt_->launches++;
        check_launch("records_kernel");
        t.layout = kRecords;
    }

    void drop_table(int64_t id) {
        auto it = tables_.find(id);
        if (it == tables_.end()) fail(KRV_INVALID_ARGUMENT, "no table " + std::to_string(id));
        for (auto &r : reqs_)
            if (r.second->table == it->second) fail(KRV_INVALID_ARGUMENT, "table has requests in flight");
        tables_.erase(it);
    }

    int64_t submit(int64_t table, const DevBatch &b, int key_col, int value_col) {
        auto it = tables_.find(table);
        if (it == tables_.end()) fail(KRV_INVALID_ARGUMENT, "no table " + std::to_string(table));
        const int nc = (int)b.cols.size();
        if (key_col < 0 || key_col >= nc || value_col < 0 || value_col >= nc)
            fail(KRV_INVALID_ARGUMENT, "request column out of range");
        if (b.cols[key_col].type.id != Type::I64 || b.cols[value_col].type.id != Type::I64)
            fail(KRV_UNSUPPORTED, "requests are (int64 key, int64 value)");
        if (b.cols[value_col].valid) fail(KRV_UNSUPPORTED, "request values without NULLs");
        auto r = std::make_shared<Req>();
        r->id = next_req_++;
        r->table = it->second;
        r->batch = b;
        r->k = b.cols[key_col];
        r->x = b.cols[value_col];
        r->rows = b.rows;
        r->bytes = (size_t)std::max<int64_t>(it->second->ngroups, 1) * 48;
        if (opt_.hbm_budget_bytes > 0 && (int64_t)r->bytes > opt_.hbm_budget_bytes)
            fail(KRV_NEED_MEMORY, "request state is larger than the server's HBM budget");
        reqs_[r->id] = r;
        pending_.push_back(r);
        return r->id;
    }

    // Retires finished ticks, then forms and launches the next work.
    // Returns the number of requests still queued or running.
    int64_t step(bool wait) {
        DeviceGuard g(rt_);
        if (opt_.mode == KRV_SERVE_PLAIN) {
            if (!pending_.empty()) {
                auto r = pending_.front();
                pending_.pop_front();
                run_plain(*r);
            }
            return (int64_t)pending_.size();
        }
        retire(false);
        if (inflight_.size() < 2 && (!pending_.empty() || !active_.empty())) launch_tick();
        if (wait && !inflight_.empty()) retire(true);
        return (int64_t)(pending_.size() + active_.size() + waiting_final_count());
    }

    // The next finished request: its id and status, and its result columns
    // (group, SUM, COUNT) when it succeeded. False when none has finished.
    bool poll(int64_t &id, krv_status &status, DevBatch &out) {
        if (done_.empty()) return false;
        auto r = done_.front();
        done_.pop_front();
        id = r->id;
        status = r->status;
        out = r->result;
        reqs_.erase(r->id);
        return true;
    }

    krv_server_stats stats() const {
        krv_server_stats s{};
        s.ticks = ticks_;
        s.requests_done = requests_done_;
        s.rows_probed = rows_probed_;
        s.pending = (int64_t)pending_.size();
        s.running = (int64_t)active_.size();
        s.budget_in_use = budget_used_;
        s.tuned = tuned_ ? 1 : 0;
        const Cand &c = cands_[best_];
        s.threads = c.threads;
        s.item_rows = c.item_rows;
        s.smem_groups = c.smem_groups;
        return s;
    }

  private:
    struct Req {
        int64_t id;
        std::shared_ptr<ResidentTable> table;
        DevBatch batch;
        DevCol k, x;
        int64_t rows = 0, next_row = 0;
        size_t bytes = 0;
        DBuf acc, out;  // accumulators (lo, hi, cnt) and output columns
        bool admitted = false;
        bool inited = false;  // accumulators cleared by a tick
        int last_tick = -1;  // tick that processes its last rows
        krv_status status = KRV_OK;
        DevBatch result;
    };
    struct Slot {
        DBuf dev;
        void *host = nullptr;
        Report *report_host = nullptr;
        size_t bytes = 0;
        cudaEvent_t start = nullptr, done = nullptr;
    };
    struct Tick {
        int slot;
        int64_t id;
        int cand;
        int64_t rows;
        std::vector<std::shared_ptr<Req>> finals;
    };
    struct Cand {
        int threads;
        int64_t item_rows;
        int smem_groups;
        double rows_per_ms_sum = 0;
        int runs = 0;
    };

    // Descriptor layout of a slot; fills `d` with device pointers when given.
    size_t layout(TickDev *d, uint8_t *base = nullptr) const {
        size_t off = 0;
        auto take = [&](size_t bytes) {
            const size_t o = off;
            off = (off + bytes + 255) / 256 * 256;
            return base + o;
        };
        uint8_t *hdr = take(sizeof(TickHeader));
        uint8_t *reqs = take(sizeof(ReqDev) * kMaxTickRequests);
        uint8_t *items = take(sizeof(Item) * kMaxTickItems);
        uint8_t *init = take(sizeof(int32_t) * kMaxTickRequests);
        uint8_t *fin = take(sizeof(int32_t) * kMaxTickRequests);
        uint8_t *rep = take(sizeof(Report) * kMaxTickRequests);
        if (d) {
            d->hdr = reinterpret_cast<TickHeader *>(hdr);
            d->reqs = reinterpret_cast<ReqDev *>(reqs);
            d->items = reinterpret_cast<Item *>(items);
            d->init = reinterpret_cast<int32_t *>(init);
            d->final = reinterpret_cast<int32_t *>(fin);
            d->report = reinterpret_cast<Report *>(rep);
        }
        return off;
    }

    void fill_empty(unsigned long long *p, uint64_t n);

    void build_candidates() {
        const int threads[2] = {256, 512};
        const int64_t items[2] = {32 << 10, 128 << 10};
        const int smem[2] = {0, kSmemGroupsMax};
        for (int a : threads)
            for (int64_t b : items)
                for (int c : smem) cands_.push_back(Cand{a, b, c});
        // Fixed shape (no tuning): 512 threads, 128 Ki-row items, shared memory
        // aggregation up to the limit.
        best_ = (int)cands_.size() - 1;
        tuned_ = !opt_.autotune;
    }

    int choose_cand() {
        if (tuned_) return best_;
        for (int i = 0; i < (int)cands_.size(); i++)
            if (cands_[i].runs < 2) return i;
        int b = 0;
        for (int i = 1; i < (int)cands_.size(); i++)
            if (cands_[i].rows_per_ms_sum / cands_[i].runs > cands_[b].rows_per_ms_sum / cands_[b].runs) b = i;
        best_ = b;
        tuned_ = true;
        return best_;
    }

    int64_t waiting_final_count() const {
        int64_t n = 0;
        for (const Tick &t : inflight_) n += (int64_t)t.finals.size();
        return n;
    }

    void admit() {
        while (!pending_.empty() && (int)active_.size() < opt_.max_tick_requests) {
            auto r = pending_.front();
            if (opt_.hbm_budget_bytes > 0 && budget_used_ + (int64_t)r->bytes > opt_.hbm_budget_bytes) break;
            pending_.pop_front();
            const size_t ng = (size_t)std::max<int64_t>(r->table->ngroups, 1);
            r->acc = DBuf(rt_, ng * 24);
            r->out = DBuf(rt_, ng * 24);
            r->admitted = true;
            budget_used_ += (int64_t)r->bytes;
            active_.push_back(r);
        }
    }

    ReqDev req_dev(const Req &r, bool smem) const {
        const ResidentTable &t = *r.table;
        const auto tv = t.join->table_dev();
        const size_t ng = (size_t)std::max<int64_t>(t.ngroups, 1);
        ReqDev d{};
        d.k = static_cast<const long long *>(r.k.data);
        d.kvalid = r.k.valid;
        d.kvoff = r.k.valid_off;
        d.x = static_cast<const long long *>(r.x.data);
        d.t = TableView{tv.slots, tv.mask, tv.next, tv.seed, static_cast<const long long *>(t.join->arena().cols[0].data),
                        t.gid.as<int32_t>(), t.rec.as<Record>(), t.direct.as<int32_t>(), t.lo, t.span, t.layout, 0};
        d.lo = r.acc.as<unsigned long long>();
        d.hi = reinterpret_cast<long long *>(d.lo + ng);
        d.cnt = d.lo + 2 * ng;
        d.gkeys = t.gkeys.as<long long>();
        d.out_g = r.out.as<long long>();
        d.out_sum = d.out_g + ng;
        d.out_cnt = d.out_g + 2 * ng;
        d.ngroups = (int32_t)t.ngroups;
        d.use_smem = smem ? 1 : 0;
        return d;
    }

    void launch_tick() {
        admit();
        if (active_.empty()) return;
        const int s = (int)(tick_seq_ & 1);
        Slot &sl = slots_[s];
        // The staging area and report of this slot belong to the tick two back:
        // it must have been retired (in order) before the slot is reused.
        while (std::any_of(inflight_.begin(), inflight_.end(), [&](const Tick &t) { return t.slot == s; }))
            retire(true);
        const int ci = choose_cand();
        const Cand &c = cands_[ci];
        TickDev hd;
        layout(&hd, static_cast<uint8_t *>(sl.host));
        // Shortest remaining first: small requests finish in the tick they join.
        std::vector<std::shared_ptr<Req>> order(active_.begin(), active_.end());
        std::stable_sort(order.begin(), order.end(), [](const std::shared_ptr<Req> &a, const std::shared_ptr<Req> &b) {
            return a->rows - a->next_row < b->rows - b->next_row;
        });
        int nreq = 0, nitems = 0, ninit = 0, nfinal = 0;
        int64_t budget = opt_.tick_rows, rows = 0;
        Tick tick{s, tick_seq_, ci, 0, {}};
        std::vector<std::shared_ptr<Req>> keep;
        for (auto &r : order) {
            const int64_t left = r->rows - r->next_row;
            int64_t take = std::min(left, budget);
            const int64_t item_rows = c.item_rows;
            const int64_t need_items = (take + item_rows - 1) / item_rows;
            if (nitems + need_items > kMaxTickItems) take = (int64_t)(kMaxTickItems - nitems) * item_rows;
            if (take <= 0 && left > 0) continue;
            const int idx = nreq++;
            const bool smem = r->table->ngroups <= c.smem_groups;
            hd.reqs[idx] = req_dev(*r, smem);
            if (!r->inited) {
                hd.init[ninit++] = idx;
                r->inited = true;
            }
            for (int64_t o = 0; o < take; o += item_rows) {
                Item &it = hd.items[nitems++];
                it.req = idx;
                it.row0 = r->next_row + o;
                it.rows = std::min(item_rows, take - o);
            }
            r->next_row += take;
            budget -= take;
            rows += take;
            if (r->next_row == r->rows) {
                hd.final[nfinal++] = idx;
                tick.finals.push_back(r);
            }
            if (nreq == kMaxTickRequests) break;
        }
        if (nreq == 0) return;
        for (auto &r : tick.finals) active_.erase(std::find(active_.begin(), active_.end(), r));
        hd.hdr->cursor = 0;
        hd.hdr->n_items = nitems;
        hd.hdr->n_init = ninit;
        hd.hdr->n_final = nfinal;
        tick.rows = rows;
        // Upload the used parts of the descriptors, then run the tick's graph.
        TickDev dd;
        layout(&dd, static_cast<uint8_t *>(sl.dev.get()));
        auto up = [&](void *dst, const void *src, size_t bytes) {
            if (bytes) KRV_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, rt_->stream));
        };
        up(dd.hdr, hd.hdr, sizeof(TickHeader));
        up(dd.reqs, hd.reqs, sizeof(ReqDev) * nreq);
        up(dd.items, hd.items, sizeof(Item) * nitems);
        up(dd.init, hd.init, sizeof(int32_t) * ninit);
        up(dd.final, hd.final, sizeof(int32_t) * nfinal);
        KRV_CUDA(cudaEventRecord(sl.start, rt_->stream));
        KRV_CUDA(cudaGraphLaunch(graph_for(s, c.threads, dd, sl), rt_->stream));
        rt_->launches += 3;
        KRV_CUDA(cudaEventRecord(sl.done, rt_->stream));
        tick_seq_++;
        ticks_++;
        rows_probed_ += rows;
        inflight_.push_back(std::move(tick));
    }

    cudaGraphExec_t graph_for(int s, int threads, const TickDev &dd, Slot &sl) {
        const int key = s * 4096 + threads;
        auto it = graphs_.find(key);
        if (it != graphs_.end()) return it->second;
        // The shape of the tick: the kernels read their counts from the
        // descriptors, so one graph serves every tick of this slot and shape.
        const int grid = rt_->sm_count * (threads == 256 ? 4 : 2);
        const size_t smem = (size_t)kSmemGroupsMax * 24;
        if (threads == 256)
            KRV_CUDA(cudaFuncSetAttribute(tick_probe_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        else
            KRV_CUDA(cudaFuncSetAttribute(tick_probe_kernel<512>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        cudaStream_t cs;
        KRV_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            tick_init_kernel<<<rt_->sm_count * 2, 256, 0, cs>>>(dd);
            if (threads == 256) tick_probe_kernel<256><<<grid, 256, smem, cs>>>(dd);
            else tick_probe_kernel<512><<<grid, 512, smem, cs>>>(dd);
            tick_final_kernel<<<rt_->sm_count * 2, 256, 0, cs>>>(dd);
            cudaMemcpyAsync(sl.report_host, dd.report, sizeof(Report) * kMaxTickRequests, cudaMemcpyDeviceToHost, cs);
            e = cudaStreamEndCapture(cs, &graph);
        }
        cudaStreamDestroy(cs);
        if (e != cudaSuccess) fail(KRV_CUDA_ERROR, std::string("tick graph capture: ") + cudaGetErrorString(e));
        cudaGraphExec_t exec = nullptr;
        e = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) fail(KRV_CUDA_ERROR, std::string("tick graph instantiate: ") + cudaGetErrorString(e));
        graphs_[key] = exec;
        return exec;
    }

    void retire(bool block) {
        while (!inflight_.empty()) {
            Tick &t = inflight_.front();
            Slot &sl = slots_[t.slot];
            if (block) {
                KRV_CUDA(cudaEventSynchronize(sl.done));
                block = false;  // wait for the oldest only
            } else {
                const cudaError_t q = cudaEventQuery(sl.done);
                if (q == cudaErrorNotReady) return;
                if (q != cudaSuccess) fail(KRV_CUDA_ERROR, std::string("tick: ") + cudaGetErrorString(q));
            }
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, sl.start, sl.done) == cudaSuccess && ms > 0.f && !tuned_ && t.rows > 0) {
                Cand &c = cands_[t.cand];
                c.rows_per_ms_sum += (double)t.rows / ms;
                c.runs++;
            }
            for (size_t i = 0; i < t.finals.size(); i++) finish_req(*t.finals[i], sl.report_host[i]);
            inflight_.pop_front();
        }
    }

    void finish_req(Req &r, const Report &rep) {
        budget_used_ -= (int64_t)r.bytes;
        r.acc.reset();
        if (rep.overflow && opt_.ansi) {
            r.status = KRV_ARITHMETIC_OVERFLOW;
            r.out.reset();
        } else {
            r.result = result_batch(r, (int64_t)rep.groups);
        }
        r.batch = DevBatch{};
        r.k = DevCol{};
        r.x = DevCol{};
        done_.push_back(reqs_.at(r.id));
        requests_done_++;
    }

    DevBatch result_batch(Req &r, int64_t groups) {
        auto hold = std::make_shared<DBuf>(std::move(r.out));
        const size_t ng = (size_t)std::max<int64_t>(r.table->ngroups, 1);
        DevBatch b;
        b.rows = groups;
        const char *names[3] = {"g", "sum", "count"};
        for (int c = 0; c < 3; c++) {
            DevCol col;
            col.type = DType{Type::I64, 0, 0};
            col.length = groups;
            col.nullable = false;
            col.name = names[c];
            col.hold_data = hold;
            col.data = hold->as<long long>() + c * ng;
            b.cols.push_back(col);
        }
        return b;
    }

    void run_plain(Req &r) {
        // (k, x) JOIN table -> (x, g), then GROUP BY g: SUM(x), COUNT(*)
        DevBatch in;
        in.rows = r.rows;
        in.cols = {r.k, r.x};
        krv_join_spec js = r.table->join->spec();
        js.probe_keys[0] = 0;
        js.n_probe_out = 1;
        js.probe_out[0] = 1;
        js.n_build_out = 1;
        js.build_out[0] = 1;
        HashJoin &j = *r.table->join;
        const krv_join_spec saved = j.spec();
        j.set_probe_shape(js);
        DevBatch pairs;
        try {
            pairs = j.probe(in);
        } catch (...) {
            j.set_probe_shape(saved);
            throw;
        }
        j.set_probe_shape(saved);
        krv_agg_spec as;
        krv_agg_spec_init(&as);
        as.n_group_by = 1;
        as.group_by[0] = 1;
        as.n_aggregates = 2;
        as.aggregates[0] = krv_agg_expr{KRV_AGG_SUM, 0, KRV_AGG_INPUT_RAW, -1, 0, 0, 0, 0};
        as.aggregates[1] = krv_agg_expr{KRV_AGG_COUNT_STAR, 0, KRV_AGG_INPUT_RAW, -1, 0, 0, 0, 0};
        as.ansi = opt_.ansi;
        as.expected_groups = std::max<int64_t>(r.table->ngroups, 1);
        std::unique_ptr<HashAggregate, void (*)(HashAggregate *)> a(make_aggregate(rt_, as), agg_destroy);
        try {
            if (pairs.rows > 0) agg_push(a.get(), pairs);
            agg_finish(a.get());
            DevBatch res = agg_result(a.get());
            if (res.cols.size() != 3) {
                // no joined row reached the aggregate: an empty result of the same shape
                res = DevBatch{};
                for (int c = 0; c < 3; c++) res.cols.push_back(make_col(rt_, DType{Type::I64, 0, 0}, 0, false, ""));
            }
            res.cols[0].name = "g";
            res.cols[1].name = "sum";
            res.cols[2].name = "count";
            r.result = res;
        } catch (const Error &e) {
            if (e.code != KRV_ARITHMETIC_OVERFLOW) throw;
            r.status = KRV_ARITHMETIC_OVERFLOW;
        }
        rows_probed_ += r.rows;
        r.batch = DevBatch{};
        done_.push_back(reqs_.at(r.id));
        requests_done_++;
    }

    Runtime *rt_;
    krv_server_options opt_;
    Slot slots_[2];
    std::map<int, cudaGraphExec_t> graphs_;
    std::vector<Cand> cands_;
    int best_ = 0;
    bool tuned_ = false;
    std::map<int64_t, std::shared_ptr<ResidentTable>> tables_;
    std::map<int64_t, std::shared_ptr<Req>> reqs_;
    std::deque<std::shared_ptr<Req>> pending_, done_;
    std::vector<std::shared_ptr<Req>> active_;
    std::deque<Tick> inflight_;
    int64_t next_table_ = 1, next_req_ = 1, tick_seq_ = 0;
    int64_t ticks_ = 0, requests_done_ = 0, rows_probed_ = 0, budget_used_ = 0;
};

namespace {
__global__ void fill_u64_kernel(unsigned long long *p, uint64_t n, unsigned long long v) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        p[i] = v;
}
}  // namespace

void Server::fill_empty(unsigned long long *p, uint64_t n) {
    fill_u64_kernel<<<grid_for(rt_, (int64_t)n, 256, 8), 256, 0, rt_->stream>>>(p, n, kGroupEmpty);
    rt_->launches++;
    check_launch("fill_u64_kernel");
}

Server *make_server(Runtime *rt, const krv_server_options &o) { return new Server(rt, o); }
int64_t server_add_table(Server *s, const DevBatch &b, int key_col, int group_col) {
    return s->add_table(b, key_col, group_col);
}
void server_drop_table(Server *s, int64_t id) { s->drop_table(id); }
int64_t server_submit(Server *s, int64_t table, const DevBatch &b, int key_col, int value_col) {
    return s->submit(table, b, key_col, value_col);
}
int64_t server_step(Server *s, bool wait) { return s->step(wait); }
bool server_poll(Server *s, int64_t &id, krv_status &status, DevBatch &out) { return s->poll(id, status, out); }
krv_server_stats server_stats(const Server *s) { return s->stats(); }
void server_destroy(Server *s) { delete s; }

}  // namespace krv
