// star.cu -- the star-join pipeline: two dimension builds that publish
// runtime key filters, the fact side filtered by both and probed against both
// tables, and a grouped float64 sum of price * (1 - discount).
//
// Two forms of the same plan:
//  - fused: the fact side is one kernel; each fact row is read once, tested
//    against dimension B's Bloom filter (staged in shared memory) and A's
//    (L2-resident), probed against both tables only when both filters pass,
//    and its value added to a per-CTA shared-memory accumulator of its group;
//    CTAs merge their accumulators at the end with compensated atomics;
//  - plain: one operator per launch through the operator classes (runtime
//    filter evaluate, compaction, join probe, join probe, projection,
//    aggregate), each materializing its output in HBM.
//
// Reference plan pieces: HashJoinNode (crates/krishiv-exec/src/join/
// mod.rs:1188-1211), runtime filters published by the build
// (join/build.rs:482) and applied in the scan's row stage
// (crates/krishiv-exec/src/operators/runtime_filter.rs:1-45), HashAggregate
// (crates/krishiv-exec/src/aggregate/sink.rs:181).
//
// The per-row value is computed as the CPU does it: (double)price, then
// 1.0 - discount and one product, each rounded (no fused multiply-add).
#include <algorithm>
#include <climits>
#include <functional>
#include <memory>

#include "krv_device.cuh"
#include "krv_filter.cuh"
#include "ops.h"
#include "star_fused.cuh"

namespace krv {

namespace {

constexpr long long kAttrEmpty = (long long)0x8080808080808080ULL;

// Rows of a dimension with pred == value: their key and attribute, compacted
// (the filter below the join build). Each warp takes 16 x 32 rows of the
// block's tile, reading pred once per row (one ballot per 32 rows); the
// block reserves its tile's output with one atomic, so the shared counter
// sees one update per 4K rows; the survivors are written in row order.
// `range` (when given) gets the selected keys' min and max, `arange` the
// selected attributes' (one update per block each). Without `pred` every row
// is selected; without `attr` the attribute written is 0.
constexpr int kSelectSteps = 16;
constexpr int kSelectThreads = 256;
constexpr int kSelectTile = kSelectThreads * kSelectSteps;
__global__ void __launch_bounds__(kSelectThreads) dim_select_kernel(const long long *key, const int32_t *pred,
                                                                    const int32_t *attr, int64_t n, int32_t value,
                                                                    long long *okey, int32_t *oattr,
                                                                    unsigned long long *count, long long *range,
                                                                    long long *arange) {
    __shared__ unsigned s_tot[kSelectThreads / 32];
    __shared__ unsigned long long s_base;
    __shared__ long long s_rng[4][kSelectThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    long long lo = LLONG_MAX, hi = LLONG_MIN, alo = LLONG_MAX, ahi = LLONG_MIN;
    for (int64_t t0 = (int64_t)blockIdx.x * kSelectTile; t0 < n; t0 += (int64_t)gridDim.x * kSelectTile) {
        const int64_t c0 = t0 + (int64_t)warp * 32 * kSelectSteps;
        unsigned ballots[kSelectSteps];
        unsigned total = 0;
#pragma unroll
        for (int s = 0; s < kSelectSteps; s++) {
            const int64_t i = c0 + s * 32 + lane;
            ballots[s] = __ballot_sync(0xFFFFFFFFu, i < n && (!pred || pred[i] == value));
            total += __popc(ballots[s]);
        }
        if (lane == 0) s_tot[warp] = total;
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned acc = 0;
            for (int w = 0; w < kSelectThreads / 32; w++) {
                const unsigned t = s_tot[w];
                s_tot[w] = acc;
                acc += t;
            }
            s_base = acc ? atomicAdd(count, (unsigned long long)acc) : 0ull;
        }
        // The selected rows' keys and attributes, all loads issued before
        // any store (a load placed after a store to the output would wait
        // for it: the compiler cannot tell the arrays apart).
        // Half the steps at a time, to stay within the registers.
        constexpr int kHalf = kSelectSteps / 2;
        __syncthreads();
        unsigned long long base = s_base + s_tot[warp];
#pragma unroll
        for (int h = 0; h < 2; h++) {
            long long ks[kHalf];
            int32_t as[kHalf];
#pragma unroll
            for (int q = 0; q < kHalf; q++) {
                const int s = h * kHalf + q;
                const int64_t i = c0 + s * 32 + lane;
                const bool mine = (ballots[s] >> lane) & 1u;
                ks[q] = mine ? key[i] : 0;
                as[q] = mine && attr ? attr[i] : 0;
            }
#pragma unroll
            for (int q = 0; q < kHalf; q++) {
                const int s = h * kHalf + q;
                if ((ballots[s] >> lane) & 1u) {
                    const unsigned long long pos = base + __popc(ballots[s] & lanemask_lt());
                    const long long k = ks[q];
                    const int32_t a = as[q];
                    okey[pos] = k;
                    oattr[pos] = a;
                    lo = k < lo ? k : lo;
                    hi = k > hi ? k : hi;
                    alo = a < alo ? a : alo;
                    ahi = a > ahi ? a : ahi;
                }
                base += __popc(ballots[s]);
            }
        }
        __syncthreads();  // s_tot is rewritten by the next tile
    }
    if (!range && !arange) return;
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        lo = min(lo, __shfl_xor_sync(0xFFFFFFFFu, lo, d));
        hi = max(hi, __shfl_xor_sync(0xFFFFFFFFu, hi, d));
        alo = min(alo, __shfl_xor_sync(0xFFFFFFFFu, alo, d));
        ahi = max(ahi, __shfl_xor_sync(0xFFFFFFFFu, ahi, d));
    }
    if (lane == 0) {
        s_rng[0][warp] = lo;
        s_rng[1][warp] = hi;
        s_rng[2][warp] = alo;
        s_rng[3][warp] = ahi;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < kSelectThreads / 32; w++) {
            lo = min(lo, s_rng[0][w]);
            hi = max(hi, s_rng[1][w]);
            alo = min(alo, s_rng[2][w]);
            ahi = max(ahi, s_rng[3][w]);
        }
        if (lo <= hi && range) {
            atomicMin(range, lo);
            atomicMax(range + 1, hi);
        }
        if (alo <= ahi && arange) {
            atomicMin(arange, alo);
            atomicMax(arange + 1, ahi);
        }
    }
}

// Dense group ids of the attribute values: one small open-addressing table.
__global__ void attr_gid_kernel(const int32_t *attr, int64_t n, long long *tkeys, int32_t *tgid, uint64_t mask,
                                int32_t *gid_out, int32_t *gattr, unsigned int *ngroups, uint32_t *status) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const long long k = attr[i];
        uint64_t pos = hash_word((uint64_t)k) & mask;
        int32_t g = -1;
        for (uint64_t p = 0; p <= mask; p++) {
            // A plain read first: few distinct values, so nearly every row finds
            // its value already there and needs no atomic.
            long long cur = __ldcg(tkeys + pos);
            if (cur == kAttrEmpty)
                cur = (long long)atomicCAS(reinterpret_cast<unsigned long long *>(tkeys + pos),
                                           (unsigned long long)kAttrEmpty, (unsigned long long)k);
            if (cur == kAttrEmpty) {
                g = (int32_t)atomicAdd(ngroups, 1u);
                gattr[g] = (int32_t)k;
                __threadfence();
                atomicExch(tgid + pos, g);
                break;
            }
            if (cur == k) {
                for (int it = 0; it < (1 << 22); it++) {
                    g = *reinterpret_cast<volatile int32_t *>(tgid + pos);
                    if (g >= 0) break;
                    __nanosleep(20);
                }
                if (g < 0) atomicOr(status, ST_TIMEOUT);
                break;
            }
            pos = (pos + 1) & mask;
        }
        gid_out[i] = g < 0 ? 0 : g;
    }
}

// The fast build's device-driven steps. `ctl` words (int64): [0..1] selected
// rows per dimension, [2..5] their key (lo, hi), [6..7] the attribute (lo, hi)
// of both dimensions, [8..9] duplicate-key flags, [10] group ids handed out by
// the attribute table, [11] status bits.
constexpr int kCtlWords = 12;
constexpr unsigned long long kMaxDirectSpan = 1ull << 26;  // key values a direct index covers
constexpr long long kDirectAttrSpan = 1024;                // attribute values that are their own group id

// Marks [0, hi - lo] of a direct index empty (-1), when the span qualifies.
__global__ void direct_fill_kernel(unsigned long long *direct, const long long *range) {
    const long long lo = range[0], hi = range[1];
    if (lo > hi) return;
    const unsigned long long span = (unsigned long long)(hi - lo);
    if (span >= kMaxDirectSpan) return;
    const unsigned long long words = span / 4 + 1;  // four int16 entries per word
    for (unsigned long long w = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; w < words;
         w += (unsigned long long)gridDim.x * blockDim.x)
        direct[w] = ~0ull;
}

// The group id of attribute value k in the shared attribute table (claimed
// when new; readers wait, bounded, for its id).
__device__ __forceinline__ int32_t attr_gid_of(long long k, long long *tkeys, int32_t *tgid, uint64_t mask,
                                               int32_t *gattr, unsigned int *ngroups, uint32_t *status) {
    uint64_t pos = hash_word((uint64_t)k) & mask;
    for (uint64_t p = 0; p <= mask; p++) {
        long long cur = __ldcg(tkeys + pos);
        if (cur == kAttrEmpty)
            cur = (long long)atomicCAS(reinterpret_cast<unsigned long long *>(tkeys + pos),
                                       (unsigned long long)kAttrEmpty, (unsigned long long)k);
        if (cur == kAttrEmpty) {
            const int32_t g = (int32_t)atomicAdd(ngroups, 1u);
            gattr[g] = (int32_t)k;
            __threadfence();
            atomicExch(tgid + pos, g);
            return g;
        }
        if (cur == k) {
            for (int it = 0; it < (1 << 22); it++) {
                const int32_t g = *reinterpret_cast<volatile int32_t *>(tgid + pos);
                if (g >= 0) return g;
                __nanosleep(20);
            }
            atomicOr(status, ST_TIMEOUT);
            return 0;
        }
        pos = (pos + 1) & mask;
    }
    return 0;
}

// Each selected row's group id at its key's place of the direct index: the
// attribute itself (minus the lowest) when both dimensions' attributes span
// fewer than kDirectAttrSpan values, else the attribute table's id. Two rows
// with one key set the dimension's duplicate flag.
__global__ void dim_index_fast_kernel(const long long *key, const int32_t *attr, long long *ctl, int d,
                                      int grouping, unsigned short *direct, long long *tkeys, int32_t *tgid,
                                      uint64_t mask, int32_t *gattr) {
    const unsigned long long n = (unsigned long long)ctl[d];
    const long long lo = ctl[2 + 2 * d], hi = ctl[3 + 2 * d];
    if (lo > hi || (unsigned long long)(hi - lo) >= kMaxDirectSpan) return;
    const long long alo = ctl[6], ahi = ctl[7];
    const bool own = ahi - alo < kDirectAttrSpan;
    unsigned int *dup = reinterpret_cast<unsigned int *>(ctl + 8 + d);
    unsigned int *ngroups = reinterpret_cast<unsigned int *>(ctl + 10);
    uint32_t *status = reinterpret_cast<uint32_t *>(ctl + 11);
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        const long long a = attr[i];
        // the other dimension's entries only mark its keys present
        const int32_t g = !grouping ? 0 : own ? (int32_t)(a - alo) : attr_gid_of(a, tkeys, tgid, mask, gattr, ngroups, status);
        const unsigned long long off = (unsigned long long)(key[i] - lo);
        const unsigned short old = atomicCAS(direct + off, (unsigned short)0xFFFFu, (unsigned short)g);
        if (old != (unsigned short)0xFFFFu) atomicOr(dup, 1u);
    }
}

// gattr[g] = lo + g: the attribute values that are their own group ids.
__global__ void attr_iota_kernel(int32_t *gattr, long long lo, int G) {
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < G; g += gridDim.x * blockDim.x) gattr[g] = (int32_t)(lo + g);
}

// The result rows: groups with joined rows in group-id order, (attr, sum of
// the double-double accumulator rounded once, sum valid unless every value
// was NULL). One block; out[0] = rows, out[1] = NULL sums, out[2..4] the
// scan statistics.
constexpr int kResultThreads = 1024;
__global__ void __launch_bounds__(kResultThreads) star_result_kernel(int G, const int32_t *gattr, const double *hi,
                                                                     const double *lo, const unsigned long long *cnt,
                                                                     const unsigned long long *nulls,
                                                                     const unsigned long long *stats, int32_t *oattr,
                                                                     double *osum, uint32_t *ovalid,
                                                                     unsigned long long *out) {
    __shared__ unsigned s_warp[kResultThreads / 32];
    __shared__ unsigned s_base, s_nulls;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        s_base = 0;
        s_nulls = 0;
    }
    for (int w = threadIdx.x; w < (G + 31) / 32; w += kResultThreads) ovalid[w] = 0;
    __syncthreads();
    for (int g0 = 0; g0 < G; g0 += kResultThreads) {
        const int g = g0 + threadIdx.x;
        const bool has = g < G && cnt[g] > 0;
        const unsigned b = __ballot_sync(0xFFFFFFFFu, has);
        if (lane == 0) s_warp[warp] = __popc(b);
        __syncthreads();
        unsigned before = s_base;
        for (int w = 0; w < warp; w++) before += s_warp[w];
        const unsigned pos = before + __popc(b & lanemask_lt());
        if (has) {
            const double h = hi[g];
            oattr[pos] = gattr[g];
            osum[pos] = isfinite(h) ? __dadd_rn(h, lo[g]) : h;
            if (cnt[g] > nulls[g]) atomicOr(ovalid + (pos >> 5), 1u << (pos & 31));
            else atomicAdd(&s_nulls, 1u);
        }
        __syncthreads();
        if (threadIdx.x == 0)
            for (int w = 0; w < kResultThreads / 32; w++) s_base += s_warp[w];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = s_base;
        out[1] = s_nulls;
        out[2] = stats[0];
        out[3] = stats[1];
        out[4] = stats[2];
    }
}

// Plain form helpers: the scan's row stage keeps rows passing both filters
// (a null `pass_*` passes every row) whose keys are both valid (a NULL key
// never joins). `ovv`, when given (zeroed words), gets bit `pos` set where
// the kept row's price and discount are both valid.
struct FactValid {
    const uint8_t *v[4];  // fk_a, fk_b, price, discount (null: no NULLs)
    int64_t o[4];
};
__global__ void __launch_bounds__(256) compact4_kernel(const uint32_t *pass_a, const uint32_t *pass_b, int64_t n,
                                                       FactValid V, const long long *c0, const long long *c1,
                                                       const long long *c2, const double *c3, long long *o0,
                                                       long long *o1, long long *o2, double *o3, uint32_t *ovv,
                                                       unsigned long long *count) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t base = blockIdx.x * (int64_t)blockDim.x; base < n; base += stride) {
        const int64_t i = base + threadIdx.x;
        bool ok = false;
        if (i < n) {
            const uint32_t a = pass_a ? pass_a[i >> 5] : ~0u, b = pass_b ? pass_b[i >> 5] : ~0u;
            ok = ((a & b) >> (i & 31)) & 1u;
            ok = ok && bit_get(V.v[0], V.o[0], i) && bit_get(V.v[1], V.o[1], i);
        }
        const unsigned ballot = __ballot_sync(0xFFFFFFFFu, ok);
        unsigned long long first = 0;
        if (lane_id() == 0 && ballot) first = atomicAdd(count, (unsigned long long)__popc(ballot));
        first = __shfl_sync(0xFFFFFFFFu, first, 0);
        const unsigned long long pos = first + __popc(ballot & lanemask_lt());
        if (ok) {
            o0[pos] = c0[i];
            o1[pos] = c1[i];
            o2[pos] = c2[i];
            o3[pos] = c3[i];
            if (ovv && bit_get(V.v[2], V.o[2], i) && bit_get(V.v[3], V.o[3], i))
                atomicOr(ovv + (pos >> 5), 1u << (pos & 31));
        }
    }
}

// Plain form: the projection price * (1 - discount).
__global__ void project_kernel(const long long *price, const double *disc, int64_t n, double *out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = __dmul_rn((double)price[i], __dsub_rn(1.0, disc[i]));
}

}  // namespace

class StarPipeline {
  public:
    StarPipeline(Runtime *rt, const krv_star_spec &s) : rt_(rt), spec_(s) {
        if (s.group_by != 0 && s.group_by != 1) fail(KRV_INVALID_ARGUMENT, "group_by is 0 (dim a) or 1 (dim b)");
        if (s.mode != KRV_STAR_FUSED && s.mode != KRV_STAR_PLAIN) fail(KRV_INVALID_ARGUMENT, "unknown star mode");
        for (int d = 0; d < 2; d++) set_dim_cols(d, s.dim_key, s.dim_pred, s.dim_attr);
    }

    struct Dim {
        std::unique_ptr<HashJoin> join;  // inner join on key, build columns (key, attr, gid)
        DBuf key, attr, gid;
        int64_t rows = 0;
    };

    // Dimension d's columns: key, predicate (-1: every row qualifies, the
    // rows being those of a join's finished build side) and attribute (-1 on
    // the dimension not grouped by).
    void set_dim_cols(int d, int key, int pred, int attr) {
        dkey_[d] = key;
        dpred_[d] = pred;
        dattr_[d] = attr;
    }
    void check_dim(const DevBatch &b, int d) const {
        const int c_key = dkey_[d], c_pred = dpred_[d], c_attr = dattr_[d];
        const int nc = (int)b.cols.size();
        if (c_key < 0 || c_key >= nc || c_pred < -1 || c_pred >= nc || c_attr < -1 || c_attr >= nc ||
            (c_attr < 0 && d == spec_.group_by))
            fail(KRV_INVALID_ARGUMENT, "dimension column out of range");
        if (b.cols[c_key].type.id != Type::I64 || (c_pred >= 0 && b.cols[c_pred].type.id != Type::I32) ||
            (c_attr >= 0 && b.cols[c_attr].type.id != Type::I32))
            fail(KRV_UNSUPPORTED, "star dimension columns are (int64 key, int32 pred, int32 attr)");
        if (b.cols[c_key].valid || (c_pred >= 0 && b.cols[c_pred].valid) || (c_attr >= 0 && b.cols[c_attr].valid))
            fail(KRV_UNSUPPORTED, "star dimension columns without NULLs");
    }
    const int32_t *dim_pred(const DevBatch &b, int d) const {
        return dpred_[d] >= 0 ? static_cast<const int32_t *>(b.cols[dpred_[d]].data) : nullptr;
    }
    const int32_t *dim_attr(const DevBatch &b, int d) const {
        return dattr_[d] >= 0 ? static_cast<const int32_t *>(b.cols[dattr_[d]].data) : nullptr;
    }

    // The fused plan's build when both dimensions have unique keys over spans
    // of at most 2^26 values (the common star schema): select both, then the
    // direct indexes (key -> group id, int16), with every step sized from the
    // selection on the device; one host read of the counts, ranges and
    // duplicate flags; then the key filters from the selection's count and
    // range. False (nothing kept) when a dimension does not qualify: the
    // join-table build runs.
    int select_grid(int64_t n) const {
        return (int)std::max<int64_t>(1, std::min<int64_t>(8 * rt_->sm_count, ceil_div(n, kSelectTile)));
    }
    bool build_fast(const DevBatch *dims[2], const int32_t values[2]) {
        struct Sel {
            DBuf key, attr;
            int64_t rows = 0;
            long long lo = 0, hi = -1;
        } sel[2];
        DBuf ctl(rt_, kCtlWords * 8);
        const long long init[kCtlWords] = {0, 0, LLONG_MAX, LLONG_MIN, LLONG_MAX, LLONG_MIN, LLONG_MAX, LLONG_MIN,
                                           0, 0, 0, 0};
        KRV_CUDA(cudaMemcpyAsync(ctl.get(), init, sizeof(init), cudaMemcpyHostToDevice, rt_->stream));
        for (int d = 0; d < 2; d++) {
            const DevBatch &b = *dims[d];
            const int64_t n = b.rows;
            sel[d].key = DBuf(rt_, (size_t)std::max<int64_t>(n, 1) * 8);
            sel[d].attr = DBuf(rt_, (size_t)std::max<int64_t>(n, 1) * 4);
            if (n > 0) {
                dim_select_kernel<<<select_grid(n), kSelectThreads, 0, rt_->stream>>>(
                    static_cast<const long long *>(b.cols[dkey_[d]].data), dim_pred(b, d), dim_attr(b, d), n,
                    values[d], sel[d].key.as<long long>(),
                    sel[d].attr.as<int32_t>(), ctl.as<unsigned long long>() + d, ctl.as<long long>() + 2 + 2 * d,
                    d == spec_.group_by ? ctl.as<long long>() + 6 : nullptr);
                rt_->launches++;
                check_launch("dim_select_kernel");
            }
        }
        for (int d = 0; d < 2; d++) {
            if (!direct_full_[d].get()) direct_full_[d] = DBuf(rt_, (size_t)(kMaxDirectSpan + 4) * 2);
            direct_fill_kernel<<<2 * rt_->sm_count, 256, 0, rt_->stream>>>(direct_full_[d].as<unsigned long long>(),
                                                                           ctl.as<long long>() + 2 + 2 * d);
            rt_->launches++;
            check_launch("direct_fill_kernel");
        }
        for (int d = 0; d < 2; d++) {
            const int64_t n = dims[d]->rows;
            if (n <= 0) continue;
            dim_index_fast_kernel<<<grid_for(rt_, std::max<int64_t>(1, n / 16), 256, 8), 256, 0, rt_->stream>>>(
                sel[d].key.as<long long>(), sel[d].attr.as<int32_t>(), ctl.as<long long>(), d,
                d == spec_.group_by ? 1 : 0, direct_full_[d].as<unsigned short>(), gkeys_.as<long long>(),
                gtab_.as<int32_t>(), gmask_,
                gattr_.as<int32_t>());
            rt_->launches++;
            check_launch("dim_index_fast_kernel");
        }
        long long got[kCtlWords];
        read_device(rt_, ctl.get(), sizeof(got), got);
        if ((uint32_t)got[11] & ST_TIMEOUT) fail(KRV_TIMEOUT, "star build: a wait for a group id gave up");
        for (int d = 0; d < 2; d++) {
            sel[d].rows = got[d];
            sel[d].lo = got[2 + 2 * d];
            sel[d].hi = got[3 + 2 * d];
            if (sel[d].rows <= 0) return false;
            const __int128 span = (__int128)sel[d].hi - (__int128)sel[d].lo;
            if (span < 0 || span >= (__int128)kMaxDirectSpan) return false;
            if ((uint32_t)got[8 + d]) return false;  // duplicate dimension keys: the join-table build
        }
        const long long alo = got[6], ahi = got[7];
        if (ahi - alo < kDirectAttrSpan) {
            ngroups_host_ = (int)(ahi - alo + 1);
            attr_iota_kernel<<<1, 1024, 0, rt_->stream>>>(gattr_.as<int32_t>(), alo, ngroups_host_);
            rt_->launches++;
            check_launch("attr_iota_kernel");
        } else {
            ngroups_host_ = (int)(uint32_t)got[10];
        }
        if (ngroups_host_ > (int)gmask_ / 2) fail(KRV_UNSUPPORTED, "more than 32768 distinct attribute values");
        // key filters from the selection's stats (keys unique: distinct = rows)
        std::shared_ptr<KeyFilterImpl> filt[2];
        if (spec_.use_filters) {
            krv_key_filter_options fo;
            krv_key_filter_options_default(&fo);
            for (int d = 0; d < 2; d++) {
                DevCol kc;
                kc.type = DType{Type::I64, 0, 0};
                kc.length = sel[d].rows;
                kc.nullable = false;
                kc.data = sel[d].key.get();
                const KeyStats ks{sel[d].rows, sel[d].rows, sel[d].lo, sel[d].hi};
                filt[d] = build_key_filter(rt_, fo, kc, &ks);
            }
        }
        for (int d = 0; d < 2; d++) {
            dims_[d] = Dim{};
            dims_[d].rows = sel[d].rows;
            filt_[d] = filt[d];
            direct_[d] = StarDirect{direct_full_[d].get(), sel[d].lo, (unsigned long long)(sel[d].hi - sel[d].lo), 2};
        }
        counters_.dim_a_keys = sel[0].rows;
        counters_.dim_b_keys = sel[1].rows;
        return true;
    }

    void build_dim(const DevBatch &d, int di, int32_t value, Dim &out) {
        check_dim(d, di);
        const int64_t n = d.rows;
        out.key = DBuf(rt_, (size_t)std::max<int64_t>(n, 1) * 8);
        out.attr = DBuf(rt_, (size_t)std::max<int64_t>(n, 1) * 4);
        DBuf cnt(rt_, 8);
        KRV_CUDA(cudaMemsetAsync(cnt.get(), 0, 8, rt_->stream));
        if (n > 0) {
            dim_select_kernel<<<select_grid(n), kSelectThreads, 0, rt_->stream>>>(
                static_cast<const long long *>(d.cols[dkey_[di]].data), dim_pred(d, di), dim_attr(d, di), n, value,
                out.key.as<long long>(), out.attr.as<int32_t>(), cnt.as<unsigned long long>(), nullptr, nullptr);
            rt_->launches++;
            check_launch("dim_select_kernel");
        }
        out.rows = (int64_t)read_scalar<unsigned long long>(rt_, cnt.get());
        // Dense group ids of the grouping dimension's attribute (the other's
        // are never read: zeros).
        out.gid = DBuf(rt_, (size_t)std::max<int64_t>(out.rows, 1) * 4);
        if (di != spec_.group_by) KRV_CUDA(cudaMemsetAsync(out.gid.get(), 0, out.gid.bytes(), rt_->stream));
        if (out.rows > 0 && di == spec_.group_by) {
            attr_gid_kernel<<<grid_for(rt_, out.rows, 256, 8), 256, 0, rt_->stream>>>(
                out.attr.as<int32_t>(), out.rows, gkeys_.as<long long>(), gtab_.as<int32_t>(), gmask_, out.gid.as<int32_t>(),
                gattr_.as<int32_t>(), ngroups_.as<unsigned int>(), status_word(rt_));
            rt_->launches++;
            check_launch("attr_gid_kernel");
        }
        // The compacted (key, attr, gid) columns become the join's build arena
        // as they are: no copy.
        DevBatch b;
        b.rows = out.rows;
        auto own = [&](DBuf &buf, Type t, const char *name) {
            DevCol c;
            c.type = DType{t, 0, 0};
            c.length = out.rows;
            c.name = name;
            c.nullable = false;
            c.hold_data = std::make_shared<DBuf>(std::move(buf));
            c.data = c.hold_data->get();
            return c;
        };
        b.cols = {own(out.key, Type::I64, "key"), own(out.attr, Type::I32, "attr"), own(out.gid, Type::I32, "gid")};
        krv_join_spec js;
        krv_join_spec_init(&js);
        js.join_type = KRV_JOIN_INNER;
        js.n_keys = 1;
        js.probe_keys[0] = 0;
        js.build_keys[0] = 0;
        js.runtime_filter = spec_.use_filters;
        out.join.reset(new HashJoin(rt_, js));
        out.join->build_adopt(std::move(b));
        out.join->build_finish();
    }

    void build(const DevBatch &a, const DevBatch &b) {
        DeviceGuard g(rt_);
        // Attribute -> dense group id table (at most 2^16 distinct values).
        gmask_ = (1u << 16) - 1;
        gkeys_ = DBuf(rt_, (gmask_ + 1) * 8);
        gtab_ = DBuf(rt_, (gmask_ + 1) * 4);
        gattr_ = DBuf(rt_, (gmask_ + 1) * 4);
        ngroups_ = DBuf(rt_, 8);
        KRV_CUDA(cudaMemsetAsync(gkeys_.get(), 0x80, (gmask_ + 1) * 8, rt_->stream));
        KRV_CUDA(cudaMemsetAsync(gtab_.get(), 0xFF, (gmask_ + 1) * 4, rt_->stream));
        KRV_CUDA(cudaMemsetAsync(ngroups_.get(), 0, 8, rt_->stream));
        clear_status(rt_);
        dims_[0] = Dim{};
        dims_[1] = Dim{};
        filt_[0].reset();
        filt_[1].reset();
        for (int d = 0; d < 2; d++) {
            direct_[d] = StarDirect{nullptr, 0, 0, 0};
            direct_buf_[d].reset();
        }
        check_dim(a, 0);
        check_dim(b, 1);
        const DevBatch *dims[2] = {&a, &b};
        const int32_t values[2] = {spec_.pred_a, spec_.pred_b};
        const bool fast = spec_.mode == KRV_STAR_FUSED && build_fast(dims, values);
        if (!fast) {
            // The join-table build: reset the group ids the fast attempt made.
            KRV_CUDA(cudaMemsetAsync(gkeys_.get(), 0x80, (gmask_ + 1) * 8, rt_->stream));
            KRV_CUDA(cudaMemsetAsync(gtab_.get(), 0xFF, (gmask_ + 1) * 4, rt_->stream));
            KRV_CUDA(cudaMemsetAsync(ngroups_.get(), 0, 8, rt_->stream));
            clear_status(rt_);
            // Only the grouping dimension's attribute names groups; the other's
            // ids are never read.
            build_dim(a, 0, spec_.pred_a, dims_[0]);
            build_dim(b, 1, spec_.pred_b, dims_[1]);
            if (take_status(rt_) & ST_TIMEOUT) fail(KRV_TIMEOUT, "star build: a wait for a group id gave up");
            ngroups_host_ = (int)read_scalar<unsigned int>(rt_, ngroups_.get());
            if (ngroups_host_ > (int)gmask_ / 2) fail(KRV_UNSUPPORTED, "more than 32768 distinct attribute values");
            filt_[0] = dims_[0].join->key_filter();
            filt_[1] = dims_[1].join->key_filter();
        }
        const size_t G = (size_t)std::max(ngroups_host_, 1);
        sum_hi_ = DBuf(rt_, G * 8);
        sum_lo_ = DBuf(rt_, G * 8);
        cnt_ = DBuf(rt_, G * 8);
        nulls_ = DBuf(rt_, G * 8);
        stats_ = DBuf(rt_, 32);
        reset();
        if (!fast) {
            counters_.dim_a_keys = dims_[0].join->counters().build_keys;
            counters_.dim_b_keys = dims_[1].join->counters().build_keys;
        }
        auto fa = filt_[0], fb = filt_[1];
        counters_.filter_a_form = fa ? fa->info.form : -1;
        counters_.filter_b_form = fb ? fb->info.form : -1;
        counters_.filter_a_bytes = fa ? fa->info.bloom_bytes : 0;
        counters_.filter_b_bytes = fb ? fb->info.bloom_bytes : 0;
        if (spec_.mode == KRV_STAR_FUSED && spec_.use_filters) {
            if (fa) build_bits(0, *fa);
            if (fb) build_bits(1, *fb);
        }
        if (spec_.mode == KRV_STAR_FUSED && !fast) {
            build_direct(0);
            build_direct(1);
        }
        built_ = true;
    }

    void reset() {
        counters_.fact_rows = 0;
        counters_.passed_filters = 0;
        counters_.joined_rows = 0;
        if (!sum_hi_.get()) return;  // nothing built yet
        const size_t G = (size_t)std::max(ngroups_host_, 1);
        KRV_CUDA(cudaMemsetAsync(sum_hi_.get(), 0, G * 8, rt_->stream));
        KRV_CUDA(cudaMemsetAsync(sum_lo_.get(), 0, G * 8, rt_->stream));
        KRV_CUDA(cudaMemsetAsync(cnt_.get(), 0, G * 8, rt_->stream));
        KRV_CUDA(cudaMemsetAsync(nulls_.get(), 0, G * 8, rt_->stream));
        KRV_CUDA(cudaMemsetAsync(stats_.get(), 0, 32, rt_->stream));
        counters_.fact_rows = 0;
        if (plain_agg_) {
            agg_destroy(plain_agg_);
            plain_agg_ = nullptr;
        }
    }

    void check_fact(const DevBatch &f) const {
        const int nc = (int)f.cols.size();
        const int c[4] = {spec_.fact_fk_a, spec_.fact_fk_b, spec_.fact_price, spec_.fact_discount};
        const Type t[4] = {Type::I64, Type::I64, Type::I64, Type::F64};
        for (int i = 0; i < 4; i++) {
            if (c[i] < 0 || c[i] >= nc) fail(KRV_INVALID_ARGUMENT, "fact column out of range");
            if (f.cols[c[i]].type.id != t[i])
                fail(KRV_UNSUPPORTED, "star fact columns are (int64 fk_a, int64 fk_b, int64 price, float64 discount)");
        }
    }

    StarTable view(const Dim &d) const {
        if (!d.join) return StarTable{};  // the fast build keeps direct indexes only
        auto t = d.join->table_dev();
        return StarTable{t.slots, t.mask, t.next, t.seed, static_cast<const long long *>(d.join->arena().cols[0].data),
                         static_cast<const int32_t *>(d.join->arena().cols[2].data)};
    }

    template <int BMODE, bool VEC, bool KB32>
    void launch_scan(const StarArgs &A, int grid, size_t smem) {
        const bool nulls = A.v_fk_a || A.v_fk_b || A.v_price || A.v_disc;
        auto kern = nulls ? star_scan_kernel<BMODE, VEC, KB32, true> : star_scan_kernel<BMODE, VEC, KB32, false>;
        KRV_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<grid, kScanThreads, smem, rt_->stream>>>(A);
        rt_->launches++;
        check_launch("star_scan_kernel");
    }

    template <bool DIRECT, bool KB32>
    void launch_join(const StarArgs &A, int regions, int slices, int G) {
        const bool nulls = A.v_fk_a || A.v_fk_b || A.v_price || A.v_disc;
        auto kern = nulls ? star_join_kernel<DIRECT, KB32, true> : star_join_kernel<DIRECT, KB32, false>;
        const size_t smem = star_join_smem(G);
        KRV_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<regions * slices, kJoinThreads, smem, rt_->stream>>>(A, regions, slices, G);
        rt_->launches++;
        check_launch("star_join_kernel");
    }

    void probe_fused(const DevBatch &f) {
        StarArgs A{};
        A.fk_a = static_cast<const long long *>(f.cols[spec_.fact_fk_a].data);
        A.fk_b = static_cast<const long long *>(f.cols[spec_.fact_fk_b].data);
        A.price = static_cast<const long long *>(f.cols[spec_.fact_price].data);
        A.disc = static_cast<const double *>(f.cols[spec_.fact_discount].data);
        A.n = f.rows;
        if (A.n <= 0) return;
        if (A.n >= (int64_t)0xFFFFFFFFll) fail(KRV_UNSUPPORTED, "fact batches of 2^32 rows or more");
        auto fa = filt_[0], fb = filt_[1];
        A.use_filters = spec_.use_filters && fa && fb;
        if (A.use_filters) {
            A.fa = key_filter_dev(*fa);
            A.fb = key_filter_dev(*fb);
        }
        A.group_by = spec_.group_by;
        A.ta = view(dims_[0]);
        A.tb = view(dims_[1]);
        A.da = direct_[0];
        A.db = direct_[1];
        A.ngroups = ngroups_host_;
        A.sum_hi = sum_hi_.as<double>();
        A.sum_lo = sum_lo_.as<double>();
        A.cnt = cnt_.as<unsigned long long>();
        A.nulls = nulls_.as<unsigned long long>();
        A.stats = stats_.as<unsigned long long>();
        const DevCol &ca = f.cols[spec_.fact_fk_a], &cb = f.cols[spec_.fact_fk_b];
        const DevCol &cp = f.cols[spec_.fact_price], &cd = f.cols[spec_.fact_discount];
        A.v_fk_a = ca.valid;
        A.o_fk_a = ca.valid_off;
        A.v_fk_b = cb.valid;
        A.o_fk_b = cb.valid_off;
        A.v_price = cp.valid;
        A.o_price = cp.valid_off;
        A.v_disc = cd.valid;
        A.o_disc = cd.valid_off;
        // B's filter answer bitmap (built with the dimensions) is staged in
        // shared memory when it fits.
        A.bits_b = A.use_filters && bits_[1].get() ? bits_[1].as<uint32_t>() : nullptr;
        const size_t limit = (size_t)rt_->max_smem_optin - 1024;
        const bool staged = A.bits_b && star_scan_smem((int)bits_words_[1]) <= limit;
        A.bits_b_smem_words = staged ? (int)bits_words_[1] : 0;
        const void *host_fk_b = f.cols[spec_.fact_fk_b].host;
        if (host_fk_b && A.n >= 2 * kStreamRows) probe_streamed(A, static_cast<const long long *>(host_fk_b));
        else scan_join(A);
    }

    // A fact batch in page-locked host memory: fk_b, read whole, crosses the
    // host link as bulk copies into HBM (the link's copy rate, well above what
    // kernel loads of host memory reach), kStreamRows rows at a time with
    // kStreamStages chunks in flight on a copy stream; each chunk's scan and
    // join run as the next chunks arrive and read fk_a, price and discount in
    // place, so only the sectors of surviving rows cross the link.
    void probe_streamed(const StarArgs &A0, const long long *host_fk_b) {
        if (!cs_) {
            KRV_CUDA(cudaStreamCreateWithFlags(&cs_, cudaStreamNonBlocking));
            KRV_CUDA(cudaEventCreateWithFlags(&start_, cudaEventDisableTiming));
            for (int s = 0; s < kStreamStages; s++) {
                KRV_CUDA(cudaEventCreateWithFlags(&ready_[s], cudaEventDisableTiming));
                KRV_CUDA(cudaEventCreateWithFlags(&free_[s], cudaEventDisableTiming));
                stage_[s] = DBuf(rt_, (size_t)kStreamRows * 8);
            }
        }
        // The copies start after the work queued before them (the staging
        // buffers' readers in an earlier probe).
        KRV_CUDA(cudaEventRecord(start_, rt_->stream));
        KRV_CUDA(cudaStreamWaitEvent(cs_, start_, 0));
        const int64_t chunks = ceil_div(A0.n, kStreamRows);
        for (int64_t c = 0; c < chunks; c++) {
            const int s = (int)(c % kStreamStages);
            const int64_t r0 = c * kStreamRows, n = std::min(kStreamRows, A0.n - r0);
            if (c >= kStreamStages) KRV_CUDA(cudaStreamWaitEvent(cs_, free_[s], 0));
            KRV_CUDA(cudaMemcpyAsync(stage_[s].get(), host_fk_b + r0, (size_t)n * 8, cudaMemcpyHostToDevice, cs_));
            KRV_CUDA(cudaEventRecord(ready_[s], cs_));
            KRV_CUDA(cudaStreamWaitEvent(rt_->stream, ready_[s], 0));
            StarArgs A = A0;
            A.fk_b = stage_[s].as<long long>();
            A.fk_a += r0;
            A.price += r0;
            A.disc += r0;
            A.o_fk_a += r0;
            A.o_fk_b += r0;
            A.o_price += r0;
            A.o_disc += r0;
            A.n = n;
            // The join reads the survivor list, not fk_b: the stage is free
            // once the scan is done.
            scan_join(A, &free_[s]);
        }
    }

    // The scan (stage 1) and the join (stage 2) over one range of fact rows;
    // `scanned`, if given, is recorded between them.
    void scan_join(StarArgs &A, cudaEvent_t *scanned = nullptr) {
        // The survivor list: one region per scan CTA, as large as the rows it scans.
        const int64_t tiles = ceil_div(A.n, kScanTile);
        const int grid = (int)std::min<int64_t>(rt_->sm_count, tiles);
        A.region = (uint64_t)ceil_div(tiles, grid) * kScanTile;
        const uint64_t entries = A.region * (uint64_t)grid;
        // B's key range below 2^32: a survivor keeps fk_b - lo in 32 bits.
        const bool kb32 = A.use_filters && A.fb.has_range &&
                          (unsigned long long)(A.fb.hi - A.fb.lo) < 0xFFFFFFFFull;
        if (surv_cap_ < entries || surv_kb64_ != !kb32) {
            surv_row_ = DBuf(rt_, entries * 4);
            surv_kb_ = DBuf(rt_, entries * (kb32 ? 4 : 8));
            surv_cap_ = entries;
            surv_kb64_ = !kb32;
        }
        if (region_count_.bytes() < (size_t)grid * 8) region_count_ = DBuf(rt_, (size_t)rt_->sm_count * 8);
        A.surv_row = surv_row_.as<uint32_t>();
        A.surv_kb32 = kb32 ? surv_kb_.as<uint32_t>() : nullptr;
        A.surv_kb64 = kb32 ? nullptr : surv_kb_.as<long long>();
        A.region_count = region_count_.as<unsigned long long>();
        // 16-byte vector loads of fk_b need a 16-byte aligned column.
        const bool vec = (reinterpret_cast<uintptr_t>(A.fk_b) & 15) == 0;
        const size_t smem = star_scan_smem(A.bits_b_smem_words);
        if (A.bits_b_smem_words > 0) {
            if (vec && kb32) launch_scan<1, true, true>(A, grid, smem);
            else if (vec) launch_scan<1, true, false>(A, grid, smem);
            else if (kb32) launch_scan<1, false, true>(A, grid, smem);
            else launch_scan<1, false, false>(A, grid, smem);
        } else {
            if (vec && kb32) launch_scan<0, true, true>(A, grid, smem);
            else if (vec) launch_scan<0, true, false>(A, grid, smem);
            else if (kb32) launch_scan<0, false, true>(A, grid, smem);
            else launch_scan<0, false, false>(A, grid, smem);
        }
        if (scanned) KRV_CUDA(cudaEventRecord(*scanned, rt_->stream));
        // Join over the survivors: several CTAs per region, so hundreds of
        // thousands of independent probes hide the memory latency.
        const int G = std::max(1, std::min(ngroups_host_, 256));
        const int slices = 4;
        const bool direct = A.da.width && A.db.width;
        if (direct && kb32) launch_join<true, true>(A, grid, slices, G);
        else if (direct) launch_join<true, false>(A, grid, slices, G);
        else if (kb32) launch_join<false, true>(A, grid, slices, G);
        else launch_join<false, false>(A, grid, slices, G);
    }

    // A direct index (key -> group id) of dimension d when its keys are
    // unique and span at most 2^26 values and the ids fit 1 or 2 bytes.
    void build_direct(int d) {
        direct_[d] = StarDirect{nullptr, 0, 0, 0};
        direct_buf_[d].reset();
        const HashJoin &j = *dims_[d].join;
        const int64_t rows = j.indexed_rows();
        if (rows <= 0 || j.counters().build_keys != rows || j.counters().build_rows != rows) return;
        const __int128 span = (__int128)j.key_hi() - (__int128)j.key_lo();
        if (span < 0 || span >= ((__int128)1 << 26)) return;
        const int width = ngroups_host_ < 127 ? 1 : ngroups_host_ < 32767 ? 2 : 0;
        if (!width) return;
        const size_t bytes = ((size_t)span + 1) * width;
        direct_buf_[d] = DBuf(rt_, bytes);
        KRV_CUDA(cudaMemsetAsync(direct_buf_[d].get(), 0xFF, bytes, rt_->stream));
        const long long *keys = static_cast<const long long *>(j.arena().cols[0].data);
        const int32_t *gid = static_cast<const int32_t *>(j.arena().cols[2].data);
        if (width == 1)
            direct_index_kernel<int8_t><<<grid_for(rt_, rows, 256, 8), 256, 0, rt_->stream>>>(
                keys, gid, rows, j.key_lo(), direct_buf_[d].as<int8_t>());
        else
            direct_index_kernel<int16_t><<<grid_for(rt_, rows, 256, 8), 256, 0, rt_->stream>>>(
                keys, gid, rows, j.key_lo(), direct_buf_[d].as<int16_t>());
        rt_->launches++;
        check_launch("direct_index_kernel");
        direct_[d] = StarDirect{direct_buf_[d].get(), j.key_lo(), (unsigned long long)span, width};
    }

    // The answer bitmap of dimension d's filter over its key range, when the
    // range has at most 2^28 values (32 MiB).
    void build_bits(int d, const KeyFilterImpl &f) {
        bits_[d].reset();
        bits_words_[d] = 0;
        if (f.info.form == KRV_FILTER_EMPTY || !f.info.has_range) return;
        const __int128 range = (__int128)f.info.hi - (__int128)f.info.lo + 1;
        if (range <= 0 || range > ((__int128)1 << 28)) return;
        const uint64_t values = (uint64_t)range;
        const uint64_t words = (values + 127) / 128 * 4;  // whole 16-byte groups
        // Only a bitmap that fits in shared memory pays for its evaluation: one
        // evaluated in L2 costs about what the per-row probes it replaces do.
        if (star_scan_smem((int)std::min<uint64_t>(words, 1u << 30)) > (size_t)rt_->max_smem_optin - 1024)
            return;
        bits_[d] = DBuf(rt_, words * 4);
        filter_bitmap_kernel<<<grid_for(rt_, (int64_t)(words * 32), 256, 8), 256, 0, rt_->stream>>>(
            key_filter_dev(f), f.info.lo, words, values, bits_[d].as<uint32_t>());
        rt_->launches++;
        check_launch("filter_bitmap_kernel");
        bits_words_[d] = (int64_t)words;
    }

    void probe_plain(const DevBatch &f) {
        auto fa = filt_[0], fb = filt_[1];
        const int64_t n = f.rows;
        const DevCol &ca = f.cols[spec_.fact_fk_a], &cb = f.cols[spec_.fact_fk_b];
        const DevCol &cp = f.cols[spec_.fact_price], &cd = f.cols[spec_.fact_discount];
        // 1-2. the row stage: both runtime filters, then compaction (also
        // when columns have NULLs: rows with a NULL key go, and the price
        // column of the kept rows carries whether their value is valid)
        DevBatch kept;
        const bool filters = spec_.use_filters && fa && fb;
        const bool nullable = ca.valid || cb.valid || cp.valid || cd.valid;
        if (filters || nullable) {
            DevCol pb, pa;
            if (filters) {
                pb = evaluate_key_filter(*fb, cb);
                pa = evaluate_key_filter(*fa, ca);
            }
            DevCol o0 = make_col(rt_, ca.type, n, false, "fk_a"), o1 = make_col(rt_, cb.type, n, false, "fk_b");
            DevCol o2 = make_col(rt_, cp.type, n, false, "price"), o3 = make_col(rt_, cd.type, n, false, "discount");
            const bool value_nulls = cp.valid || cd.valid;
            if (value_nulls) {
                o2.hold_valid = std::make_shared<DBuf>(rt_, (size_t)ceil_div(std::max<int64_t>(n, 1), 32) * 4);
                KRV_CUDA(cudaMemsetAsync(o2.hold_valid->get(), 0, o2.hold_valid->bytes(), rt_->stream));
                o2.valid = o2.hold_valid->as<uint8_t>();
                o2.valid_off = 0;
                o2.nullable = true;
            }
            DBuf cnt(rt_, 8);
            KRV_CUDA(cudaMemsetAsync(cnt.get(), 0, 8, rt_->stream));
            if (n > 0) {
                const FactValid V{{ca.valid, cb.valid, cp.valid, cd.valid},
                                  {ca.valid_off, cb.valid_off, cp.valid_off, cd.valid_off}};
                compact4_kernel<<<grid_for(rt_, n, 256, 8), 256, 0, rt_->stream>>>(
                    filters ? (const uint32_t *)pa.data : nullptr, filters ? (const uint32_t *)pb.data : nullptr, n, V,
                    (const long long *)ca.data, (const long long *)cb.data, (const long long *)cp.data,
                    (const double *)cd.data, (long long *)o0.data, (long long *)o1.data, (long long *)o2.data,
                    (double *)o3.data, value_nulls ? o2.hold_valid->as<uint32_t>() : nullptr,
                    cnt.as<unsigned long long>());
                rt_->launches++;
                check_launch("compact4_kernel");
            }
            kept.rows = (int64_t)read_scalar<unsigned long long>(rt_, cnt.get());
            kept.cols = {o0, o1, o2, o3};
            for (auto &c : kept.cols) c.length = kept.rows;
            if (filters) counters_.passed_filters += kept.rows;
        } else {
            kept.rows = n;
            kept.cols = {ca, cb, cp, cd};
        }
        // 3. fact' JOIN dim_a -> (fk_b, price, discount, a.gid)
        krv_join_spec js;
        krv_join_spec_init(&js);
        js.join_type = KRV_JOIN_INNER;
        js.n_keys = 1;
        js.probe_keys[0] = 0;
        js.n_probe_out = 3;
        js.probe_out[0] = 1;
        js.probe_out[1] = 2;
        js.probe_out[2] = 3;
        js.n_build_out = 1;
        js.build_out[0] = 2;
        DevBatch j1 = probe_with(*dims_[0].join, kept, js);
        // 4. JOIN dim_b -> (price, discount, a.gid, b.gid)
        js.probe_keys[0] = 0;
        js.probe_out[0] = 1;
        js.probe_out[1] = 2;
        js.probe_out[2] = 3;
        DevBatch j2 = probe_with(*dims_[1].join, j1, js);
        counters_.joined_rows += j2.rows;
        // 5. projection: (gid, price * (1 - discount))
        DevCol val = make_col(rt_, DType{Type::F64, 0, 0}, j2.rows, false, "value");
        if (j2.rows > 0) {
            project_kernel<<<grid_for(rt_, j2.rows, 256, 8), 256, 0, rt_->stream>>>(
                (const long long *)j2.cols[0].data, (const double *)j2.cols[1].data, j2.rows, (double *)val.data);
            rt_->launches++;
            check_launch("project_kernel");
        }
        if (j2.cols[0].valid) {  // a NULL price or discount: a NULL value, skipped by SUM
            val.valid = j2.cols[0].valid;
            val.valid_off = j2.cols[0].valid_off;
            val.hold_valid = j2.cols[0].hold_valid;
            val.nullable = true;
        }
        DevBatch proj;
        proj.rows = j2.rows;
        proj.cols = {j2.cols[spec_.group_by == 0 ? 2 : 3], val};
        // 6. GROUP BY gid: SUM(value), COUNT(*)
        if (!plain_agg_) {
            krv_agg_spec as;
            krv_agg_spec_init(&as);
            as.n_group_by = 1;
            as.group_by[0] = 0;
            as.n_aggregates = 2;
            as.aggregates[0] = krv_agg_expr{KRV_AGG_SUM, 1, KRV_AGG_INPUT_RAW, -1, 0, 0, 0, 0};
            as.aggregates[1] = krv_agg_expr{KRV_AGG_COUNT_STAR, 0, KRV_AGG_INPUT_RAW, -1, 0, 0, 0, 0};
            as.expected_groups = std::max(ngroups_host_, 1);
            as.mode = KRV_AGG_MODE_GLOBAL;
            plain_agg_ = make_aggregate(rt_, as);
        }
        if (proj.rows > 0) agg_push(plain_agg_, proj);
    }

    // A probe of `in` against the built join `j` with another projection.
    DevBatch probe_with(HashJoin &j, const DevBatch &in, const krv_join_spec &proj) {
        const krv_join_spec saved = j.spec();
        j.set_probe_shape(proj);
        DevBatch out = j.probe(in);
        j.set_probe_shape(saved);
        return out;
    }

    void probe(const DevBatch &f) {
        if (!built_) fail(KRV_INVALID_ARGUMENT, "star probe before build");
        DeviceGuard g(rt_);
        check_fact(f);
        counters_.fact_rows += f.rows;
        if (spec_.mode == KRV_STAR_FUSED) probe_fused(f);
        else probe_plain(f);
    }

    DevBatch result() {
        DeviceGuard g(rt_);
        DevBatch out;
        const int G = std::max(ngroups_host_, 0);
        std::vector<int32_t> gattr(G);
        if (spec_.mode == KRV_STAR_FUSED) {
            // Compacted on the device; one host read of the row count and the
            // statistics.
            const int64_t cap = std::max(G, 1);
            DevCol a = make_col(rt_, DType{Type::I32, 0, 0}, cap, false, "attr");
            DevCol sc = make_col(rt_, DType{Type::F64, 0, 0}, cap, false, "sum");
            auto valid = std::make_shared<DBuf>(rt_, (size_t)ceil_div(cap, 32) * 4);
            DBuf info(rt_, 5 * 8);
            star_result_kernel<<<1, kResultThreads, 0, rt_->stream>>>(
                G, gattr_.as<int32_t>(), sum_hi_.as<double>(), sum_lo_.as<double>(), cnt_.as<unsigned long long>(),
                nulls_.as<unsigned long long>(), stats_.as<unsigned long long>(), const_cast<int32_t *>(
                    static_cast<const int32_t *>(a.data)), const_cast<double *>(static_cast<const double *>(sc.data)),
                valid->as<uint32_t>(), info.as<unsigned long long>());
            rt_->launches++;
            check_launch("star_result_kernel");
            unsigned long long r[5];
            read_device(rt_, info.get(), sizeof(r), r);
            counters_.passed_filters = (int64_t)r[2];
            counters_.joined_rows = (int64_t)r[3];
            counters_.fk_a_sectors = (int64_t)r[4];
            a.length = sc.length = (int64_t)r[0];
            if (r[1]) {
                sc.hold_valid = valid;
                sc.valid = valid->as<uint8_t>();
                sc.valid_off = 0;
                sc.nullable = true;
            }
            out.rows = (int64_t)r[0];
            out.cols = {a, sc};
            return out;
        }
        if (G > 0) {
            KRV_CUDA(cudaMemcpyAsync(gattr.data(), gattr_.get(), (size_t)G * 4, cudaMemcpyDeviceToHost, rt_->stream));
        }
        KRV_CUDA(cudaStreamSynchronize(rt_->stream));
        std::vector<int32_t> oa;
        std::vector<double> os;
        std::vector<uint8_t> ov;
        if (plain_agg_) {
            DevBatch r = agg_result(plain_agg_);
            const int64_t m = r.rows;
            std::vector<int32_t> gid(m);
            std::vector<double> sum(m);
            if (m > 0) {
                KRV_CUDA(cudaMemcpyAsync(gid.data(), r.cols[0].data, (size_t)m * 4, cudaMemcpyDeviceToHost, rt_->stream));
                KRV_CUDA(cudaMemcpyAsync(sum.data(), r.cols[1].data, (size_t)m * 8, cudaMemcpyDeviceToHost, rt_->stream));
                KRV_CUDA(cudaStreamSynchronize(rt_->stream));
            }
            const int64_t sv_bytes = ceil_div(std::max<int64_t>(r.cols[1].valid_off + m, 1), 8);
            std::vector<uint8_t> sv((size_t)sv_bytes, 0xFF);
            if (m > 0 && r.cols[1].valid)
                KRV_CUDA(cudaMemcpyAsync(sv.data(), r.cols[1].valid, (size_t)sv_bytes, cudaMemcpyDeviceToHost,
                                         rt_->stream));
            KRV_CUDA(cudaStreamSynchronize(rt_->stream));
            for (int64_t i = 0; i < m; i++) {
                oa.push_back(gattr[gid[i]]);
                os.push_back(sum[i]);
                const int64_t b = r.cols[1].valid_off + i;
                ov.push_back(r.cols[1].valid ? (uint8_t)((sv[b >> 3] >> (b & 7)) & 1) : (uint8_t)1);
            }
        }
        return host_result(oa, os, ov);
    }

    // The result batch (attr, sum); `valid[i]` = 0 makes sum i NULL.
    DevBatch host_result(const std::vector<int32_t> &attr, const std::vector<double> &sum,
                         const std::vector<uint8_t> &valid) {
        DevBatch out;
        const int64_t m = (int64_t)attr.size();
        bool any_null = false;
        for (uint8_t v : valid) any_null |= !v;
        DevCol a = make_col(rt_, DType{Type::I32, 0, 0}, m, false, "attr");
        DevCol s = make_col(rt_, DType{Type::F64, 0, 0}, m, any_null, "sum");
        std::vector<uint8_t> bits((size_t)ceil_div(std::max<int64_t>(m, 1), 8), 0);
        for (int64_t i = 0; i < m; i++)
            if (valid[i]) bits[i >> 3] |= (uint8_t)(1u << (i & 7));
        if (m > 0) {
            KRV_CUDA(cudaMemcpyAsync(const_cast<void *>(a.data), attr.data(), (size_t)m * 4, cudaMemcpyHostToDevice, rt_->stream));
            KRV_CUDA(cudaMemcpyAsync(const_cast<void *>(s.data), sum.data(), (size_t)m * 8, cudaMemcpyHostToDevice, rt_->stream));
            if (any_null)
                KRV_CUDA(cudaMemcpyAsync(const_cast<uint8_t *>(s.valid), bits.data(), bits.size(), cudaMemcpyHostToDevice,
                                         rt_->stream));
            KRV_CUDA(cudaStreamSynchronize(rt_->stream));
        }
        out.rows = m;
        out.cols = {a, s};
        return out;
    }

    krv_star_counters counters() const { return counters_; }
    bool fused() const { return spec_.mode == KRV_STAR_FUSED; }

  private:
    Runtime *rt_;
    krv_star_spec spec_;
    Dim dims_[2];
    std::shared_ptr<KeyFilterImpl> filt_[2];  // the dimensions' key filters
    DBuf gkeys_, gtab_, gattr_, ngroups_;
    uint32_t gmask_ = 0;
    int ngroups_host_ = 0;
    int dkey_[2] = {0, 0}, dpred_[2] = {1, 1}, dattr_[2] = {2, 2};  // each dimension's columns
    DBuf sum_hi_, sum_lo_, cnt_, nulls_, stats_;
    DBuf bits_[2];               // filter answer bitmaps of dimensions a and b
    DBuf direct_buf_[2];         // direct key -> group id indexes
    DBuf surv_row_, surv_kb_, region_count_;  // fact rows that passed B's filter
    uint64_t surv_cap_ = 0;
    bool surv_kb64_ = false;
    StarDirect direct_[2] = {};
    DBuf direct_full_[2];  // the fast build's direct indexes (kMaxDirectSpan entries each)
    int64_t bits_words_[2] = {0, 0};
    HashAggregate *plain_agg_ = nullptr;
    bool built_ = false;
    krv_star_counters counters_{};
    // Staging of fk_b from host memory (probe_streamed).
    static constexpr int64_t kStreamRows = 8ll << 20;  // 64 MiB of fk_b per chunk
    static constexpr int kStreamStages = 3;
    cudaStream_t cs_ = nullptr;
    cudaEvent_t start_ = nullptr, ready_[kStreamStages] = {}, free_[kStreamStages] = {};
    DBuf stage_[kStreamStages];

  public:
    ~StarPipeline() {
        if (plain_agg_) agg_destroy(plain_agg_);
        if (cs_) {
            cudaStreamSynchronize(cs_);
            cudaStreamSynchronize(rt_->stream);
            for (int s = 0; s < kStreamStages; s++) {
                cudaEventDestroy(ready_[s]);
                cudaEventDestroy(free_[s]);
            }
            cudaEventDestroy(start_);
            cudaStreamDestroy(cs_);
        }
    }
};

StarPipeline *make_star(Runtime *rt, const krv_star_spec &spec) { return new StarPipeline(rt, spec); }

// ---- the star plan from an operator chain ---------------------------------------
namespace {
// Where a column of a join's output comes from: the fact batch, or a build
// column of join a (side 1) or b (side 2).
struct ColFrom {
    int side, col;
};
// The columns of one join's output: its probe projection, then its build
// projection (join/mod.rs output order; a negative count takes them all).
ColFrom out_col(const krv_join_spec &s, int j, int n_probe_in, int n_build, int build_side,
                const std::function<ColFrom(int)> &probe_from) {
    const int np = s.n_probe_out < 0 ? n_probe_in : s.n_probe_out;
    const int nb = s.n_build_out < 0 ? n_build : s.n_build_out;
    if (j < 0 || j >= np + nb) fail(KRV_INVALID_ARGUMENT, "star chain: column out of range");
    if (j < np) return probe_from(s.n_probe_out < 0 ? j : s.probe_out[j]);
    const int b = s.n_build_out < 0 ? j - np : s.build_out[j - np];
    return ColFrom{build_side, b};
}
// A finished join's build rows as a star dimension: its columns, validity
// dropped where the column holds no NULL.
DevBatch dim_view(const HashJoin &J) {
    DevBatch d = J.arena();
    for (DevCol &c : d.cols)
        if (!c.nullable) c.valid = nullptr;
    return d;
}
}  // namespace

StarPipeline *make_star_from_joins(Runtime *rt, const HashJoin &ja, const HashJoin &jb, const krv_star_chain &c) {
    const HashJoin *J[2] = {&ja, &jb};
    for (const HashJoin *j : J) {
        const krv_join_spec &s = j->spec();
        if (s.join_type != KRV_JOIN_INNER || s.n_keys != 1 || s.null_safe[0] || j->has_residual())
            fail(KRV_UNSUPPORTED, "star chain: joins are inner, on one `=` key, without residual filter");
        if (!j->built()) fail(KRV_INVALID_ARGUMENT, "star chain: a join's build side is not finished");
        if (j->arena().cols.empty()) fail(KRV_UNSUPPORTED, "star chain: a join without build columns");
    }
    const krv_join_spec &sa = ja.spec(), &sb = jb.spec();
    const int nba = (int)ja.arena().cols.size(), nbb = (int)jb.arena().cols.size();
    const int npa = sa.n_probe_out < 0 ? c.n_fact_columns : sa.n_probe_out;
    const int nout_a = npa + (sa.n_build_out < 0 ? nba : sa.n_build_out);
    auto from_fact = [](int j) { return ColFrom{0, j}; };
    auto from_a = [&](int j) { return out_col(sa, j, c.n_fact_columns, nba, 1, from_fact); };
    auto from_b = [&](int j) { return out_col(sb, j, nout_a, nbb, 2, from_a); };
    const ColFrom fk_b = from_a(sb.probe_keys[0]);
    const ColFrom grp = from_b(c.group_col), price = from_b(c.price_col), disc = from_b(c.discount_col);
    if (fk_b.side != 0 || price.side != 0 || disc.side != 0)
        fail(KRV_UNSUPPORTED, "star chain: join_b's key, price and discount are fact columns");
    if (grp.side == 0) fail(KRV_UNSUPPORTED, "star chain: the grouped column is a dimension's");
    krv_star_spec spec;
    krv_star_spec_init(&spec);
    spec.fact_fk_a = sa.probe_keys[0];
    spec.fact_fk_b = fk_b.col;
    spec.fact_price = price.col;
    spec.fact_discount = disc.col;
    spec.group_by = grp.side - 1;
    spec.use_filters = sa.runtime_filter && sb.runtime_filter ? 1 : 0;
    spec.mode = c.mode;
    std::unique_ptr<StarPipeline> sp(new StarPipeline(rt, spec));
    for (int d = 0; d < 2; d++)
        sp->set_dim_cols(d, J[d]->spec().build_keys[0], -1, d == spec.group_by ? grp.col : -1);
    sp->build(dim_view(ja), dim_view(jb));
    return sp.release();
}
void star_build(StarPipeline *s, const DevBatch &a, const DevBatch &b) { s->build(a, b); }
void star_probe(StarPipeline *s, const DevBatch &fact) { s->probe(fact); }
DevBatch star_result(StarPipeline *s) { return s->result(); }
void star_reset(StarPipeline *s) { s->reset(); }
krv_star_counters star_counters(const StarPipeline *s) { return s->counters(); }
bool star_fused(const StarPipeline *s) { return s->fused(); }
void star_destroy(StarPipeline *s) { delete s; }

}  // namespace krv
