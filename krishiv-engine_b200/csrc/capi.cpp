// capi.cpp -- the extern "C" entry points of krv_gpu.h. No C++ exception
// crosses this boundary: every call runs under `guard`, which turns an error
// into a krv_status and the thread's last-error text.
#include <cuda_runtime.h>

#include <algorithm>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "krv_gpu.h"
#include "krv_internal.h"
#include "ops.h"

using krv::DevBatch;
using krv::Error;

struct krv_runtime {
    krv::Runtime rt;
};
struct krv_join {
    krv_runtime *owner;
    std::unique_ptr<krv::HashJoin> j;
    krv::GraceJoin *g = nullptr;  // a partitioned join instead of `j`
    std::vector<DevBatch> pending;
    ~krv_join() {
        if (g) krv::grace_destroy(g);
    }
    const krv_join_spec &spec() const { return g ? krv::grace_spec(g) : j->spec(); }
};
struct krv_agg {
    krv_runtime *owner;
    krv::HashAggregate *a = nullptr;
    std::vector<DevBatch> pending;
    bool produced = false;
};
struct krv_key_filter {
    std::shared_ptr<krv::KeyFilterImpl> f;
};
struct krv_star {
    krv_runtime *owner;
    krv::StarPipeline *s = nullptr;
};
struct krv_server {
    krv_runtime *owner;
    krv::Server *s = nullptr;
};

namespace {

template <class F>
krv_status guard(F &&f) {
    try {
        krv::set_last_error(KRV_OK, "", 0);
        // An error a runtime call left earlier on this thread (one this
        // library already reported, or the caller's own) is not this call's.
        cudaGetLastError();
        return f();
    } catch (const Error &e) {
        krv::set_last_error(e.code, e.msg, e.need_bytes);
        return e.code;
    } catch (const std::bad_alloc &) {
        krv::set_last_error(KRV_NEED_MEMORY, "host allocation failed", 0);
        return KRV_NEED_MEMORY;
    } catch (const std::exception &e) {
        krv::set_last_error(KRV_INTERNAL, e.what(), 0);
        return KRV_INTERNAL;
    } catch (...) {
        krv::set_last_error(KRV_INTERNAL, "unknown error", 0);
        return KRV_INTERNAL;
    }
}

void need(const void *p, const char *what) {
    if (!p) krv::fail(KRV_INVALID_ARGUMENT, std::string("null ") + what);
}

// Splits `b` into slices of at most `max_rows` (a multiple of 64, so every
// slice starts on a byte of its bitmaps); the first is returned.
DevBatch take_first(DevBatch b, int64_t max_rows, std::vector<DevBatch> &pending) {
    if (max_rows <= 0 || b.rows <= max_rows) return b;
    const int64_t step = std::max<int64_t>(64, max_rows / 64 * 64);
    std::vector<DevBatch> parts;
    for (int64_t from = 0; from < b.rows; from += step) {
        DevBatch s;
        s.rows = std::min(step, b.rows - from);
        for (const auto &c : b.cols) s.cols.push_back(krv::slice_col(c, from, s.rows));
        parts.push_back(std::move(s));
    }
    for (size_t i = parts.size(); i-- > 1;) pending.push_back(std::move(parts[i]));
    return std::move(parts[0]);
}

DevBatch pop(std::vector<DevBatch> &pending) {
    DevBatch b = std::move(pending.back());
    pending.pop_back();
    return b;
}

// The first piece of several output batches; the rest wait in `pending`.
DevBatch take_all(std::vector<DevBatch> bs, int64_t max_rows, std::vector<DevBatch> &pending) {
    std::vector<DevBatch> pieces;
    for (DevBatch &b : bs) {
        std::vector<DevBatch> rest;
        DevBatch first = take_first(std::move(b), max_rows, rest);
        pieces.push_back(std::move(first));
        for (size_t i = rest.size(); i-- > 0;) pieces.push_back(std::move(rest[i]));
    }
    for (size_t i = pieces.size(); i-- > 1;) pending.push_back(std::move(pieces[i]));
    return std::move(pieces[0]);
}

}  // namespace

// The functions below were declared extern "C" in krv_gpu.h, so their
// definitions have C linkage; the helper templates between them do not.
const char *krv_version(void) { return "krv-gpu 0.1.0 (sm_100a)"; }

krv_status krv_runtime_create(int32_t device, int64_t hbm_budget_bytes, void *cuda_stream, krv_runtime **out) {
    return guard([&] {
        need(out, "out");
        *out = nullptr;
        int count = 0;
        KRV_CUDA(cudaGetDeviceCount(&count));
        if (device < 0 || device >= count) krv::fail(KRV_INVALID_ARGUMENT, "no CUDA device " + std::to_string(device));
        int prev = 0;
        cudaGetDevice(&prev);
        KRV_CUDA(cudaSetDevice(device));
        auto h = std::make_unique<krv_runtime>();
        krv::Runtime &rt = h->rt;
        rt.device = device;
        rt.budget = hbm_budget_bytes > 0 ? hbm_budget_bytes : 0;
        if (cuda_stream) {
            rt.stream = static_cast<cudaStream_t>(cuda_stream);
        } else {
            KRV_CUDA(cudaStreamCreateWithFlags(&rt.stream, cudaStreamNonBlocking));
            rt.own_stream = true;
        }
        rt.pool = std::make_shared<krv::Pool>();
        rt.pool->budget = rt.budget;
        rt.pool->stream = rt.stream;
        rt.pool->device = device;
        KRV_CUDA(cudaDeviceGetAttribute(&rt.sm_count, cudaDevAttrMultiProcessorCount, device));
        KRV_CUDA(cudaDeviceGetAttribute(&rt.max_smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
        // Keep freed stream-ordered memory in the pool between calls.
        cudaMemPool_t pool;
        KRV_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
        uint64_t threshold = UINT64_MAX;
        KRV_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold));
        KRV_CUDA(cudaMalloc(&rt.status_dev, 64));
        KRV_CUDA(cudaMemset(rt.status_dev, 0, 64));
        // page-locked, mapped: the status words and small results read back by a kernel
        KRV_CUDA(cudaHostAlloc(&rt.status_host, 4096, cudaHostAllocMapped));
        KRV_CUDA(cudaHostGetDevicePointer(&rt.status_host_dev, rt.status_host, 0));
        cudaSetDevice(prev);
        *out = h.release();
        return KRV_OK;
    });
}

void krv_runtime_destroy(krv_runtime *h) {
    if (!h) return;
    krv::Runtime &rt = h->rt;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(rt.device);
    cudaStreamSynchronize(rt.stream);
    rt.pool->alive.store(false);
    cudaFree(rt.status_dev);
    cudaFreeHost(rt.status_host);
    if (rt.own_stream) cudaStreamDestroy(rt.stream);
    cudaSetDevice(prev);
    delete h;
}

krv_status krv_runtime_synchronize(krv_runtime *h) {
    return guard([&] {
        need(h, "runtime");
        KRV_CUDA(cudaStreamSynchronize(h->rt.stream));
        return KRV_OK;
    });
}
int64_t krv_runtime_used_bytes(const krv_runtime *h) { return h ? h->rt.pool->used.load() : 0; }
int64_t krv_runtime_budget_bytes(const krv_runtime *h) { return h ? h->rt.budget : 0; }
void *krv_runtime_stream(const krv_runtime *h) { return h ? (void *)h->rt.stream : nullptr; }
int64_t krv_runtime_launches(const krv_runtime *h) { return h ? h->rt.launches.load() : 0; }

// ---- join -------------------------------------------------------------------------
void krv_join_spec_init(krv_join_spec *s) {
    if (!s) return;
    *s = krv_join_spec{};
    s->n_keys = 1;
    s->n_probe_out = -1;
    s->n_build_out = -1;
}

krv_status krv_join_create(krv_runtime *rt, const krv_join_spec *spec, krv_join **out) {
    return guard([&] {
        need(rt, "runtime");
        need(spec, "spec");
        need(out, "out");
        *out = nullptr;
        auto h = std::make_unique<krv_join>();
        h->owner = rt;
        h->j.reset(new krv::HashJoin(&rt->rt, *spec));
        *out = h.release();
        return KRV_OK;
    });
}

void krv_grace_options_init(krv_grace_options *o) {
    if (!o) return;
    *o = krv_grace_options{};
    o->probe_filter_bits = 10;
}
krv_status krv_join_create_partitioned(krv_runtime *rt, const krv_join_spec *spec, const krv_grace_options *opt,
                                       krv_join **out) {
    return guard([&] {
        need(rt, "runtime");
        need(spec, "spec");
        need(out, "out");
        *out = nullptr;
        krv_grace_options o;
        if (opt) o = *opt;
        else krv_grace_options_init(&o);
        krv::DeviceGuard g(&rt->rt);
        auto h = std::make_unique<krv_join>();
        h->owner = rt;
        h->g = krv::make_grace(&rt->rt, *spec, o);
        *out = h.release();
        return KRV_OK;
    });
}
int64_t krv_join_spilled_partitions(const krv_join *j) {
    return j && j->g ? krv::grace_spilled_partitions(j->g) : 0;
}
int64_t krv_join_filtered_probe_rows(const krv_join *j) {
    return j && j->g ? krv::grace_filtered_probe_rows(j->g) : 0;
}

krv_status krv_join_build_push(krv_join *j, const ArrowArray *batch, const ArrowSchema *schema) {
    return guard([&] {
        need(j, "join");
        krv::DeviceGuard g(&j->owner->rt);
        krv::HostBorrow hb(&j->owner->rt);
        DevBatch b = krv::import_host(&j->owner->rt, batch, schema, krv::HostRead::Copy, krv::Var::Allow);
        if (j->g) krv::grace_build_push(j->g, b);
        else j->j->build_push(b);
        return KRV_OK;
    });
}
krv_status krv_join_build_push_device(krv_join *j, const ArrowDeviceArray *batch, const ArrowSchema *schema) {
    return guard([&] {
        need(j, "join");
        krv::DeviceGuard g(&j->owner->rt);
        DevBatch b = krv::import_device(&j->owner->rt, batch, schema, krv::Var::Allow);
        if (j->g) krv::grace_build_push(j->g, b);
        else j->j->build_push(b);
        return KRV_OK;
    });
}
krv_status krv_join_build_finish(krv_join *j) {
    return guard([&] {
        need(j, "join");
        krv::DeviceGuard g(&j->owner->rt);
        if (j->g) krv::grace_build_finish(j->g);
        else j->j->build_finish();
        return KRV_OK;
    });
}

template <bool Device, class In, class Out>
static krv_status join_probe_impl(krv_join *j, const In *in, const ArrowSchema *in_schema, Out *out,
                                  ArrowSchema *out_schema) {
    return guard([&] {
        need(j, "join");
        need(out, "out");
        krv::Runtime *rt = &j->owner->rt;
        krv::DeviceGuard g(rt);
        DevBatch b;
        if (in) {
            if (!j->pending.empty()) krv::fail(KRV_INVALID_ARGUMENT, "drain pending output (input NULL) first");
            DevBatch inb;
            std::unique_ptr<krv::HostBorrow> hb;
            if constexpr (Device) {
                inb = krv::import_device(rt, in, in_schema, krv::Var::Allow);
            } else {
                hb.reset(new krv::HostBorrow(rt));
                inb = krv::import_host(rt, in, in_schema, krv::HostRead::Copy, krv::Var::Allow);
            }
            if (j->g) {
                std::vector<DevBatch> outs = krv::grace_probe(j->g, inb);
                if (outs.empty()) outs.push_back(krv::grace_empty_output(j->g));
                b = take_all(std::move(outs), j->spec().max_output_rows, j->pending);
            } else {
                b = take_first(j->j->probe(inb), j->j->spec().max_output_rows, j->pending);
            }
        } else {
            if (j->pending.empty()) krv::fail(KRV_INVALID_ARGUMENT, "no pending output and no input");
            b = pop(j->pending);
        }
        if constexpr (Device) krv::export_device(rt, b, out, out_schema);
        else krv::export_host(rt, b, out, out_schema);
        return j->pending.empty() ? KRV_NEED_MORE_INPUT : KRV_HAVE_MORE_OUTPUT;
    });
}

krv_status krv_join_probe(krv_join *j, const ArrowArray *in, const ArrowSchema *in_schema, ArrowArray *out,
                          ArrowSchema *out_schema) {
    return join_probe_impl<false>(j, in, in_schema, out, out_schema);
}
krv_status krv_join_probe_device(krv_join *j, const ArrowDeviceArray *in, const ArrowSchema *in_schema,
                                 ArrowDeviceArray *out, ArrowSchema *out_schema) {
    return join_probe_impl<true>(j, in, in_schema, out, out_schema);
}

template <bool Device, class Out>
static krv_status join_finish_impl(krv_join *j, Out *out, ArrowSchema *out_schema) {
    return guard([&] {
        need(j, "join");
        need(out, "out");
        krv::Runtime *rt = &j->owner->rt;
        krv::DeviceGuard g(rt);
        DevBatch b;
        if (!j->pending.empty()) {
            b = pop(j->pending);
        } else if (j->g) {
            DevBatch next;
            if (krv::grace_finish_next(j->g, next)) b = take_first(std::move(next), j->spec().max_output_rows, j->pending);
            else b = krv::grace_empty_output(j->g);
        } else {
            b = take_first(j->j->finish(), j->j->spec().max_output_rows, j->pending);
        }
        if constexpr (Device) krv::export_device(rt, b, out, out_schema);
        else krv::export_host(rt, b, out, out_schema);
        const bool more = !j->pending.empty() || (j->g && !krv::grace_done(j->g));
        return more ? KRV_HAVE_MORE_OUTPUT : KRV_FINISHED;
    });
}
krv_status krv_join_finish(krv_join *j, ArrowArray *out, ArrowSchema *out_schema) {
    return join_finish_impl<false>(j, out, out_schema);
}
krv_status krv_join_finish_device(krv_join *j, ArrowDeviceArray *out, ArrowSchema *out_schema) {
    return join_finish_impl<true>(j, out, out_schema);
}

krv_status krv_join_key_filter(krv_join *j, krv_key_filter **out) {
    return guard([&] {
        need(j, "join");
        need(out, "out");
        *out = nullptr;
        if (j->g) krv::fail(KRV_UNSUPPORTED, "partitioned joins publish no key filter");
        auto f = j->j->key_filter();
        if (!f) krv::fail(KRV_UNSUPPORTED, "this join published no key filter (runtime_filter off or not one int64 key)");
        *out = new krv_key_filter{f};
        return KRV_OK;
    });
}
krv_status krv_join_set_filter(krv_join *j, const krv_join_filter *filter) {
    return guard([&] {
        need(j, "join");
        need(filter, "filter");
        if (j->g) krv::fail(KRV_UNSUPPORTED, "a residual filter on a partitioned join");
        krv::DeviceGuard g(&j->owner->rt);
        j->j->set_filter(*filter);
        return KRV_OK;
    });
}
krv_status krv_join_counters_get(const krv_join *j, krv_join_counters *out) {
    return guard([&] {
        need(j, "join");
        need(out, "out");
        *out = j->g ? krv::grace_counters(j->g) : j->j->counters();
        return KRV_OK;
    });
}
krv_status krv_hash_rows_device(krv_runtime *rt, const ArrowDeviceArray *batch, const ArrowSchema *schema,
                                const int32_t *key_columns, const int32_t *null_safe, int32_t n_keys, uint64_t seed,
                                int32_t depth, int32_t radix, uint64_t *out_h, uint64_t *out_g, int32_t *out_part) {
    return guard([&] {
        need(rt, "runtime");
        need(key_columns, "key_columns");
        krv::Runtime *r = &rt->rt;
        krv::DeviceGuard g(r);
        DevBatch b = krv::import_device(r, batch, schema);
        krv::hash_rows(r, b, key_columns, n_keys, null_safe, seed, depth, radix, out_h, out_g, out_part);
        return KRV_OK;
    });
}
void krv_join_destroy(krv_join *j) {
    if (!j) return;
    krv::DeviceGuard g(&j->owner->rt);
    delete j;
}

// ---- aggregate -----------------------------------------------------------------------
void krv_agg_spec_init(krv_agg_spec *s) {
    if (!s) return;
    *s = krv_agg_spec{};
    s->n_group_by = 1;
    s->ansi = 1;
    for (int e = 0; e < KRV_MAX_AGGREGATES; e++) s->aggregates[e].column2 = -1;
}

krv_status krv_agg_create(krv_runtime *rt, const krv_agg_spec *spec, krv_agg **out) {
    return guard([&] {
        need(rt, "runtime");
        need(spec, "spec");
        need(out, "out");
        *out = nullptr;
        auto h = std::make_unique<krv_agg>();
        h->owner = rt;
        h->a = krv::make_aggregate(&rt->rt, *spec);
        *out = h.release();
        return KRV_OK;
    });
}
krv_status krv_agg_push(krv_agg *a, const ArrowArray *batch, const ArrowSchema *schema) {
    return guard([&] {
        need(a, "aggregate");
        krv::DeviceGuard g(&a->owner->rt);
        krv::HostBorrow hb(&a->owner->rt);
        krv::agg_push(a->a, krv::import_host(&a->owner->rt, batch, schema, krv::HostRead::Copy, krv::Var::Allow));
        return KRV_OK;
    });
}
krv_status krv_agg_push_device(krv_agg *a, const ArrowDeviceArray *batch, const ArrowSchema *schema) {
    return guard([&] {
        need(a, "aggregate");
        krv::DeviceGuard g(&a->owner->rt);
        krv::agg_push(a->a, krv::import_device(&a->owner->rt, batch, schema, krv::Var::Allow));
        return KRV_OK;
    });
}
krv_status krv_agg_finish(krv_agg *a) {
    return guard([&] {
        need(a, "aggregate");
        krv::agg_finish(a->a);
        return KRV_OK;
    });
}

template <bool Device, class Out>
static krv_status agg_output_impl(krv_agg *a, Out *out, ArrowSchema *out_schema) {
    return guard([&] {
        need(a, "aggregate");
        need(out, "out");
        krv::Runtime *rt = &a->owner->rt;
        krv::DeviceGuard g(rt);
        DevBatch b;
        if (!a->produced) {
            a->produced = true;
            krv_agg_spec spec{};
            (void)spec;
            DevBatch all = krv::agg_result(a->a);
            b = take_first(std::move(all), 0, a->pending);
        } else if (!a->pending.empty()) {
            b = pop(a->pending);
        } else {
            krv::fail(KRV_INVALID_ARGUMENT, "the aggregate's output was already returned");
        }
        if constexpr (Device) krv::export_device(rt, b, out, out_schema);
        else krv::export_host(rt, b, out, out_schema);
        return a->pending.empty() ? KRV_FINISHED : KRV_HAVE_MORE_OUTPUT;
    });
}
krv_status krv_agg_next_output(krv_agg *a, ArrowArray *out, ArrowSchema *out_schema) {
    return agg_output_impl<false>(a, out, out_schema);
}
krv_status krv_agg_next_output_device(krv_agg *a, ArrowDeviceArray *out, ArrowSchema *out_schema) {
    return agg_output_impl<true>(a, out, out_schema);
}
int64_t krv_agg_groups(const krv_agg *a) { return a ? krv::agg_groups(a->a) : 0; }
void krv_agg_destroy(krv_agg *a) {
    if (!a) return;
    krv::DeviceGuard g(&a->owner->rt);
    krv::agg_destroy(a->a);
    delete a;
}

// ---- key filter ---------------------------------------------------------------------
template <bool Device, class In>
static krv_status filter_build_impl(krv_runtime *rt, const krv_key_filter_options *opt, const In *batch,
                                    const ArrowSchema *schema, int32_t column, krv_key_filter **out) {
    return guard([&] {
        need(rt, "runtime");
        need(out, "out");
        *out = nullptr;
        krv::DeviceGuard g(&rt->rt);
        krv_key_filter_options o;
        if (opt) o = *opt;
        else krv_key_filter_options_default(&o);
        krv::HostBorrow hb(&rt->rt);
        DevBatch b;
        if constexpr (Device) b = krv::import_device(&rt->rt, batch, schema);
        else b = krv::import_host(&rt->rt, batch, schema);
        if (column < 0 || column >= (int)b.cols.size()) krv::fail(KRV_INVALID_ARGUMENT, "column out of range");
        *out = new krv_key_filter{krv::build_key_filter(&rt->rt, o, b.cols[column])};
        return KRV_OK;
    });
}
krv_status krv_key_filter_build(krv_runtime *rt, const krv_key_filter_options *opt, const ArrowArray *batch,
                                const ArrowSchema *schema, int32_t column, krv_key_filter **out) {
    return filter_build_impl<false>(rt, opt, batch, schema, column, out);
}
krv_status krv_key_filter_build_device(krv_runtime *rt, const krv_key_filter_options *opt,
                                       const ArrowDeviceArray *batch, const ArrowSchema *schema, int32_t column,
                                       krv_key_filter **out) {
    return filter_build_impl<true>(rt, opt, batch, schema, column, out);
}

template <bool Device, class In, class Out>
static krv_status filter_eval_impl(krv_key_filter *f, const In *batch, const ArrowSchema *schema, int32_t column,
                                   Out *out, ArrowSchema *out_schema) {
    return guard([&] {
        need(f, "key filter");
        need(out, "out");
        krv::Runtime *rt = f->f->rt;
        krv::DeviceGuard g(rt);
        krv::HostBorrow hb(rt);
        DevBatch b;
        if constexpr (Device) b = krv::import_device(rt, batch, schema);
        else b = krv::import_host(rt, batch, schema);
        if (column < 0 || column >= (int)b.cols.size()) krv::fail(KRV_INVALID_ARGUMENT, "column out of range");
        DevBatch r;
        r.rows = b.rows;
        r.cols.push_back(krv::evaluate_key_filter(*f->f, b.cols[column]));
        if constexpr (Device) krv::export_device(rt, r, out, out_schema);
        else krv::export_host(rt, r, out, out_schema);
        return KRV_OK;
    });
}
krv_status krv_key_filter_evaluate(krv_key_filter *f, const ArrowArray *batch, const ArrowSchema *schema,
                                   int32_t column, ArrowArray *out, ArrowSchema *out_schema) {
    return filter_eval_impl<false>(f, batch, schema, column, out, out_schema);
}
krv_status krv_key_filter_evaluate_device(krv_key_filter *f, const ArrowDeviceArray *batch, const ArrowSchema *schema,
                                          int32_t column, ArrowDeviceArray *out, ArrowSchema *out_schema) {
    return filter_eval_impl<true>(f, batch, schema, column, out, out_schema);
}
krv_status krv_parquet_decode_chunk(krv_runtime *rt, const void *chunk, int64_t chunk_bytes,
                                    const krv_parquet_column *column, const krv_key_filter *filter,
                                    ArrowDeviceArray *out, ArrowSchema *out_schema, krv_parquet_info *info) {
    return guard([&] {
        need(rt, "runtime");
        need(column, "column");
        need(out, "out");
        need(out_schema, "out_schema");
        krv::DeviceGuard g(&rt->rt);
        krv::ParquetChunk r = krv::decode_parquet_chunk(&rt->rt, static_cast<const uint8_t *>(chunk), chunk_bytes,
                                                        *column, filter ? filter->f.get() : nullptr);
        krv::export_device(&rt->rt, r.batch, out, out_schema);
        if (info) *info = r.info;
        return KRV_OK;
    });
}
krv_status krv_key_filter_info_get(const krv_key_filter *f, krv_key_filter_info *out) {
    return guard([&] {
        need(f, "key filter");
        need(out, "out");
        *out = f->f->info;
        return KRV_OK;
    });
}
krv_status krv_key_filter_bloom_bytes(const krv_key_filter *f, void *host_out, int64_t nbytes) {
    return guard([&] {
        need(f, "key filter");
        need(host_out, "host_out");
        if (f->f->info.form != KRV_FILTER_BLOOM) krv::fail(KRV_INVALID_ARGUMENT, "the filter has no Bloom form");
        if (nbytes < f->f->info.bloom_bytes) krv::fail(KRV_INVALID_ARGUMENT, "buffer smaller than the filter");
        krv::Runtime *rt = f->f->rt;
        krv::DeviceGuard g(rt);
        KRV_CUDA(cudaMemcpyAsync(host_out, f->f->bloom.get(), (size_t)f->f->info.bloom_bytes, cudaMemcpyDeviceToHost,
                                 rt->stream));
        KRV_CUDA(cudaStreamSynchronize(rt->stream));
        return KRV_OK;
    });
}
void krv_key_filter_destroy(krv_key_filter *f) { delete f; }

// ---- star pipeline -------------------------------------------------------------------
void krv_star_spec_init(krv_star_spec *s) {
    if (!s) return;
    *s = krv_star_spec{};
    s->dim_key = 0;
    s->dim_pred = 1;
    s->dim_attr = 2;
    s->fact_fk_a = 0;
    s->fact_fk_b = 1;
    s->fact_price = 2;
    s->fact_discount = 3;
    s->use_filters = 1;
    s->mode = KRV_STAR_FUSED;
}
krv_status krv_star_create(krv_runtime *rt, const krv_star_spec *spec, krv_star **out) {
    return guard([&] {
        need(rt, "runtime");
        need(spec, "spec");
        need(out, "out");
        *out = nullptr;
        auto h = std::make_unique<krv_star>();
        h->owner = rt;
        h->s = krv::make_star(&rt->rt, *spec);
        *out = h.release();
        return KRV_OK;
    });
}
krv_status krv_star_from_joins(krv_runtime *rt, const krv_join *join_a, const krv_join *join_b,
                               const krv_star_chain *chain, krv_star **out) {
    return guard([&] {
        need(rt, "runtime");
        need(join_a, "join_a");
        need(join_b, "join_b");
        need(chain, "chain");
        need(out, "out");
        *out = nullptr;
        if (join_a->g || join_b->g) krv::fail(KRV_UNSUPPORTED, "star chain: partitioned joins are not fused");
        krv::DeviceGuard g(&rt->rt);
        auto h = std::make_unique<krv_star>();
        h->owner = rt;
        h->s = krv::make_star_from_joins(&rt->rt, *join_a->j, *join_b->j, *chain);
        *out = h.release();
        return KRV_OK;
    });
}
krv_status krv_star_build(krv_star *s, const ArrowArray *a, const ArrowSchema *sa, const ArrowArray *b,
                          const ArrowSchema *sb) {
    return guard([&] {
        need(s, "star");
        krv::Runtime *rt = &s->owner->rt;
        krv::DeviceGuard g(rt);
        krv::HostBorrow hb(rt);
        // The build reads each dimension column once: page-locked columns are
        // read in place.
        krv::star_build(s->s, krv::import_host(rt, a, sa, krv::HostRead::InPlace),
                        krv::import_host(rt, b, sb, krv::HostRead::InPlace));
        return KRV_OK;
    });
}
krv_status krv_star_build_device(krv_star *s, const ArrowDeviceArray *a, const ArrowSchema *sa,
                                 const ArrowDeviceArray *b, const ArrowSchema *sb) {
    return guard([&] {
        need(s, "star");
        krv::Runtime *rt = &s->owner->rt;
        krv::DeviceGuard g(rt);
        krv::star_build(s->s, krv::import_device(rt, a, sa), krv::import_device(rt, b, sb));
        return KRV_OK;
    });
}
krv_status krv_star_probe(krv_star *s, const ArrowArray *fact, const ArrowSchema *schema) {
    return guard([&] {
        need(s, "star");
        krv::Runtime *rt = &s->owner->rt;
        krv::DeviceGuard g(rt);
        krv::HostBorrow hb(rt);
        // The fused probe streams fk_b once and reads fk_a, price and discount
        // only for the rows that pass the filters: page-locked columns are
        // imported in place (fk_b then crosses in bulk copies, the others
        // only by the sectors the kernels read).
        const krv::HostRead mode = krv::star_fused(s->s) ? krv::HostRead::InPlace : krv::HostRead::Copy;
        krv::star_probe(s->s, krv::import_host(rt, fact, schema, mode));
        return KRV_OK;
    });
}
krv_status krv_star_probe_device(krv_star *s, const ArrowDeviceArray *fact, const ArrowSchema *schema) {
    return guard([&] {
        need(s, "star");
        krv::Runtime *rt = &s->owner->rt;
        krv::DeviceGuard g(rt);
        krv::star_probe(s->s, krv::import_device(rt, fact, schema));
        return KRV_OK;
    });
}
krv_status krv_star_result(krv_star *s, ArrowArray *out, ArrowSchema *out_schema) {
    return guard([&] {
        need(s, "star");
        need(out, "out");
        krv::Runtime *rt = &s->owner->rt;
        krv::DeviceGuard g(rt);
        krv::export_host(rt, krv::star_result(s->s), out, out_schema);
        return KRV_OK;
    });
}
krv_status krv_star_reset(krv_star *s) {
    return guard([&] {
        need(s, "star");
        krv::DeviceGuard g(&s->owner->rt);
        krv::star_reset(s->s);
        return KRV_OK;
    });
}
krv_status krv_star_counters_get(const krv_star *s, krv_star_counters *out) {
    return guard([&] {
        need(s, "star");
        need(out, "out");
        *out = krv::star_counters(s->s);
        return KRV_OK;
    });
}
void krv_star_destroy(krv_star *s) {
    if (!s) return;
    krv::DeviceGuard g(&s->owner->rt);
    krv::star_destroy(s->s);
    delete s;
}

// ---- request server -----------------------------------------------------------------
void krv_server_options_init(krv_server_options *o) {
    if (!o) return;
    *o = krv_server_options{};
    o->mode = KRV_SERVE_BATCHED;
    o->autotune = 1;
    o->ansi = 1;
    o->max_tick_requests = 512;
    o->tick_rows = 64ll << 20;
    o->hbm_budget_bytes = 0;
}
krv_status krv_server_create(krv_runtime *rt, const krv_server_options *o, krv_server **out) {
    return guard([&] {
        need(rt, "runtime");
        need(out, "out");
        *out = nullptr;
        krv_server_options opt;
        if (o) opt = *o;
        else krv_server_options_init(&opt);
        krv::DeviceGuard g(&rt->rt);
        auto h = std::make_unique<krv_server>();
        h->owner = rt;
        h->s = krv::make_server(&rt->rt, opt);
        *out = h.release();
        return KRV_OK;
    });
}
krv_status krv_server_add_table(krv_server *s, const ArrowDeviceArray *batch, const ArrowSchema *schema,
                                int32_t key_column, int32_t group_column, int64_t *table_id) {
    return guard([&] {
        need(s, "server");
        need(table_id, "table_id");
        krv::Runtime *rt = &s->owner->rt;
        krv::DeviceGuard g(rt);
        *table_id = krv::server_add_table(s->s, krv::import_device(rt, batch, schema), key_column, group_column);
        return KRV_OK;
    });
}
krv_status krv_server_drop_table(krv_server *s, int64_t table_id) {
    return guard([&] {
        need(s, "server");
        krv::DeviceGuard g(&s->owner->rt);
        krv::server_drop_table(s->s, table_id);
        return KRV_OK;
    });
}
krv_status krv_server_submit(krv_server *s, int64_t table_id, const ArrowDeviceArray *probe,
                             const ArrowSchema *schema, int32_t key_column, int32_t value_column,
                             int64_t *request_id) {
    return guard([&] {
        need(s, "server");
        need(request_id, "request_id");
        krv::Runtime *rt = &s->owner->rt;
        krv::DeviceGuard g(rt);
        *request_id = krv::server_submit(s->s, table_id, krv::import_device(rt, probe, schema), key_column,
                                         value_column);
        return KRV_OK;
    });
}
krv_status krv_server_step(krv_server *s, int32_t wait, int64_t *outstanding) {
    return guard([&] {
        need(s, "server");
        const int64_t n = krv::server_step(s->s, wait != 0);
        if (outstanding) *outstanding = n;
        return KRV_OK;
    });
}
krv_status krv_server_poll(krv_server *s, int64_t *request_id, krv_status *request_status, ArrowDeviceArray *out,
                           ArrowSchema *out_schema) {
    return guard([&] {
        need(s, "server");
        need(request_id, "request_id");
        need(request_status, "request_status");
        need(out, "out");
        need(out_schema, "out_schema");
        out->array.release = nullptr;
        out_schema->release = nullptr;
        krv::Runtime *rt = &s->owner->rt;
        krv::DeviceGuard g(rt);
        DevBatch b;
        int64_t id = 0;
        krv_status st = KRV_OK;
        if (!krv::server_poll(s->s, id, st, b)) return (krv_status)KRV_FINISHED;
        *request_id = id;
        *request_status = st;
        if (st == KRV_OK) krv::export_device(rt, b, out, out_schema);
        return (krv_status)KRV_OK;
    });
}
krv_status krv_server_stats_get(const krv_server *s, krv_server_stats *out) {
    return guard([&] {
        need(s, "server");
        need(out, "out");
        *out = krv::server_stats(s->s);
        return KRV_OK;
    });
}
void krv_server_destroy(krv_server *s) {
    if (!s) return;
    krv::DeviceGuard g(&s->owner->rt);
    krv::server_destroy(s->s);
    delete s;
}

// ---- generators ---------------------------------------------------------------------
krv_status krv_gen_fill(krv_runtime *rt, const krv_gen_spec *spec, int64_t n, void *out, void *out_valid) {
    return guard([&] {
        need(rt, "runtime");
        need(spec, "spec");
        need(out, "out");
        krv::gen_fill(&rt->rt, *spec, n, out, out_valid);
        return KRV_OK;
    });
}
