// ops.h -- the operator classes behind the C ABI (krv_gpu.h). Each mirrors
// the Krishiv engine operator it replaces; the file:line of that operator is
// on the class.
#pragma once

#include <memory>
#include <vector>

#include "krv_internal.h"

namespace krv {

// ---- device key views ----------------------------------------------------------
struct KeyColDev {
    const void *data;
    const uint8_t *valid;
    int64_t voff;
    int32_t width;      // 4, 8 or 16
    int32_t is_float;   // float64 key: normalized before hashing/comparing
};
struct KeysDev {
    KeyColDev c[KRV_MAX_KEYS];
    int32_t n;
    uint32_t null_safe;  // bit k: key k is compared with <=>
};
KeysDev keys_of(const DevBatch &b, const int32_t *cols, int n, const int32_t *null_safe);
// The join's key hash of every row (h, g = fin(h ^ seed), partition id at
// depth / radix); any output may be null. Device outputs of b.rows values.
void hash_rows(Runtime *rt, const DevBatch &b, const int32_t *cols, int n, const int32_t *null_safe, uint64_t seed,
               int depth, int radix, uint64_t *out_h, uint64_t *out_g, int32_t *out_part);

// ---- runtime key filter (crates/krishiv-io/src/runtime_filter/filter.rs:627) ----
struct KeyFilterImpl {
    Runtime *rt = nullptr;
    krv_key_filter_info info{};
    krv_key_filter_options opt{};
    DBuf bloom;          // Parquet SBBF words (info.bloom_bytes)
    DBuf exact_slots;    // exact set: open-addressing int64 set (EMPTY = INT64_MIN)
    uint64_t exact_mask = 0;
    int32_t exact_has_min = 0;  // INT64_MIN is in the exact set
};
// KeyFilterBuilder add + finish over the valid rows of an int64 column.
// What a join build already knows about its keys: the kept rows, the
// distinct keys and their range.
struct KeyStats {
    int64_t rows;
    int64_t distinct;
    long long lo, hi;
};
std::shared_ptr<KeyFilterImpl> build_key_filter(Runtime *rt, const krv_key_filter_options &opt,
                                                const DevCol &keys, const KeyStats *known = nullptr);
// KeyFilter::evaluate: a boolean column (bit-packed, no NULLs).
DevCol evaluate_key_filter(const KeyFilterImpl &f, const DevCol &keys);
// Device view for fused kernels.
struct KeyFilterDev {
    int32_t form;
    int32_t has_range;
    int64_t lo, hi;
    const uint32_t *bloom;
    uint64_t nblocks;
    const unsigned long long *exact;
    uint64_t exact_mask;
    int32_t exact_has_min;
    int32_t nulls_pass;
};
KeyFilterDev key_filter_dev(const KeyFilterImpl &f);

// ---- group key codes (keydict.cu) ------------------------------------------------
class KeyDict;
KeyDict *make_key_dict(Runtime *rt, const std::vector<DevCol> &meta);
void key_dict_destroy(KeyDict *d);
DBuf key_dict_encode(KeyDict *d, const DevBatch &b, const std::vector<int> &cols, bool insert = true);
std::vector<DevCol> key_dict_decode(KeyDict *d, const long long *codes, int64_t n);
int64_t key_dict_size(const KeyDict *d);
void key_dict_strings(const KeyDict *d, const long long **off, const int32_t **len, const uint8_t **heap);

// ---- residual join filter, device form (join/probe.rs:425-436) -------------------
// A conjunction of comparisons; a pair counts only where every one is TRUE
// (a NULL operand is not TRUE).
struct FilterOpDev {
    int32_t side;      // 0 the probe row's column, 1 the build row's, 2 a constant
    int32_t width;     // 4 or 8 (columns)
    int32_t is_float;  // a float64 column or constant
    int32_t pad;
    const void *data;
    const uint8_t *valid;
    int64_t voff;
    long long ci;
    double cf;
};
struct FilterTermDev {
    int32_t op;        // KRV_CMP_*
    int32_t as_float;  // compare as float64 (Spark's order)
    FilterOpDev l, r;
};
struct FilterDev {
    FilterTermDev t[KRV_MAX_FILTER_TERMS];
    int32_t n;
};

// ---- string and binary columns on the join path (varcol.cu) ----------------------
// A source of string values by row: Arrow int32 offsets into `bytes` (offs,
// value r = bytes[offs[r] .. offs[r + 1])), or a start and a length per row
// (starts / lens, the build arena's form).
struct VarSrc {
    const int32_t *offs;
    const long long *starts;
    const int32_t *lens;
    const uint8_t *bytes;
    const uint8_t *valid;
    int64_t voff;
};
// The build arena's form of one string column.
struct VarArena {
    std::shared_ptr<DBuf> starts, lens, heap;
    int64_t heap_size = 0, heap_cap = 0;
};
// Appends n rows of string column c at arena row base_row (starts and lens
// must hold base_row + n rows).
void var_arena_append(Runtime *rt, VarArena &a, const DevCol &c, int64_t base_row, int64_t n);
// The string column of m output rows whose values are src's rows idx[j]
// (idx null: row j; -1: NULL).
DevCol var_gather(Runtime *rt, const VarSrc &src, const long long *idx, int64_t m, DType type, bool nullable,
                  const std::string &name);

// ---- hash join (crates/krishiv-exec/src/join/mod.rs:1014 HashJoin) -------------
class HashJoin {
  public:
    HashJoin(Runtime *rt, const krv_join_spec &spec);
    void build_push(DevBatch b);
    // Takes a batch whose columns own their device memory as the whole build
    // side, without copying (one batch, before any push).
    void build_adopt(DevBatch b);
    void build_finish();
    // Joins one probe batch; returns the output batch (all rows of it).
    DevBatch probe(const DevBatch &in);
    // Rows emitted after the last probe batch (right/full joins).
    DevBatch finish();
    std::shared_ptr<KeyFilterImpl> key_filter() const { return filter_; }
    krv_join_counters counters() const { return counters_; }
    const krv_join_spec &spec() const { return spec_; }
    bool built() const { return built_; }
    bool has_residual() const { return residual_set_; }
    // Takes the probe key columns and the output projection of `s` (a plan
    // that probes one built table with batches of another shape).
    void set_probe_shape(const krv_join_spec &s) {
        for (int i = 0; i < KRV_MAX_KEYS; i++) spec_.probe_keys[i] = s.probe_keys[i];
        spec_.n_probe_out = s.n_probe_out;
        spec_.n_build_out = s.n_build_out;
        for (int i = 0; i < KRV_MAX_OUT_COLUMNS; i++) {
            spec_.probe_out[i] = s.probe_out[i];
            spec_.build_out[i] = s.build_out[i];
        }
        probe_types_.clear();
        probe_names_.clear();
        probe_nullable_.clear();
    }

    // Sets the residual filter (before the first build push).
    void set_filter(const krv_join_filter &f);

    // Pending output batches for the bounded-output protocol.
    std::vector<DevBatch> pending;
    ~HashJoin();

    // Device view of the built table (for fused pipelines).
    struct TableDev {
        unsigned long long *slots;
        uint64_t mask;
        const uint32_t *next;
        uint64_t seed;
    };
    TableDev table_dev() const;
    const DevBatch &arena() const { return arena_; }
    // The build rows pushed so far, before build_finish (data only).
    DevBatch staged() const;
    // What the build saw of a one-int64-key table: indexed rows and key range.
    int64_t indexed_rows() const { return indexed_rows_; }
    long long key_lo() const { return key_lo_; }
    long long key_hi() const { return key_hi_; }

  private:
    void append_arena(const DevBatch &b);
    // String or binary join keys: the key dictionary codes each key tuple as
    // one int64 (the build side inserts, the probe side looks up, -1 for a
    // key the build never saw); the table and kernels then join on that code.
    // String columns leave the batches the table sees, so none may be
    // projected into the output. spec_ then describes those batches; outer
    // is the caller's spec.
    struct Coded {
        KeyDict *dict = nullptr;
        krv_join_spec outer{};
        bool probe_mapped = false;
        ~Coded() {
            if (dict) key_dict_destroy(dict);
        }
    };
    std::unique_ptr<Coded> coded_;
    bool decided_ = false;
    // The residual filter (JoinSpec::filter), set before the build.
    krv_join_filter residual_{};
    bool residual_set_ = false;
    FilterDev filter_dev(const DevBatch &in) const;
    void decide(const DevBatch &b);
    DevBatch coded_batch(const DevBatch &b, bool build);
    // The column shape (types, names, nullability) of the probe output.
    void remember_shape(const DevBatch &out) {
        out_meta_.clear();
        for (const DevCol &c : out.cols) {
            DevCol m;
            m.type = c.type;
            m.name = c.name;
            m.nullable = c.nullable;
            out_meta_.push_back(m);
        }
    }
    std::vector<DevCol> out_meta_;
    int64_t indexed_rows_ = 0;
    long long key_lo_ = 0, key_hi_ = -1;
    Runtime *rt_;
    krv_join_spec spec_;
    std::vector<DevCol> arena_cols_;    // growable build arena
    std::vector<std::shared_ptr<DBuf>> arena_data_, arena_valid_;
    std::vector<VarArena> arena_var_;   // string columns: per-row starts, lengths and the byte heap
    // The string columns of an output batch: gathered from the probe batch
    // or the arena by the row index columns the kernels wrote.
    struct VarOut {
        int pos;        // output column
        int side;       // 0 probe, 1 build
        int col;        // source column
    };
    VarSrc var_src(int side, int col, const DevBatch *probe) const;
    DevCol empty_col(const DevCol &meta) const;
    int64_t arena_cap_ = 0;
    DevBatch arena_;                    // view of the arena
    bool have_schema_ = false;
    DBuf slots_, next_, marks_, counters_dev_;
    DBuf direct_;  // unique dense keys: key - key_lo_ -> build row
    unsigned long long direct_span_ = 0;
    uint64_t mask_ = 0;
    int64_t build_rows_ = 0;
    bool built_ = false;
    bool any_null_build_ = false;
    bool finished_ = false;
    std::vector<DType> probe_types_;
    std::vector<std::string> probe_names_;
    std::vector<bool> probe_nullable_;
    std::shared_ptr<KeyFilterImpl> filter_;
    krv_join_counters counters_{};
};

// ---- partitioned (grace) hash join (crates/krishiv-exec/src/join/grace.rs) ------
class GraceJoin;
GraceJoin *make_grace(Runtime *rt, const krv_join_spec &spec, const krv_grace_options &opt);
void grace_destroy(GraceJoin *g);
void grace_build_push(GraceJoin *g, const DevBatch &b);
void grace_build_finish(GraceJoin *g);
std::vector<DevBatch> grace_probe(GraceJoin *g, const DevBatch &b);
bool grace_finish_next(GraceJoin *g, DevBatch &out);
bool grace_done(const GraceJoin *g);
DevBatch grace_empty_output(GraceJoin *g);
const krv_join_spec &grace_spec(const GraceJoin *g);
krv_join_counters grace_counters(const GraceJoin *g);
int64_t grace_spilled_partitions(const GraceJoin *g);
int64_t grace_filtered_probe_rows(const GraceJoin *g);

// ---- Parquet column chunks decoded on the device (parquet.cu) ---------------------
struct ParquetChunk {
    DevBatch batch;  // the decoded column, then (with a filter) the filter's boolean column
    krv_parquet_info info;
};
ParquetChunk decode_parquet_chunk(Runtime *rt, const uint8_t *chunk, int64_t bytes, const krv_parquet_column &col,
                                  const KeyFilterImpl *filter);

// ---- grouped hash aggregate (crates/krishiv-exec/src/aggregate/sink.rs:181) ----
class HashAggregate;
HashAggregate *make_aggregate(Runtime *rt, const krv_agg_spec &spec);
void agg_push(HashAggregate *a, const DevBatch &b);
void agg_finish(HashAggregate *a);
DevBatch agg_result(HashAggregate *a);
int64_t agg_groups(const HashAggregate *a);
void agg_destroy(HashAggregate *a);

// ---- star pipeline -------------------------------------------------------------
class StarPipeline;
StarPipeline *make_star(Runtime *rt, const krv_star_spec &spec);
StarPipeline *make_star_from_joins(Runtime *rt, const HashJoin &ja, const HashJoin &jb, const krv_star_chain &c);
void star_build(StarPipeline *s, const DevBatch &a, const DevBatch &b);
void star_probe(StarPipeline *s, const DevBatch &fact);
DevBatch star_result(StarPipeline *s);
void star_reset(StarPipeline *s);
krv_star_counters star_counters(const StarPipeline *s);
bool star_fused(const StarPipeline *s);  // KRV_STAR_FUSED plan
void star_destroy(StarPipeline *s);

// ---- request server (serve.cu) -------------------------------------------------------
class Server;
Server *make_server(Runtime *rt, const krv_server_options &o);
int64_t server_add_table(Server *s, const DevBatch &b, int key_col, int group_col);
void server_drop_table(Server *s, int64_t id);
int64_t server_submit(Server *s, int64_t table, const DevBatch &b, int key_col, int value_col);
int64_t server_step(Server *s, bool wait);
bool server_poll(Server *s, int64_t &id, krv_status &status, DevBatch &out);
krv_server_stats server_stats(const Server *s);
void server_destroy(Server *s);

// ---- generators ------------------------------------------------------------------
void gen_fill(Runtime *rt, const krv_gen_spec &spec, int64_t n, void *out, void *out_valid);

// ---- small device utilities (util.cu) --------------------------------------------
// Copies n bits from (src, src_off) into (dst, dst_off); dst bits must be zero.
void append_bits(Runtime *rt, const uint8_t *src, int64_t src_off, int64_t n, uint8_t *dst,
                 int64_t dst_off);
// Sets n bits starting at dst_off to 1 (dst bits must be zero).
void set_bits(Runtime *rt, uint8_t *dst, int64_t dst_off, int64_t n);

}  // namespace krv
