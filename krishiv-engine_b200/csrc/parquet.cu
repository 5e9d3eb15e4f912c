// parquet.cu -- Parquet column chunks decoded on the device, with a runtime
// key filter evaluated on their encoded pages.
//
// Reference: the engine's Parquet reader decodes row groups on the host
// (crates/krishiv-io/src/parquet/decode.rs, through the parquet crate) and
// evaluates pushed predicates on a chunk's dictionary entries, once per entry
// (parquet/dict_probe.rs: `all_dictionary`, `passes`), so that a predicate on
// a dictionary-encoded column costs one test per entry and a lookup per row;
// a row group none of whose entries passes is skipped (`any_entry_in`).
// Here the chunk's bytes cross to HBM as the file stores them and:
//  - the host walks the page headers (Thrift compact protocol: parquet.thrift
//    PageHeader, DataPageHeader, DataPageHeaderV2, DictionaryPageHeader) and
//    lays every page out at a 16-byte aligned place of a staging buffer;
//  - stage_kernel (one CTA per page) copies each page's raw bytes there and
//    snappy_kernel decompresses Snappy (the raw format Parquet uses), one
//    warp per fragment of a page (runs of about 64 KiB of output that the
//    host finds by walking the tags), the stream and the last 32 KiB of
//    output in shared memory;
//  - dict_filter_kernel tests every dictionary entry against the key filter
//    (one byte per entry);
//  - page_decode_kernel (one CTA per data page, tiles of 1024 rows) decodes
//    the definition levels and the dictionary indices (RLE / bit-packed
//    hybrid: one thread lists the runs a tile needs, every thread decodes
//    its rows from them), ranks the tile's non-NULL rows with a block scan,
//    and writes the Arrow column, its validity and the filter's bit per row
//    (a dictionary entry's answer, or the member test of a PLAIN value);
//  - BYTE_ARRAY columns: ba_walk_kernel walks the PLAIN values of the
//    dictionary page and of PLAIN data pages into a (start, length) table,
//    page_decode_kernel writes each row's reference into it, and the string
//    gather of the join's payloads makes the UTF-8 / binary column.
// Flat columns only (max repetition level 0, max definition level 0 or 1);
// physical types INT32, INT64, DOUBLE and BYTE_ARRAY; PLAIN, PLAIN_DICTIONARY and
// RLE_DICTIONARY values; UNCOMPRESSED and SNAPPY chunks; data pages v1 and
// v2. Anything else returns KRV_UNSUPPORTED; bytes that do not decode return
// KRV_INVALID_ARGUMENT. Kernels read only inside their page's bytes.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "krv_filter.cuh"
#include "ops.h"

namespace krv {

namespace {

// parquet.thrift enums
constexpr int kPageData = 0, kPageIndex = 1, kPageDict = 2, kPageDataV2 = 3;
constexpr int kEncPlain = 0, kEncPlainDict = 2, kEncRle = 3, kEncRleDict = 8;
constexpr int kTile = 1024;        // rows per tile of page_decode_kernel
constexpr int kDecodeThreads = 256;
constexpr int kStageThreads = 256;
constexpr uint32_t ST_CORRUPT = 1u << 8;  // a page's bytes do not decode

// ---- host: the page headers ---------------------------------------------------------
struct Thrift {
    const uint8_t *p, *end;
    int depth = 0;
    [[noreturn]] static void corrupt(const char *what) {
        fail(KRV_INVALID_ARGUMENT, std::string("corrupt Parquet page header: ") + what);
    }
    uint8_t byte() {
        if (p >= end) corrupt("truncated");
        return *p++;
    }
    uint64_t varint() {
        uint64_t v = 0;
        for (int s = 0; s < 64; s += 7) {
            const uint8_t b = byte();
            v |= (uint64_t)(b & 0x7F) << s;
            if (!(b & 0x80)) return v;
        }
        corrupt("varint longer than 10 bytes");
    }
    int64_t zigzag() {
        const uint64_t v = varint();
        return (int64_t)(v >> 1) ^ -(int64_t)(v & 1);
    }
    void skip_bytes(uint64_t n) {
        if (n > (uint64_t)(end - p)) corrupt("truncated");
        p += n;
    }
    void skip(int type) {
        switch (type) {
        case 1: case 2: return;  // a struct field's bool lives in its type nibble
        case 3: skip_bytes(1); return;
        case 4: case 5: case 6: varint(); return;
        case 7: skip_bytes(8); return;
        case 8: skip_bytes(varint()); return;
        case 9: case 10: {  // list, set
            const uint8_t h = byte();
            uint64_t n = h >> 4;
            const int et = h & 15;
            if (n == 15) n = varint();
            for (uint64_t i = 0; i < n; i++) skip_elem(et);
            return;
        }
        case 11: {  // map
            const uint64_t n = varint();
            if (n == 0) return;
            const uint8_t kv = byte();
            for (uint64_t i = 0; i < n; i++) {
                skip_elem(kv >> 4);
                skip_elem(kv & 15);
            }
            return;
        }
        case 12: skip_struct(); return;
        default: corrupt("unknown field type");
        }
    }
    void skip_elem(int type) {
        if (type == 1 || type == 2) skip_bytes(1);  // bools inside containers are one byte
        else skip(type);
    }
    // Calls f(field id, type) for every field of a struct; f reads or skips it.
    template <class F> void fields(F &&f) {
        if (++depth > 32) corrupt("nested too deep");
        int16_t last = 0;
        for (;;) {
            const uint8_t h = byte();
            if (h == 0) break;
            const int type = h & 15, delta = h >> 4;
            const int16_t id = delta ? (int16_t)(last + delta) : (int16_t)zigzag();
            last = id;
            f(id, type);
        }
        depth--;
    }
    void skip_struct() {
        fields([&](int, int t) { skip(t); });
    }
    int32_t i32(int type) {
        if (type != 5) corrupt("expected an i32");
        const int64_t v = zigzag();
        if (v < INT32_MIN || v > INT32_MAX) corrupt("i32 out of range");
        return (int32_t)v;
    }
};

struct PageHdr {
    int type = -1;
    int32_t usize = -1, csize = -1;
    int32_t nvalues = -1, encoding = -1, def_encoding = kEncRle;
    int32_t def_len = 0, rep_len = 0;
    bool compressed = true;  // v2: is_compressed
};

PageHdr parse_page_header(Thrift &t) {
    PageHdr h;
    t.fields([&](int id, int type) {
        switch (id) {
        case 1: h.type = t.i32(type); break;
        case 2: h.usize = t.i32(type); break;
        case 3: h.csize = t.i32(type); break;
        case 5:  // DataPageHeader
            if (type != 12) Thrift::corrupt("data_page_header");
            t.fields([&](int f, int ft) {
                if (f == 1) h.nvalues = t.i32(ft);
                else if (f == 2) h.encoding = t.i32(ft);
                else if (f == 3) h.def_encoding = t.i32(ft);
                else t.skip(ft);
            });
            break;
        case 7:  // DictionaryPageHeader
            if (type != 12) Thrift::corrupt("dictionary_page_header");
            t.fields([&](int f, int ft) {
                if (f == 1) h.nvalues = t.i32(ft);
                else if (f == 2) h.encoding = t.i32(ft);
                else t.skip(ft);
            });
            break;
        case 8:  // DataPageHeaderV2
            if (type != 12) Thrift::corrupt("data_page_header_v2");
            t.fields([&](int f, int ft) {
                if (f == 1) h.nvalues = t.i32(ft);
                else if (f == 4) h.encoding = t.i32(ft);
                else if (f == 5) h.def_len = t.i32(ft);
                else if (f == 6) h.rep_len = t.i32(ft);
                else if (f == 7) h.compressed = ft == 1;  // bool: 1 true, 2 false
                else t.skip(ft);
            });
            break;
        default: t.skip(type);
        }
    });
    return h;
}

// ---- device descriptors ---------------------------------------------------------------
struct StageDev {
    int64_t src, dst;   // page payload in the chunk; its staged place
    int32_t csize, usize;
    int32_t raw;        // leading bytes copied as they are (v2 levels)
    int32_t snappy;     // the rest is Snappy-compressed
};
// A run of a Snappy stream's elements that decodes alone: its first element
// in the chunk, its first output byte in the staging buffer, their lengths.
struct FragDev {
    int64_t src, dst;
    int32_t slen, dlen;
};
struct PageDev {
    int64_t staged;     // offset of the staged (uncompressed) page
    int64_t row0;       // the page's first row in the chunk
    int32_t usize;
    int32_t nvalues;
    int32_t v2;         // levels without a length prefix (data page v2)
    int32_t dict;       // values are dictionary indices
    int32_t def_len;    // v2: bytes of the definition levels
    int32_t pad;
};
// OUT_REF (BYTE_ARRAY): each row's value is written as a reference, its
// dictionary entry or dict_n + (its page's first row) + (its rank among the
// page's non-NULL values), into the (start, length) table the walk filled;
// -1 for NULL. The string column is then gathered by those references.
enum OutKind : int32_t { OUT_SAME = 0, OUT_I32_TO_I64 = 1, OUT_TO_DEC128 = 2, OUT_REF = 3 };
struct DecodeArgs {
    const PageDev *pages;
    const uint8_t *staged;
    int32_t max_def;
    int32_t pwidth;     // bytes per PLAIN value: 4 or 8
    int32_t out_kind;
    int32_t is_int;     // the values are integers (the filter tests them)
    void *out;
    uint32_t *valid;    // null when the column is required
    const uint8_t *dict;
    int64_t dict_n;
    const uint8_t *dict_pass;  // the filter's answer per dictionary entry (null without a filter)
    int32_t has_filter;
    int32_t pad;
    KeyFilterDev f;
    uint32_t *pass;     // the filter's bit per row
    unsigned long long *counts;  // [0] rows passing the filter
    uint32_t *status;
    long long *ref;      // OUT_REF: each row's value reference
    const int32_t *walked;  // OUT_REF: the values the walk found in each PLAIN page
};
// A BYTE_ARRAY page whose values are walked: PLAIN values, each a 4-byte
// little-endian length and its bytes, one after another.
struct WalkDev {
    int64_t staged;     // the staged page
    int64_t base;       // its first value's slot in the (start, length) table
    int32_t usize;
    int32_t kind;       // 0 dictionary page, 1 data page v1, 2 data page v2
    int32_t def_len;    // v2: bytes of the definition levels
    int32_t limit;      // the values it may hold
    int32_t page;       // the data page's index (walked[page]); -1 for the dictionary
    int32_t pad;
};

// ---- stage: copy or Snappy-decompress each page ------------------------------------------
// Copies n bytes (any alignment) with `threads` threads, thread t taking
// bytes t, t + threads, ...: every thread issues kCopyDepth loads before its
// stores, so that many bytes are in flight per thread instead of one
// load-to-store round trip per byte. src and dst do not overlap.
constexpr int kCopyDepth = 16;
__device__ __forceinline__ void copy_bytes(uint8_t *dst, const uint8_t *src, int64_t n, int t, int threads) {
    for (int64_t i0 = 0; i0 < n; i0 += (int64_t)threads * kCopyDepth) {
        uint8_t v[kCopyDepth];
#pragma unroll
        for (int u = 0; u < kCopyDepth; u++) {
            const int64_t i = i0 + (int64_t)u * threads + t;
            v[u] = i < n ? src[i] : 0;
        }
#pragma unroll
        for (int u = 0; u < kCopyDepth; u++) {
            const int64_t i = i0 + (int64_t)u * threads + t;
            if (i < n) dst[i] = v[u];
        }
    }
}

// Snappy (raw format): a varint of the uncompressed length, then elements:
// literals (tag & 3 == 0) and back-references with 1-, 2- or 4-byte offsets.
// One warp decodes a page; its lanes all parse the same tags (uniform
// control flow) and share each element's bytes. The latency of a page is
// its chain of elements (a dictionary page of small integers is hundreds of
// thousands of short elements), so each element's work stays in shared
// memory: the compressed stream passes through an 8 KiB window, loaded in
// bulk as parsing reaches its end, and the last 32 KiB of output are kept
// in a ring, from which a back-reference reads its bytes (one from further
// back reads global memory). A back-reference that overlaps its own output
// is copied in steps of its offset.
constexpr int kSnappyWin = 8192;
constexpr int kSnappyRing = 32768;
constexpr int kSnappySmem = kSnappyWin + kSnappyRing;

struct SnappyWarp {
    const uint8_t *src;
    int64_t slen;
    uint8_t *dst;
    int64_t dlen;
    uint8_t *win, *ring;
    int64_t w0 = 0, wn = 0;  // the window holds src[w0, w0 + wn)
    unsigned lane;

    __device__ void refill(int64_t at) {
        __syncwarp();
        w0 = at;
        wn = min((int64_t)kSnappyWin, slen - at);
        copy_bytes(win, src + at, wn, (int)lane, 32);
        __syncwarp();
    }
    __device__ __forceinline__ uint8_t at(int64_t i) const { return win[i - w0]; }
    // Output bytes [op, op + n) from stream bytes [ip, ip + n).
    __device__ void literal(int64_t ip, int64_t op, int64_t n) {
        if (ip + n <= w0 + wn) {
            for (int64_t i = lane; i < n; i += 32) {
                const uint8_t b = win[ip - w0 + i];
                dst[op + i] = b;
                ring[(op + i) & (kSnappyRing - 1)] = b;
            }
            return;
        }
        for (int64_t i0 = 0; i0 < n; i0 += 32 * kCopyDepth) {  // beyond the window: global, many loads in flight
            uint8_t v[kCopyDepth];
#pragma unroll
            for (int u = 0; u < kCopyDepth; u++) {
                const int64_t i = i0 + u * 32 + lane;
                v[u] = i < n ? src[ip + i] : 0;
            }
#pragma unroll
            for (int u = 0; u < kCopyDepth; u++) {
                const int64_t i = i0 + u * 32 + lane;
                if (i < n) {
                    dst[op + i] = v[u];
                    ring[(op + i) & (kSnappyRing - 1)] = v[u];
                }
            }
        }
    }
    // Output bytes [op, op + n) from output bytes [op - off, op - off + n), off >= n.
    __device__ void backref(int64_t op, int64_t off, int64_t n) {
        const bool near = off <= kSnappyRing - 64;  // read and written ring slots never meet
        for (int64_t i = lane; i < n; i += 32) {
            const uint8_t b = near ? ring[(op - off + i) & (kSnappyRing - 1)] : dst[op - off + i];
            dst[op + i] = b;
            ring[(op + i) & (kSnappyRing - 1)] = b;
        }
    }

    // The elements of one fragment: stream bytes [0, slen) to output bytes
    // [0, dlen); a back-reference reaching before the fragment is corrupt.
    __device__ bool run() {
        if (slen == 0) return dlen == 0;
        refill(0);
        int64_t ip = 0, op = 0;
        while (ip < slen) {
            if (ip + 5 > w0 + wn && w0 + wn < slen) refill(ip);  // a tag and up to 4 more bytes
            const uint8_t tag = at(ip++);
            const int kind = tag & 3;
            int64_t len, off = 0;
            if (kind == 0) {
                len = tag >> 2;
                if (len >= 60) {
                    const int nb = (int)len - 59;
                    if (ip + nb > slen) return false;
                    len = 0;
                    for (int i = 0; i < nb; i++) len |= (int64_t)at(ip + i) << (8 * i);
                    ip += nb;
                }
                len += 1;
                if (ip + len > slen || op + len > dlen) return false;
                literal(ip, op, len);
                ip += len;
                op += len;
            } else {
                if (kind == 1) {
                    if (ip + 1 > slen) return false;
                    len = 4 + ((tag >> 2) & 7);
                    off = ((int64_t)(tag >> 5) << 8) | at(ip);
                    ip += 1;
                } else if (kind == 2) {
                    if (ip + 2 > slen) return false;
                    len = 1 + (tag >> 2);
                    off = (int64_t)at(ip) | ((int64_t)at(ip + 1) << 8);
                    ip += 2;
                } else {
                    if (ip + 4 > slen) return false;
                    len = 1 + (tag >> 2);
                    off = (int64_t)at(ip) | ((int64_t)at(ip + 1) << 8) | ((int64_t)at(ip + 2) << 16) |
                          ((int64_t)at(ip + 3) << 24);
                    ip += 4;
                }
                if (off <= 0 || off > op || op + len > dlen) return false;
                if (off >= len) {
                    backref(op, off, len);
                } else {
                    for (int64_t done = 0; done < len; done += off) {
                        backref(op + done, off, min(off, len - done));
                        __syncwarp();
                    }
                }
                op += len;
            }
            __syncwarp();
        }
        return op == dlen;
    }
};

// Copies each page's leading raw bytes (all of an uncompressed page, a v2
// page's levels) to its staged place, one CTA per page.
__global__ void __launch_bounds__(kStageThreads) stage_kernel(const StageDev *pages, const uint8_t *chunk,
                                                              uint8_t *staged) {
    const StageDev P = pages[blockIdx.x];
    const uint8_t *src = chunk + P.src;
    uint8_t *dst = staged + P.dst;
    const int64_t raw = P.snappy ? P.raw : P.usize;  // uncompressed: the whole page is copied
    if (((uintptr_t)src & 15) == 0) {  // dst is 16-byte aligned: whole 16-byte words where src is too
        const int64_t words = raw / 16;
        for (int64_t i = threadIdx.x; i < words; i += blockDim.x)
            reinterpret_cast<uint4 *>(dst)[i] = reinterpret_cast<const uint4 *>(src)[i];
        for (int64_t i = words * 16 + threadIdx.x; i < raw; i += blockDim.x) dst[i] = src[i];
    } else {
        copy_bytes(dst, src, raw, threadIdx.x, blockDim.x);
    }
}

// Decompresses the Snappy fragments: one warp (CTA) per fragment.
__global__ void __launch_bounds__(32) snappy_kernel(const FragDev *frags, const uint8_t *chunk, uint8_t *staged,
                                                    uint32_t *status) {
    extern __shared__ __align__(16) uint8_t snappy_smem[];
    const FragDev F = frags[blockIdx.x];
    SnappyWarp w;
    w.src = chunk + F.src;
    w.slen = F.slen;
    w.dst = staged + F.dst;
    w.dlen = F.dlen;
    w.win = snappy_smem;
    w.ring = snappy_smem + kSnappyWin;
    w.lane = threadIdx.x;
    if (!w.run() && threadIdx.x == 0) atomicOr(status, ST_CORRUPT);
}

// ---- the filter over the dictionary entries ------------------------------------------------
__device__ __forceinline__ int64_t load_int(const uint8_t *p, int width) {
    if (width == 4) {
        uint32_t v;
        memcpy(&v, p, 4);
        return (int64_t)(int32_t)v;
    }
    uint64_t v;
    memcpy(&v, p, 8);
    return (int64_t)v;
}

__global__ void dict_filter_kernel(KeyFilterDev f, const uint8_t *dict, int64_t n, int width, uint8_t *pass,
                                   unsigned long long *npass) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const bool p = filter_pass(f, load_int(dict + i * width, width));
        pass[i] = p;
        if (p) atomicAdd(npass, 1ull);
    }
}

// ---- the data pages -------------------------------------------------------------------------
// RLE / bit-packed hybrid (Parquet Encodings.md): runs, each a ULEB128 header;
// header & 1 == 0: an RLE run of header >> 1 copies of one value stored in
// ceil(bit_width / 8) bytes; else (header >> 1) groups of 8 bit-packed values.
// Offsets are bytes from the staged page's start (pages are at most 256 MiB).
struct Hybrid {
    int32_t p, end;     // the stream's next byte and its end
    int32_t bw;
    int32_t kind;       // 0 RLE, 1 bit-packed
    int64_t left;       // values left in the current run
    uint32_t value;     // RLE: the value
    int32_t base;       // bit-packed: the run's first byte
    int32_t bytes;      // bit-packed: the run's bytes
    int32_t bit;        // bit-packed: bit of the next value within the run
};
struct Run {
    int32_t first;      // the run's first value within the tile's list
    uint32_t value;     // RLE: the value
    int32_t base;       // bit-packed: the run's first byte; -1 for an RLE run
    int32_t bytes;
    int32_t bit;        // bit of the run's first listed value
};

__device__ bool next_run(Hybrid &h, const uint8_t *page) {
    for (int guard = 0; guard < 1 << 20; guard++) {
        uint64_t hdr = 0;
        for (int s = 0;; s += 7) {
            if (h.p >= h.end || s > 35) return false;
            const uint8_t b = page[h.p++];
            hdr |= (uint64_t)(b & 0x7F) << s;
            if (!(b & 0x80)) break;
        }
        if (!(hdr & 1)) {
            h.kind = 0;
            h.left = (int64_t)(hdr >> 1);
            const int nb = (h.bw + 7) / 8;
            if (h.end - h.p < nb) return false;
            uint32_t v = 0;
            for (int i = 0; i < nb; i++) v |= (uint32_t)page[h.p + i] << (8 * i);
            h.p += nb;
            if (h.bw < 32 && (v >> h.bw)) return false;
            h.value = v;
        } else {
            h.kind = 1;
            const int64_t groups = (int64_t)(hdr >> 1);
            const int64_t bytes = groups * h.bw;
            if (bytes > (int64_t)(h.end - h.p)) return false;
            h.left = groups * 8;
            h.base = h.p;
            h.bytes = (int32_t)bytes;
            h.bit = 0;
            h.p += (int32_t)bytes;
        }
        if (h.left > 0) return true;
    }
    return false;
}

// Lists the runs covering the next `need` values (thread 0 only).
__device__ bool emit_runs(Hybrid &h, const uint8_t *page, int need, Run *runs, int &nruns) {
    nruns = 0;
    int at = 0;
    while (at < need) {
        if (h.left == 0 && !next_run(h, page)) return false;
        const int take = (int)(h.left < (int64_t)(need - at) ? h.left : (int64_t)(need - at));
        Run r;
        r.first = at;
        r.value = h.value;
        r.base = h.kind ? h.base : -1;
        r.bytes = h.bytes;
        r.bit = h.bit;
        runs[nruns++] = r;
        if (h.kind == 1) h.bit += take * h.bw;
        h.left -= take;
        at += take;
    }
    return true;
}

// Value j (0-based within the tile's list) of the runs.
__device__ __forceinline__ uint32_t run_value(const Run *runs, int nruns, int j, int bw, const uint8_t *page) {
    int lo = 0, hi = nruns - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (runs[mid].first <= j) lo = mid;
        else hi = mid - 1;
    }
    const Run &r = runs[lo];
    if (r.base < 0) return r.value;
    const int64_t b = (int64_t)r.bit + (int64_t)(j - r.first) * bw;
    const int64_t byte0 = b >> 3;
    const uint8_t *q = page + r.base;
    uint64_t w = 0;
    for (int i = 0; i < 5 && byte0 + i < r.bytes; i++) w |= (uint64_t)q[byte0 + i] << (8 * i);
    return (uint32_t)((w >> (b & 7)) & (bw == 32 ? 0xFFFFFFFFull : ((1ull << bw) - 1)));
}

__device__ __forceinline__ void bitmap_or(uint32_t *words, int64_t row, unsigned bits32) {
    // bits32: 32 consecutive rows starting at `row`
    if (!bits32) return;
    const int64_t w = row >> 5;
    const int s = (int)(row & 31);
    atomicOr(words + w, bits32 << s);
    if (s) {
        const unsigned hi = bits32 >> (32 - s);
        if (hi) atomicOr(words + w + 1, hi);
    }
}

// The PLAIN BYTE_ARRAY values of a dictionary page or a data page, one warp
// (lane 0) per page: each value's start in the staging buffer and its length
// into the table, every length checked against the page.
__global__ void __launch_bounds__(32) ba_walk_kernel(const WalkDev *items, const uint8_t *staged, int max_def,
                                                     long long *starts, int32_t *lens, int32_t *walked,
                                                     uint32_t *status) {
    if (threadIdx.x != 0) return;
    const WalkDev W = items[blockIdx.x];
    const uint8_t *page = staged + W.staged;
    auto le32 = [&](int64_t at) {
        return (uint32_t)page[at] | ((uint32_t)page[at + 1] << 8) | ((uint32_t)page[at + 2] << 16) |
               ((uint32_t)page[at + 3] << 24);
    };
    int64_t pos = 0;
    const int64_t end = W.usize;
    if (W.kind == 1 && max_def > 0) {  // v1: the levels' 4-byte length, then the levels
        if (end < 4 || (int64_t)le32(0) > end - 4) {
            atomicOr(status, ST_CORRUPT);
            return;
        }
        pos = 4 + (int64_t)le32(0);
    } else if (W.kind == 2) {
        pos = W.def_len;
    }
    int32_t n = 0;
    while (pos < end && n < W.limit) {
        if (end - pos < 4) break;
        const int64_t len = le32(pos);
        if (len > end - pos - 4) break;
        starts[W.base + n] = (long long)(W.staged + pos + 4);
        lens[W.base + n] = (int32_t)len;
        pos += 4 + len;
        n++;
    }
    if (W.page >= 0) walked[W.page] = n;
    if (pos != end || (W.page < 0 && n != W.limit)) atomicOr(status, ST_CORRUPT);
}

__global__ void __launch_bounds__(kDecodeThreads) page_decode_kernel(DecodeArgs A) {
    constexpr int U = kTile / kDecodeThreads;
    __shared__ Hybrid s_def, s_idx;
    // one list: the definition levels' runs of a tile are read before the
    // scan's barrier, the indices' runs written after it
    __shared__ Run s_runs[kTile];
    __shared__ int s_nd, s_ni, s_ok;
    __shared__ int s_warp[kDecodeThreads / 32];
    __shared__ const uint8_t *s_values;
    __shared__ int64_t s_values_len;
    const PageDev P = A.pages[blockIdx.x];
    const uint8_t *page = A.staged + P.staged;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        s_ok = 1;
        const uint8_t *p = page, *end = page + P.usize;
        if (A.max_def > 0) {
            int64_t len;
            if (P.v2) {
                len = P.def_len;
            } else {
                if (end - p < 4) s_ok = 0;
                len = s_ok ? (int64_t)((uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) |
                                       ((uint32_t)p[3] << 24))
                           : 0;
                p += s_ok ? 4 : 0;
            }
            if (len < 0 || len > end - p) s_ok = 0;
            if (s_ok) {
                s_def = Hybrid{(int32_t)(p - page), (int32_t)(p - page + len), 1, 0, 0, 0, 0, 0, 0};
                p += len;
            }
        } else if (P.v2) {
            p += P.def_len;  // no levels are stored for a required column (def_len 0)
        }
        if (s_ok && P.dict) {
            if (p >= end) {
                // no index bytes: only an all-NULL page may have none (a run is never asked for)
                s_idx = Hybrid{P.usize, P.usize, 0, 0, 0, 0, 0, 0, 0};
            } else {
                const int bw = *p++;
                if (bw > 32) s_ok = 0;
                s_idx = Hybrid{(int32_t)(p - page), P.usize, bw, 0, 0, 0, 0, 0, 0};
            }
        }
        s_values = p;
        s_values_len = end - p;
    }
    __syncthreads();
    if (!s_ok) {
        if (tid == 0) atomicOr(A.status, ST_CORRUPT);
        return;
    }
    const bool aligned = ((uintptr_t)s_values & (uintptr_t)(A.pwidth - 1)) == 0;
    int64_t nn_base = 0;  // non-NULL values before this tile
    for (int t0 = 0; t0 < P.nvalues; t0 += kTile) {
        const int n = min(kTile, P.nvalues - t0);
        if (tid == 0 && A.max_def > 0 && !emit_runs(s_def, page, n, s_runs, s_nd)) s_ok = 0;
        __syncthreads();
        if (!s_ok) break;
        bool v[U];
        int cnt = 0;
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int i = tid * U + u;  // consecutive rows per thread: ranks by a scan of counts
            v[u] = i < n && (A.max_def == 0 || run_value(s_runs, s_nd, i, 1, page) == 1);
            cnt += v[u];
        }
        // block exclusive scan of cnt
        int incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) s_warp[warp] = incl;
        __syncthreads();
        int wbase = 0, total = 0;
        for (int w = 0; w < kDecodeThreads / 32; w++) {
            if (w < warp) wbase += s_warp[w];
            total += s_warp[w];
        }
        int rank = wbase + incl - cnt;
        if (tid == 0 && P.dict && total > 0 && !emit_runs(s_idx, page, total, s_runs, s_ni)) s_ok = 0;
        __syncthreads();
        if (!s_ok) break;
        unsigned vbits = 0, pbits = 0;
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int i = tid * U + u;
            if (i >= n) break;
            const int64_t row = P.row0 + t0 + i;
            if (A.out_kind == OUT_REF) {
                long long rf = -1;
                if (v[u]) {
                    const int64_t k = rank++;  // within the tile; nn_base + k within the page
                    if (P.dict) {
                        const uint32_t idx = run_value(s_runs, s_ni, (int)k, s_idx.bw, page);
                        if ((int64_t)idx >= A.dict_n) {
                            atomicOr(A.status, ST_CORRUPT);
                            continue;
                        }
                        rf = (long long)idx;
                    } else {
                        if (nn_base + k >= A.walked[blockIdx.x]) {
                            atomicOr(A.status, ST_CORRUPT);
                            continue;
                        }
                        rf = (long long)(A.dict_n + P.row0 + nn_base + k);
                    }
                }
                A.ref[row] = rf;
                continue;
            }
            int64_t ival = 0;
            uint64_t raw = 0;
            bool pass = A.f.nulls_pass != 0;
            if (v[u]) {
                const int64_t k = nn_base + rank++;
                const uint8_t *src = nullptr;
                bool dict_hit = false;
                uint32_t idx = 0;
                if (P.dict) {
                    idx = run_value(s_runs, s_ni, (int)(k - nn_base), s_idx.bw, page);
                    if ((int64_t)idx >= A.dict_n) {
                        atomicOr(A.status, ST_CORRUPT);
                        continue;
                    }
                    src = A.dict + (int64_t)idx * A.pwidth;
                    dict_hit = true;
                } else {
                    if ((k + 1) * A.pwidth > s_values_len) {
                        atomicOr(A.status, ST_CORRUPT);
                        continue;
                    }
                    src = s_values + k * A.pwidth;
                }
                if (A.pwidth == 4) {
                    uint32_t w;
                    if (dict_hit || aligned) w = *reinterpret_cast<const uint32_t *>(src);
                    else memcpy(&w, src, 4);
                    raw = w;
                    ival = (int64_t)(int32_t)w;
                } else {
                    uint64_t w;
                    if (dict_hit || aligned) w = *reinterpret_cast<const uint64_t *>(src);
                    else memcpy(&w, src, 8);
                    raw = w;
                    ival = (int64_t)w;
                }
                vbits |= 1u << u;
                if (A.has_filter) pass = dict_hit && A.dict_pass ? A.dict_pass[idx] != 0 : filter_pass(A.f, ival);
            }
            if (A.has_filter && pass) pbits |= 1u << u;
            if (A.out_kind == OUT_SAME) {
                if (A.pwidth == 4) static_cast<uint32_t *>(A.out)[row] = (uint32_t)raw;
                else static_cast<uint64_t *>(A.out)[row] = raw;
            } else if (A.out_kind == OUT_I32_TO_I64) {
                static_cast<int64_t *>(A.out)[row] = ival;
            } else {
                static_cast<int64_t *>(A.out)[2 * row] = ival;
                static_cast<int64_t *>(A.out)[2 * row + 1] = ival < 0 ? -1 : 0;
            }
        }
        // U consecutive rows per thread: 8 threads hold 32 consecutive rows
        static_assert(U == 4, "bitmap packing assumes 4 rows per thread");
        const int sub = lane & 7;
        unsigned vw = vbits << (4 * sub), pw = pbits << (4 * sub);
#pragma unroll
        for (int o = 1; o < 8; o <<= 1) {
            vw |= __shfl_xor_sync(0xFFFFFFFFu, vw, o);
            pw |= __shfl_xor_sync(0xFFFFFFFFu, pw, o);
        }
        if (sub == 0) {
            const int64_t row = P.row0 + t0 + tid * U;
            if (A.valid) bitmap_or(A.valid, row, vw);
            if (A.has_filter) {
                bitmap_or(A.pass, row, pw);
                if (pw) atomicAdd(A.counts, (unsigned long long)__popc(pw));
            }
        }
        nn_base += total;
        __syncthreads();
    }
    if (!s_ok && tid == 0) atomicOr(A.status, ST_CORRUPT);
}

}  // namespace

// ---- the operator ----------------------------------------------------------------------------
namespace {
// The fragments of one page's Snappy stream. A page's elements are a chain
// (each starts where the last ended), so one warp decoding a large page is
// slow; but a Snappy compressor codes its input in independent blocks of
// 64 KiB (Google's snappy::Compress), so the stream splits into runs of
// elements whose back-references stay inside the run. The host walks the
// tags (skipping literal bytes), starts a fragment at the first element
// boundary after each 64 KiB of output, and merges a fragment back into the
// one before whenever a back-reference reaches behind its start, so every
// fragment decodes alone whatever compressor wrote the stream. The host
// copies no data: the warps decompress every byte. A stream that does not
// parse stays one fragment, whose warp reports it.
constexpr int64_t kFragBytes = 65536;
void plan_fragments(const uint8_t *chunk, const StageDev &s, std::vector<FragDev> &out) {
    const uint8_t *p = chunk + s.src + s.raw;
    const int64_t slen = (int64_t)s.csize - s.raw, dlen = (int64_t)s.usize - s.raw;
    if (slen == 0) {
        if (dlen != 0) fail(KRV_INVALID_ARGUMENT, "corrupt Parquet page: an empty Snappy stream");
        return;
    }
    int64_t ip = 0;
    uint64_t n = 0;
    for (int sh = 0;; sh += 7) {
        if (ip >= slen || sh > 28) fail(KRV_INVALID_ARGUMENT, "corrupt Parquet page: the Snappy length");
        const uint8_t b = p[ip++];
        n |= (uint64_t)(b & 0x7F) << sh;
        if (!(b & 0x80)) break;
    }
    if ((int64_t)n != dlen) fail(KRV_INVALID_ARGUMENT, "corrupt Parquet page: the Snappy length");
    std::vector<std::pair<int64_t, int64_t>> starts{{ip, 0}};  // (stream, output) offsets of each fragment
    if (dlen > 2 * kFragBytes) {
        int64_t op = 0;
        while (ip < slen) {
            const uint8_t tag = p[ip++];
            int64_t len, off = 0;
            const int kind = tag & 3;
            if (kind == 0) {
                len = tag >> 2;
                if (len >= 60) {
                    const int nb = (int)len - 59;
                    if (ip + nb > slen) break;
                    len = 0;
                    for (int i = 0; i < nb; i++) len |= (int64_t)p[ip + i] << (8 * i);
                    ip += nb;
                }
                len += 1;
                if (ip + len > slen) break;
                ip += len;
            } else {
                const int nb = kind == 1 ? 1 : kind == 2 ? 2 : 4;
                if (ip + nb > slen) break;
                if (kind == 1) {
                    len = 4 + ((tag >> 2) & 7);
                    off = ((int64_t)(tag >> 5) << 8) | p[ip];
                } else {
                    len = 1 + (tag >> 2);
                    for (int i = 0; i < nb; i++) off |= (int64_t)p[ip + i] << (8 * i);
                }
                ip += nb;
                if (off <= 0 || off > op) break;
                while (starts.size() > 1 && op - off < starts.back().second) starts.pop_back();
            }
            op += len;
            if (op > dlen) break;
            if (op - starts.back().second >= kFragBytes && ip < slen) starts.push_back({ip, op});
        }
    }
    for (size_t k = 0; k < starts.size(); k++) {
        const int64_t ip0 = starts[k].first, op0 = starts[k].second;
        const int64_t ip1 = k + 1 < starts.size() ? starts[k + 1].first : slen;
        const int64_t op1 = k + 1 < starts.size() ? starts[k + 1].second : dlen;
        out.push_back(FragDev{s.src + s.raw + ip0, s.dst + s.raw + op0, (int32_t)(ip1 - ip0), (int32_t)(op1 - op0)});
    }
}
}  // namespace

ParquetChunk decode_parquet_chunk(Runtime *rt, const uint8_t *chunk, int64_t bytes, const krv_parquet_column &col,
                                  const KeyFilterImpl *filter) {
    if (!chunk && bytes > 0) fail(KRV_INVALID_ARGUMENT, "chunk is NULL");
    if (bytes < 0) fail(KRV_INVALID_ARGUMENT, "chunk_bytes < 0");
    if (col.num_values < 0) fail(KRV_INVALID_ARGUMENT, "num_values < 0");
    if (col.max_def_level < 0 || col.max_def_level > 1)
        fail(KRV_UNSUPPORTED, "the GPU Parquet decoder takes flat columns (max definition level 0 or 1)");
    if (col.codec != KRV_PQ_UNCOMPRESSED && col.codec != KRV_PQ_SNAPPY)
        fail(KRV_UNSUPPORTED, "Parquet codec " + std::to_string(col.codec) + " on the GPU decoder (UNCOMPRESSED, SNAPPY)");
    int pwidth = 0;  // 0: BYTE_ARRAY (a 4-byte length before each value)
    if (col.physical_type == KRV_PQ_INT32) pwidth = 4;
    else if (col.physical_type == KRV_PQ_INT64 || col.physical_type == KRV_PQ_DOUBLE) pwidth = 8;
    else if (col.physical_type != KRV_PQ_BYTE_ARRAY)
        fail(KRV_UNSUPPORTED, "Parquet physical type " + std::to_string(col.physical_type) + " on the GPU decoder");
    const bool var = col.physical_type == KRV_PQ_BYTE_ARRAY;
    if (!col.format) fail(KRV_INVALID_ARGUMENT, "format is NULL");
    const DType out_t = parse_format(col.format);
    int out_kind = -1;
    if (col.physical_type == KRV_PQ_INT32) {
        if (out_t.id == Type::I32 || out_t.id == Type::Date32) out_kind = OUT_SAME;
        else if (out_t.id == Type::I64 || out_t.id == Type::Dec64) out_kind = OUT_I32_TO_I64;
        else if (out_t.id == Type::Dec128) out_kind = OUT_TO_DEC128;
    } else if (col.physical_type == KRV_PQ_INT64) {
        if (out_t.id == Type::I64 || out_t.id == Type::Dec64) out_kind = OUT_SAME;
        else if (out_t.id == Type::Dec128) out_kind = OUT_TO_DEC128;
    } else if (col.physical_type == KRV_PQ_DOUBLE) {
        if (out_t.id == Type::F64) out_kind = OUT_SAME;
    } else if (out_t.id == Type::Utf8 || out_t.id == Type::Binary) {
        out_kind = OUT_REF;
    }
    if (out_kind < 0) fail(KRV_UNSUPPORTED, std::string("Parquet column decoded as ") + col.format);
    const bool is_int = col.physical_type == KRV_PQ_INT32 || col.physical_type == KRV_PQ_INT64;
    if (filter && !is_int) fail(KRV_UNSUPPORTED, "key filters test integer columns");

    // The page headers, on the host.
    std::vector<StageDev> stages;
    std::vector<PageDev> pages;
    int64_t staged_bytes = 0, rows = 0;
    int dict_stage = -1;
    int64_t dict_n = 0;
    bool all_dict = true;  // every data page is dictionary encoded (dict_probe.rs `all_dictionary`)
    Thrift t{chunk, chunk + bytes};
    while (t.p < t.end && rows < col.num_values) {
        const PageHdr h = parse_page_header(t);
        const int64_t at = t.p - chunk;
        if (h.csize < 0 || h.usize < 0 || h.csize > t.end - t.p)
            fail(KRV_INVALID_ARGUMENT, "corrupt Parquet page header: page sizes");
        if (h.usize > (1 << 28)) fail(KRV_UNSUPPORTED, "Parquet pages of more than 256 MiB on the GPU decoder");
        t.p += h.csize;
        if (h.type == kPageIndex) continue;
        if (h.type != kPageData && h.type != kPageDataV2 && h.type != kPageDict)
            fail(KRV_UNSUPPORTED, "Parquet page type " + std::to_string(h.type));
        if (h.nvalues < 0) fail(KRV_INVALID_ARGUMENT, "corrupt Parquet page header: num_values");
        StageDev s{};
        s.src = at;
        s.dst = staged_bytes;
        s.csize = h.csize;
        s.usize = h.usize;
        s.snappy = col.codec == KRV_PQ_SNAPPY && (h.type != kPageDataV2 || h.compressed);
        if (h.type == kPageDataV2) {
            if (h.rep_len != 0) fail(KRV_UNSUPPORTED, "repeated Parquet columns on the GPU decoder");
            if (h.def_len < 0 || h.def_len > h.csize || h.def_len > h.usize)
                fail(KRV_INVALID_ARGUMENT, "corrupt Parquet page header: level lengths");
            if (col.max_def_level == 0 && h.def_len != 0)
                fail(KRV_INVALID_ARGUMENT, "definition levels in a required column");
            s.raw = h.def_len;
        }
        if (!s.snappy && h.csize != h.usize) fail(KRV_INVALID_ARGUMENT, "corrupt Parquet page: sizes of an uncompressed page differ");
        if (h.type == kPageDict) {
            if (dict_stage >= 0 || !pages.empty()) fail(KRV_INVALID_ARGUMENT, "a dictionary page after the first page");
            if (h.encoding != kEncPlain && h.encoding != kEncPlainDict)
                fail(KRV_UNSUPPORTED, "Parquet dictionary encoding " + std::to_string(h.encoding));
            if ((int64_t)h.nvalues * (var ? 4 : pwidth) > h.usize) fail(KRV_INVALID_ARGUMENT, "corrupt Parquet dictionary page");
            dict_stage = (int)stages.size();
            dict_n = h.nvalues;
        } else {
            PageDev p{};
            p.staged = staged_bytes;
            p.row0 = rows;
            p.usize = h.usize;
            p.nvalues = h.nvalues;
            p.v2 = h.type == kPageDataV2;
            p.def_len = h.def_len;
            if (h.encoding == kEncPlainDict || h.encoding == kEncRleDict) {
                if (dict_stage < 0) fail(KRV_INVALID_ARGUMENT, "a dictionary-encoded Parquet page without a dictionary");
                p.dict = 1;
            } else if (h.encoding != kEncPlain) {
                fail(KRV_UNSUPPORTED, "Parquet encoding " + std::to_string(h.encoding) + " on the GPU decoder");
            } else {
                all_dict = false;
            }
            if (!p.v2 && col.max_def_level > 0 && h.def_encoding != kEncRle)
                fail(KRV_UNSUPPORTED, "Parquet definition level encoding " + std::to_string(h.def_encoding));
            pages.push_back(p);
            rows += h.nvalues;
        }
        stages.push_back(s);
        staged_bytes += ((int64_t)h.usize + 15) / 16 * 16;
    }
    if (rows != col.num_values)
        fail(KRV_INVALID_ARGUMENT, "the chunk's data pages hold " + std::to_string(rows) + " values, not " +
                                       std::to_string(col.num_values));

    ParquetChunk r;
    r.info.rows = rows;
    r.info.pages = (int64_t)pages.size();
    r.info.dictionary_entries = dict_n;
    r.info.dictionary_passing = -1;
    r.info.passing_rows = -1;
    const std::string name = col.name ? col.name : "";
    DevCol out = var ? DevCol{} : make_col(rt, out_t, rows, col.max_def_level > 0, name);
    r.batch.rows = rows;
    DevCol pass;
    if (filter) {
        // bit-packed, written as 32-bit words: room for the last word
        pass.type = DType{Type::Bool, 0, 0};
        pass.length = rows;
        pass.nullable = false;
        pass.name = "pass";
        pass.hold_data = std::make_shared<DBuf>(rt, (size_t)ceil_div(rows, 32) * 4 + 8);
        pass.data = pass.hold_data->get();
        KRV_CUDA(cudaMemsetAsync(pass.hold_data->get(), 0, pass.hold_data->bytes(), rt->stream));
    }
    if (out.valid) KRV_CUDA(cudaMemsetAsync(const_cast<uint8_t *>(out.valid), 0, out.hold_valid->bytes(), rt->stream));
    if (rows > 0) {
        DBuf dchunk(rt, (size_t)bytes);
        KRV_CUDA(cudaMemcpyAsync(dchunk.get(), chunk, (size_t)bytes, cudaMemcpyHostToDevice, rt->stream));
        DBuf staged(rt, (size_t)std::max<int64_t>(staged_bytes, 16));
        DBuf dstages(rt, stages.size() * sizeof(StageDev));
        DBuf dpages(rt, std::max<size_t>(pages.size(), 1) * sizeof(PageDev));
        DBuf counts(rt, 16);
        std::vector<FragDev> frags;
        for (const StageDev &st : stages)
            if (st.snappy) plan_fragments(chunk, st, frags);
        DBuf dfrags(rt, std::max<size_t>(frags.size(), 1) * sizeof(FragDev));
        if (!frags.empty())
            KRV_CUDA(cudaMemcpyAsync(dfrags.get(), frags.data(), frags.size() * sizeof(FragDev), cudaMemcpyHostToDevice,
                                     rt->stream));
        KRV_CUDA(cudaMemcpyAsync(dstages.get(), stages.data(), stages.size() * sizeof(StageDev), cudaMemcpyHostToDevice,
                                 rt->stream));
        KRV_CUDA(cudaMemcpyAsync(dpages.get(), pages.data(), pages.size() * sizeof(PageDev), cudaMemcpyHostToDevice,
                                 rt->stream));
        KRV_CUDA(cudaMemsetAsync(counts.get(), 0, 16, rt->stream));
        clear_status(rt);
        stage_kernel<<<(unsigned)stages.size(), kStageThreads, 0, rt->stream>>>(
            dstages.as<StageDev>(), dchunk.as<uint8_t>(), staged.as<uint8_t>());
        rt->launches++;
        check_launch("stage_kernel");
        if (col.codec == KRV_PQ_SNAPPY) {
            static bool smem_set[64] = {};  // the kernel's attribute, set once per device
            int dev = 0;
            KRV_CUDA(cudaGetDevice(&dev));
            if (dev < 0 || dev >= 64 || !smem_set[dev]) {
                KRV_CUDA(cudaFuncSetAttribute(snappy_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSnappySmem));
                if (dev >= 0 && dev < 64) smem_set[dev] = true;
            }
            if (!frags.empty()) {
                snappy_kernel<<<(unsigned)frags.size(), 32, kSnappySmem, rt->stream>>>(
                    dfrags.as<FragDev>(), dchunk.as<uint8_t>(), staged.as<uint8_t>(), status_word(rt));
                rt->launches++;
                check_launch("snappy_kernel");
            }
        }
        DecodeArgs A{};
        A.pages = dpages.as<PageDev>();
        A.staged = staged.as<uint8_t>();
        A.max_def = col.max_def_level;
        A.pwidth = pwidth;
        A.out_kind = out_kind;
        A.is_int = is_int;
        A.out = const_cast<void *>(out.data);
        A.valid = out.valid ? reinterpret_cast<uint32_t *>(const_cast<uint8_t *>(out.valid)) : nullptr;
        A.status = status_word(rt);
        A.counts = counts.as<unsigned long long>();
        DBuf dict_pass;
        if (dict_stage >= 0) {
            A.dict = staged.as<uint8_t>() + stages[dict_stage].dst;
            A.dict_n = dict_n;
        }
        if (filter) {
            A.has_filter = 1;
            A.f = key_filter_dev(*filter);
            A.pass = reinterpret_cast<uint32_t *>(const_cast<void *>(pass.data));
            if (dict_stage >= 0 && dict_n > 0) {
                dict_pass = DBuf(rt, (size_t)dict_n);
                dict_filter_kernel<<<grid_for(rt, dict_n, 256, 4), 256, 0, rt->stream>>>(
                    A.f, A.dict, dict_n, pwidth, dict_pass.as<uint8_t>(), counts.as<unsigned long long>() + 1);
                rt->launches++;
                check_launch("dict_filter_kernel");
                A.dict_pass = dict_pass.as<uint8_t>();
            }
        } else {
            A.f.nulls_pass = 1;
        }
        // BYTE_ARRAY: the (start, length) table of the dictionary's entries,
        // then of every PLAIN page's values at the page's first row; each
        // row's reference into it.
        DBuf vstarts, vlens, walked, refs, dwalk;
        if (var) {
            const int64_t slots = dict_n + rows;
            vstarts = DBuf(rt, (size_t)std::max<int64_t>(slots, 1) * 8);
            vlens = DBuf(rt, (size_t)std::max<int64_t>(slots, 1) * 4);
            walked = DBuf(rt, std::max<size_t>(pages.size(), 1) * 4);
            refs = DBuf(rt, (size_t)rows * 8);
            KRV_CUDA(cudaMemsetAsync(walked.get(), 0, walked.bytes(), rt->stream));
            std::vector<WalkDev> items;
            if (dict_stage >= 0 && dict_n > 0)
                items.push_back(WalkDev{stages[dict_stage].dst, 0, stages[dict_stage].usize, 0, 0, (int32_t)dict_n, -1, 0});
            for (size_t i = 0; i < pages.size(); i++)
                if (!pages[i].dict)
                    items.push_back(WalkDev{pages[i].staged, dict_n + pages[i].row0, pages[i].usize, pages[i].v2 ? 2 : 1,
                                            pages[i].def_len, pages[i].nvalues, (int32_t)i, 0});
            if (!items.empty()) {
                dwalk = DBuf(rt, items.size() * sizeof(WalkDev));
                KRV_CUDA(cudaMemcpyAsync(dwalk.get(), items.data(), items.size() * sizeof(WalkDev),
                                         cudaMemcpyHostToDevice, rt->stream));
                ba_walk_kernel<<<(unsigned)items.size(), 32, 0, rt->stream>>>(
                    dwalk.as<WalkDev>(), staged.as<uint8_t>(), col.max_def_level, vstarts.as<long long>(),
                    vlens.as<int32_t>(), walked.as<int32_t>(), status_word(rt));
                rt->launches++;
                check_launch("ba_walk_kernel");
            }
            A.ref = refs.as<long long>();
            A.walked = walked.as<int32_t>();
            A.valid = nullptr;  // the gather writes the validity
        }
        if (!pages.empty()) {
            page_decode_kernel<<<(unsigned)pages.size(), kDecodeThreads, 0, rt->stream>>>(A);
            rt->launches++;
            check_launch("page_decode_kernel");
        }
        unsigned long long c[2];
        read_device(rt, counts.get(), 16, c);
        const uint32_t st = take_status(rt);
        if (st & ST_CORRUPT) fail(KRV_INVALID_ARGUMENT, "corrupt Parquet page: its bytes do not decode");
        if (st) fail(KRV_CUDA_ERROR, "Parquet decode status " + std::to_string(st));
        if (var) {
            const VarSrc src{nullptr, vstarts.as<long long>(), vlens.as<int32_t>(), staged.as<uint8_t>(), nullptr, 0};
            out = var_gather(rt, src, refs.as<long long>(), rows, out_t, col.max_def_level > 0, name);
        }
        if (filter) {
            r.info.passing_rows = (int64_t)c[0];
            // the dictionary decides for the chunk only when every data page uses it
            if (dict_stage >= 0 && all_dict) r.info.dictionary_passing = (int64_t)c[1];
        }
    } else {
        if (filter) r.info.passing_rows = 0;
        if (var) out = var_gather(rt, VarSrc{}, nullptr, 0, out_t, col.max_def_level > 0, name);
    }
    r.batch.cols.push_back(out);
    if (filter) r.batch.cols.push_back(pass);
    return r;
}

}  // namespace krv
