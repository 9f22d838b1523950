// Device ingest of whitespace-separated binary u32 relations: the reference's
// load_binary_u32 (crates/sparkalog-storage/src/io.rs:72-138) with the text
// parsed on the GPU instead of by one host thread.
//
// Lines are the text split at '\n'. A line is trimmed of ASCII whitespace;
// empty lines and lines starting with '#' or '%' are skipped; the Git LFS
// pointer header line is an error; any other line must hold exactly two
// whitespace-separated fields, each a u32 in Rust's `str::parse::<u32>`
// syntax (an optional '+', then decimal digits, no overflow).
//
// Pass 1 (line_ends_kernel) compacts the positions of '\n' in order with a
// decoupled look-back. Pass 2 (parse_lines_kernel) gives each thread
// ITEMS consecutive lines, parses them, and compacts the data rows in line
// order (look-back again) into the two output columns. Errors are reduced to
// the smallest failing line index with atomicMin; the host re-reads that one
// line to report its details.
//
// The same two passes read delimited text for load_delimited
// (crates/sparkalog-datalog/src/database.rs:165-177 over
// parse_delimited_parallel, ingest.rs:20-120) when every value is a u32: a
// line (a '\r' before its '\n' dropped) after the optional header that is
// not blank is a record, split at the delimiter byte; a field starting with
// '"' is a quoted string, any other field is trimmed of Unicode whitespace
// and is a u32 when it parses as one (a symbol otherwise).
#pragma once

#include "spk_common.cuh"
#include "spk_setops.cuh"

namespace spk {

constexpr u64 kNoLine = ~0ull;

__device__ __forceinline__ bool ascii_space(unsigned char c) {
    return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r';
}

// Length in bytes of the White_Space character (char::is_whitespace, which
// str::trim strips) that starts at t[p], reading below `end`; 0 if none.
__host__ __device__ __forceinline__ int ws_at(const unsigned char* t, u64 p, u64 end) {
    const unsigned c = t[p];
    if (c == ' ' || (c >= '\t' && c <= '\r')) return 1;
    if (c == 0xC2 && p + 1 < end && (t[p + 1] == 0x85 || t[p + 1] == 0xA0)) return 2;  // U+0085, U+00A0
    if (p + 2 >= end) return 0;
    const unsigned b1 = t[p + 1], b2 = t[p + 2];
    if (c == 0xE1 && b1 == 0x9A && b2 == 0x80) return 3;  // U+1680
    if (c == 0xE2 && b1 == 0x80 && ((b2 >= 0x80 && b2 <= 0x8A) || b2 == 0xA8 || b2 == 0xA9 || b2 == 0xAF))
        return 3;  // U+2000..U+200A, U+2028, U+2029, U+202F
    if (c == 0xE2 && b1 == 0x81 && b2 == 0x9F) return 3;  // U+205F
    if (c == 0xE3 && b1 == 0x80 && b2 == 0x80) return 3;  // U+3000
    return 0;
}

// Length of the White_Space character that ends just before t[p], reading at
// or above `begin`; 0 if none.
__host__ __device__ __forceinline__ int ws_before(const unsigned char* t, u64 begin, u64 p) {
    if (p > begin && ws_at(t, p - 1, p) == 1) return 1;
    if (p >= begin + 2 && ws_at(t, p - 2, p) == 2) return 2;
    if (p >= begin + 3 && ws_at(t, p - 3, p) == 3) return 3;
    return 0;
}

// [*b, *e) trimmed of White_Space at both ends.
__host__ __device__ __forceinline__ void unicode_trim(const unsigned char* t, u64* b, u64* e) {
    for (int k; *b < *e && (k = ws_at(t, *b, *e)) > 0;) *b += k;
    for (int k; *e > *b && (k = ws_before(t, *b, *e)) > 0;) *e -= k;
}

// *count += number of '\n' bytes (sizes the line-end array).
static __global__ void count_newlines_kernel(const unsigned char* text, u64 bytes, unsigned long long* count) {
    const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
    u32 c = 0;
    for (u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; i < bytes; i += stride)
        c += text[i] == '\n' ? 1u : 0u;
    c = __reduce_add_sync(0xffffffffu, c);
    if (lane_id() == 0 && c) atomicAdd(count, static_cast<unsigned long long>(c));
}

template <int THREADS, int ITEMS>
__global__ void __launch_bounds__(THREADS) line_ends_kernel(const unsigned char* text, u64 bytes, u64* ends,
                                                            u64* count, u64* status, u32* tile_counter, u32 epoch,
                                                            u32* err) {
    constexpr int kTile = THREADS * ITEMS;
    __shared__ CompactShared<THREADS> cs;
    __shared__ u64 stage[kTile];
    const u64 num_tiles = (bytes + kTile - 1) / kTile;
    if (num_tiles == 0) {
        if (blockIdx.x == 0 && threadIdx.x == 0) *count = 0;
        return;
    }
    for (;;) {
        if (threadIdx.x == 0) cs.tile = atomicAdd(tile_counter, 1u);
        __syncthreads();
        const u64 tile = cs.tile;
        if (tile >= num_tiles) break;
        const u64 base = tile * kTile + static_cast<u64>(threadIdx.x) * ITEMS;
        u32 keep = 0;
#pragma unroll
        for (int i = 0; i < ITEMS; ++i)
            if (base + i < bytes && text[base + i] == '\n') keep |= 1u << i;
        u32 excl, total;
        const u64 off = compact_offsets<THREADS>(__popc(keep), &excl, &total, tile, status, epoch, err, cs);
        u32 w = excl;
#pragma unroll
        for (int i = 0; i < ITEMS; ++i)
            if (keep & (1u << i)) stage[w++] = base + i;
        __syncthreads();
        for (u32 j = threadIdx.x; j < total; j += THREADS) ends[off + j] = stage[j];
        if (tile == num_tiles - 1 && threadIdx.x == 0) *count = off + total;
        __syncthreads();
    }
}

// u32 per Rust's from_str: optional '+', at least one decimal digit, no overflow.
__host__ __device__ __forceinline__ bool parse_u32_field(const unsigned char* p, u64 len, u32* out) {
    u64 i = 0;
    if (len > 0 && p[0] == '+') i = 1;
    if (i == len) return false;
    u64 v = 0;
    for (; i < len; ++i) {
        const unsigned c = p[i];
        if (c < '0' || c > '9') return false;
        v = v * 10 + (c - '0');
        if (v > 0xffffffffull) return false;
    }
    *out = static_cast<u32>(v);
    return true;
}

// The Git LFS pointer header line.
static __constant__ const char kLfsHeader[] = "version https://git-lfs.github.com/spec/v1";
constexpr int kLfsHeaderLen = 42;

// 0: skipped line, 1: data row, 2: field-count error, 3: u32 error, 4: LFS header.
__device__ __forceinline__ int parse_line(const unsigned char* text, u64 begin, u64 end, u32* first, u32* second) {
    while (begin < end && ascii_space(text[begin])) ++begin;
    while (end > begin && ascii_space(text[end - 1])) --end;
    if (begin == end || text[begin] == '#' || text[begin] == '%') return 0;
    if (end - begin == kLfsHeaderLen) {
        bool same = true;
        for (int k = 0; k < kLfsHeaderLen; ++k) same &= text[begin + k] == static_cast<unsigned char>(kLfsHeader[k]);
        if (same) return 4;
    }
    u64 fb[3], fe[3];
    int fields = 0;
    u64 p = begin;
    while (p < end) {
        while (p < end && ascii_space(text[p])) ++p;
        if (p == end) break;
        const u64 b = p;
        while (p < end && !ascii_space(text[p])) ++p;
        if (fields < 3) {
            fb[fields] = b;
            fe[fields] = p;
        }
        ++fields;
        if (fields > 2) break;
    }
    if (fields != 2) return 2;
    if (!parse_u32_field(text + fb[0], fe[0] - fb[0], first)) return 3;
    if (!parse_u32_field(text + fb[1], fe[1] - fb[1], second)) return 3;
    return 1;
}

// A line parser returns 0 (skipped line), 1 (a row in *first, *second),
// 2 (an error of the first class) or 3 (an error of the second class).

// load_binary_u32: class 2 a field-count or u32 error, class 3 the LFS header.
struct BinaryLineParser {
    __device__ __forceinline__ int operator()(const unsigned char* text, u64, u64 b, u64 e, bool, u32* first,
                                              u32* second) const {
        const int kind = parse_line(text, b, e, first, second);
        return kind == 4 ? 3 : (kind == 3 ? 2 : kind);
    }
};

// One record of parse_record (ingest.rs:43-120) restricted to two u32
// values: 2 for a syntax error (unterminated quote, no delimiter after a
// quoted field, an empty field, a trailing delimiter), 3 for a record that
// parses but is not two u32 values (arity, or a string or symbol value).
__device__ __forceinline__ int parse_delimited_record(const unsigned char* t, u64 b, u64 e, unsigned char delim,
                                                      u32* first, u32* second) {
    u64 pos = b;
    int fields = 0;
    bool not_u32 = false;
    for (;;) {
        if (pos < e && t[pos] == '"') {
            ++pos;
            bool closed = false;
            while (pos < e) {
                if (t[pos] == '"') {
                    if (pos + 1 < e && t[pos + 1] == '"') {
                        pos += 2;
                    } else {
                        ++pos;
                        closed = true;
                        break;
                    }
                } else {
                    ++pos;  // UTF-8 continuation bytes are never '"'
                }
            }
            if (!closed) return 2;
            not_u32 = true;
            if (pos < e && t[pos] != delim) return 2;
        } else {
            const u64 start = pos;
            while (pos < e && t[pos] != delim) ++pos;
            u64 fb = start, fe = pos;
            unicode_trim(t, &fb, &fe);
            if (fb == fe) return 2;
            u32 v = 0;
            if (parse_u32_field(t + fb, fe - fb, &v)) {
                if (fields == 0) *first = v;
                if (fields == 1) *second = v;
            } else {
                not_u32 = true;
            }
        }
        ++fields;
        if (pos == e) break;
        ++pos;
        if (pos == e) return 2;
    }
    return (fields != 2 || not_u32) ? 3 : 1;
}

// load_delimited: the header line skipped, a '\r' before the '\n' dropped,
// blank lines skipped, every other line one record.
struct DelimitedLineParser {
    unsigned char delim;
    bool header;
    __device__ __forceinline__ int operator()(const unsigned char* text, u64 line, u64 b, u64 e, bool newline,
                                              u32* first, u32* second) const {
        if (header && line == 0) return 0;
        if (newline && e > b && text[e - 1] == '\r') --e;
        u64 tb = b, te = e;
        unicode_trim(text, &tb, &te);
        if (tb == te) return 0;
        return parse_delimited_record(text, b, e, delim, first, second);
    }
};

// Line i spans [i == 0 ? 0 : ends[i - 1] + 1, i < ends_n ? ends[i] : bytes).
// first_error[0] = smallest line index whose parser returned 2,
// first_error[1] = smallest line index whose parser returned 3.
template <int THREADS, int ITEMS, class Parser>
__global__ void __launch_bounds__(THREADS) parse_lines_kernel(const unsigned char* text, u64 bytes, const u64* ends,
                                                              const u64* ends_n_ptr, u64 lines, Parser parser,
                                                              u32* out_first, u32* out_second, u64* out_count,
                                                              unsigned long long* first_error, u64* status,
                                                              u32* tile_counter, u32 epoch, u32* err) {
    constexpr int kTile = THREADS * ITEMS;
    __shared__ CompactShared<THREADS> cs;
    __shared__ u64 stage[kTile];
    const u64 ends_n = *ends_n_ptr;
    const u64 num_tiles = (lines + kTile - 1) / kTile;
    if (num_tiles == 0) {
        if (blockIdx.x == 0 && threadIdx.x == 0) *out_count = 0;
        return;
    }
    for (;;) {
        if (threadIdx.x == 0) cs.tile = atomicAdd(tile_counter, 1u);
        __syncthreads();
        const u64 tile = cs.tile;
        if (tile >= num_tiles) break;
        const u64 base = tile * kTile + static_cast<u64>(threadIdx.x) * ITEMS;
        u32 keep = 0;
        u64 row[ITEMS];
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
            row[i] = 0;
            const u64 line = base + i;
            if (line >= lines) continue;
            const u64 b = line == 0 ? 0 : ends[line - 1] + 1;
            const u64 e = line < ends_n ? ends[line] : bytes;
            u32 f = 0, s = 0;
            const int kind = parser(text, line, b, e, line < ends_n, &f, &s);
            if (kind == 1) {
                keep |= 1u << i;
                row[i] = (static_cast<u64>(f) << 32) | s;
            } else if (kind == 2) {
                atomicMin(first_error, static_cast<unsigned long long>(line));
            } else if (kind == 3) {
                atomicMin(first_error + 1, static_cast<unsigned long long>(line));
            }
        }
        u32 excl, total;
        const u64 off = compact_offsets<THREADS>(__popc(keep), &excl, &total, tile, status, epoch, err, cs);
        u32 w = excl;
#pragma unroll
        for (int i = 0; i < ITEMS; ++i)
            if (keep & (1u << i)) stage[w++] = row[i];
        __syncthreads();
        for (u32 j = threadIdx.x; j < total; j += THREADS) {
            out_first[off + j] = static_cast<u32>(stage[j] >> 32);
            out_second[off + j] = static_cast<u32>(stage[j]);
        }
        if (tile == num_tiles - 1 && threadIdx.x == 0) *out_count = off + total;
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Value interning (ValueCatalog::intern, crates/sparkalog-datalog/src/
// catalog.rs:98-127): dense ids by first appearance. The catalog keeps its
// entries as packed (value << 32 | id) sorted by value, and id -> value in
// `dict`. A batch is sorted as (value << 32 | position); the head of each
// value's run that the catalog lacks joins the new-value list with its first
// position; sorting that list by position gives the new ids in appearance
// order; then every batch row finds its id by a merge walk over the catalog.
// ---------------------------------------------------------------------------
static __global__ void value_positions_kernel(const u32* values, u64 n, u64* out) {
    const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
    for (u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
        out[i] = (static_cast<u64>(values[i]) << 32) | i;
}

__device__ __forceinline__ u64 catalog_lower_bound(const u64* keys, u64 n, u32 value) {
    const u64 key = static_cast<u64>(value) << 32;
    u64 lo = 0, hi = n;
    while (lo < hi) {
        const u64 mid = (lo + hi) >> 1;
        if (keys[mid] < key) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Heads of value runs of the sorted batch whose value the catalog lacks:
// new_list[k] = (first position << 32 | value), in no particular order.
static __global__ void new_value_heads_kernel(const u64* sorted, u64 n, const u64* keys, u64 keys_n, u64* new_list,
                                              unsigned long long* new_count) {
    const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
    for (u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const u32 v = static_cast<u32>(sorted[i] >> 32);
        if (i > 0 && static_cast<u32>(sorted[i - 1] >> 32) == v) continue;
        const u64 p = catalog_lower_bound(keys, keys_n, v);
        if (p < keys_n && static_cast<u32>(keys[p] >> 32) == v) continue;
        const unsigned long long k = atomicAdd(new_count, 1ull);
        new_list[k] = (static_cast<u64>(static_cast<u32>(sorted[i])) << 32) | v;
    }
}

// New values in appearance order get ids base, base + 1, ...
static __global__ void assign_new_ids_kernel(const u64* by_position, u64 m, u64 base, u64* pairs, u32* dict) {
    const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
    for (u64 k = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; k < m; k += stride) {
        const u32 v = static_cast<u32>(by_position[k]);
        const u64 id = base + k;
        pairs[k] = (static_cast<u64>(v) << 32) | id;
        dict[id] = v;
    }
}

// ids[position] = catalog id of each row of the sorted batch: one search for
// a thread's first row, then a walk (rows and catalog are both value-sorted).
template <int ITEMS>
__global__ void lookup_ids_kernel(const u64* sorted, u64 n, const u64* keys, u64 keys_n, u32* ids, u32* err) {
    const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x * ITEMS;
    for (u64 base = (static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x) * ITEMS; base < n; base += stride) {
        u64 p = catalog_lower_bound(keys, keys_n, static_cast<u32>(sorted[base] >> 32));
        for (int i = 0; i < ITEMS && base + i < n; ++i) {
            const u64 row = sorted[base + i];
            const u32 v = static_cast<u32>(row >> 32);
            while (p < keys_n && static_cast<u32>(keys[p] >> 32) < v) ++p;
            if (p < keys_n && static_cast<u32>(keys[p] >> 32) == v) {
                ids[static_cast<u32>(row)] = static_cast<u32>(keys[p]);
            } else {
                atomicOr(err, kErrIndexRange);
            }
        }
    }
}

// values[i] = dict[ids[i]]; an id outside the catalog sets kErrIndexRange.
static __global__ void decode_ids_kernel(const u32* ids, u64 n, const u32* dict, u64 size, u32* values, u32* err) {
    const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
    for (u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const u32 id = ids[i];
        if (id < size) {
            values[i] = dict[id];
        } else {
            values[i] = 0;
            atomicOr(err, kErrIndexRange);
        }
    }
}

}  // namespace spk
