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

// ---------------------------------------------------------------------------
// Records of mixed values (InternedValue, crates/sparkalog-datalog/src/
// catalog.rs:10-14: U32, String, Symbol), as parse_record (ingest.rs:43-120)
// yields them. A value is one 64-bit token: bits 63-62 the kind (0 U32, 1
// String, 2 Symbol); a U32 keeps its value in the low 32 bits; a String or
// Symbol keeps the byte offset (bits 61-24) and length (bits 23-0) of its
// raw text: a String's quoted span including its quotes (the only escape is a
// doubled quote, so equal raw spans are exactly equal strings), a Symbol's
// trimmed span.
// ---------------------------------------------------------------------------
constexpr u64 kTokenMaxLength = (1ull << 24) - 1;
constexpr u64 kTokenMaxOffset = (1ull << 38) - 1;

__device__ __forceinline__ u64 make_token(u32 kind, u64 offset, u64 length) {
    return (static_cast<u64>(kind) << 62) | (offset << 24) | length;
}
__device__ __forceinline__ u32 token_kind(u64 t) { return static_cast<u32>(t >> 62); }
__device__ __forceinline__ u64 token_offset(u64 t) { return (t >> 24) & kTokenMaxOffset; }
__device__ __forceinline__ u32 token_length(u64 t) { return static_cast<u32>(t & kTokenMaxLength); }

// 1: two values in *t0, *t1; 2: a syntax error; 3: not two values; 4: a
// String or Symbol longer than kTokenMaxLength bytes.
__device__ __forceinline__ int parse_value_record(const unsigned char* t, u64 b, u64 e, unsigned char delim, u64* t0,
                                                  u64* t1) {
    u64 pos = b;
    int fields = 0;
    bool too_long = false;
    for (;;) {
        u64 token = 0;
        if (pos < e && t[pos] == '"') {
            const u64 start = pos;
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
            if (pos < e && t[pos] != delim) return 2;
            if (pos - start > kTokenMaxLength) too_long = true;
            token = make_token(1, start, (pos - start) & kTokenMaxLength);
        } else {
            const u64 start = pos;
            while (pos < e && t[pos] != delim) ++pos;
            u64 fb = start, fe = pos;
            unicode_trim(t, &fb, &fe);
            if (fb == fe) return 2;
            u32 v = 0;
            if (parse_u32_field(t + fb, fe - fb, &v)) {
                token = v;
            } else {
                if (fe - fb > kTokenMaxLength) too_long = true;
                token = make_token(2, fb, (fe - fb) & kTokenMaxLength);
            }
        }
        if (fields == 0) *t0 = token;
        if (fields == 1) *t1 = token;
        ++fields;
        if (pos == e) break;
        ++pos;
        if (pos == e) return 2;
    }
    if (fields != 2) return 3;
    return too_long ? 4 : 1;
}

// Line i spans [i == 0 ? 0 : ends[i - 1] + 1, i < ends_n ? ends[i] : bytes).
// Every kept line leaves two tokens at out[2 row], out[2 row + 1] (rows in
// line order); first_error[0] / [1] / [2] = smallest line with a syntax
// error / not two values / a too-long value.
template <int THREADS, int ITEMS>
__global__ void __launch_bounds__(THREADS) parse_value_lines_kernel(const unsigned char* text, u64 bytes,
                                                                    const u64* ends, const u64* ends_n_ptr, u64 lines,
                                                                    unsigned char delim, bool header, u64* out,
                                                                    u64* out_count, unsigned long long* first_error,
                                                                    u64* status, u32* tile_counter, u32 epoch,
                                                                    u32* err) {
    constexpr int kTile = THREADS * ITEMS;
    __shared__ CompactShared<THREADS> cs;
    __shared__ u64 stage[2 * kTile];
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
        u64 a[ITEMS], c[ITEMS];
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
            a[i] = c[i] = 0;
            const u64 line = base + i;
            if (line >= lines) continue;
            if (header && line == 0) continue;
            const u64 b = line == 0 ? 0 : ends[line - 1] + 1;
            u64 e = line < ends_n ? ends[line] : bytes;
            if (line < ends_n && e > b && text[e - 1] == '\r') --e;
            u64 tb = b, te = e;
            unicode_trim(text, &tb, &te);
            if (tb == te) continue;
            const int kind = parse_value_record(text, b, e, delim, &a[i], &c[i]);
            if (kind == 1) keep |= 1u << i;
            else atomicMin(first_error + (kind == 2 ? 0 : (kind == 3 ? 1 : 2)), static_cast<unsigned long long>(line));
        }
        u32 excl, total;
        const u64 off = compact_offsets<THREADS>(__popc(keep), &excl, &total, tile, status, epoch, err, cs);
        u32 w = excl;
#pragma unroll
        for (int i = 0; i < ITEMS; ++i)
            if (keep & (1u << i)) {
                stage[2 * w] = a[i];
                stage[2 * w + 1] = c[i];
                ++w;
            }
        __syncthreads();
        for (u32 j = threadIdx.x; j < 2 * total; j += THREADS) out[2 * off + j] = stage[j];
        if (tile == num_tiles - 1 && threadIdx.x == 0) *out_count = off + total;
        __syncthreads();
    }
}

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

// values[i] = dict[ids[i]]; an id outside the catalog, or one of a String
// or Symbol value (kinds[id] != 0, when the catalog holds any), sets
// kErrIndexRange.
static __global__ void decode_ids_kernel(const u32* ids, u64 n, const u32* dict, const u32* kinds, u64 size,
                                         u32* values, u32* err) {
    const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
    for (u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const u32 id = ids[i];
        if (id < size && (!kinds || kinds[id] == 0)) {
            values[i] = dict[id];
        } else {
            values[i] = 0;
            atomicOr(err, kErrIndexRange);
        }
    }
}

// ---------------------------------------------------------------------------
// Interning of mixed values. U32 values take the path above. A String or
// Symbol is keyed by (kind << 62 | a 62-bit hash of its raw bytes); values
// with equal keys are grouped by sorting (group index << 32 | position), and
// every value's bytes are compared with its group's first value and with the
// catalog's stored value of that key, so a hash collision between different
// values is detected (kErrHashCollision) instead of merging them. New values
// of both sorts are then numbered together by first position.
// ---------------------------------------------------------------------------
constexpr u32 kErrHashCollision = 1u << 5;
constexpr u32 kNewValue = 0xffffffffu;

__device__ __forceinline__ u64 mix64(u64 x) {
    // The splitmix64 finaliser (Steele, Lea, Flood 2014).
    x ^= x >> 30;
    x *= 0xBF58476D1CE4E5B9ull;
    x ^= x >> 27;
    x *= 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

__device__ __forceinline__ u64 value_key(const unsigned char* p, u32 len, u32 kind) {
    u64 h = mix64(0x9E3779B97F4A7C15ull ^ (static_cast<u64>(kind) << 56) ^ len);
    u32 i = 0;
    for (; i + 8 <= len; i += 8) {
        u64 w = 0;
        for (int b = 0; b < 8; ++b) w |= static_cast<u64>(p[i + b]) << (8 * b);
        h = mix64(h ^ w);
    }
    u64 w = 0;
    for (u32 b = 0; i + b < len; ++b) w |= static_cast<u64>(p[i + b]) << (8 * b);
    h = mix64(h ^ w ^ 0x5555555555555555ull);
    return (static_cast<u64>(kind) << 62) | (h >> 2);
}

__device__ __forceinline__ bool same_bytes(const unsigned char* a, const unsigned char* b, u32 len) {
    for (u32 i = 0; i < len; ++i)
        if (a[i] != b[i]) return false;
    return true;
}

// U32 tokens to ukeys (value << 32 | position), String/Symbol tokens to
// (skeys, spos); each list compacted by an atomic counter (its order does
// not matter: both are sorted next).
static __global__ void classify_tokens_kernel(const u64* tokens, u64 n, const unsigned char* text, u64* ukeys,
                                              unsigned long long* ucount, u64* skeys, u32* spos,
                                              unsigned long long* scount) {
    const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
    for (u64 p = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; p < n; p += stride) {
        const u64 t = tokens[p];
        const u32 kind = token_kind(t);
        if (kind == 0) {
            ukeys[atomicAdd(ucount, 1ull)] = (static_cast<u64>(static_cast<u32>(t)) << 32) | p;
        } else {
            const unsigned long long k = atomicAdd(scount, 1ull);
            skeys[k] = value_key(text + token_offset(t), token_length(t), kind);
            spos[k] = static_cast<u32>(p);
        }
    }
}

__device__ __forceinline__ u64 lower_bound_u64(const u64* a, u64 n, u64 key) {
    u64 lo = 0, hi = n;
    while (lo < hi) {
        const u64 mid = (lo + hi) >> 1;
        if (a[mid] < key) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// pairs[k] = (group << 32 | position), group = first index of the key in
// the sorted keys (one per distinct key).
static __global__ void group_pairs_kernel(const u64* skeys, const u32* spos, u64 ns, const u64* sorted_keys,
                                          u64* pairs) {
    const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
    for (u64 k = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; k < ns; k += stride)
        pairs[k] = (lower_bound_u64(sorted_keys, ns, skeys[k]) << 32) | spos[k];
}

// The catalog's String/Symbol values: raw bytes in an arena, one
// (offset, length) per string index, and the lookup index sorted by key
// (keys, the value id, the string index).
struct StringTable {
    const unsigned char* arena;
    const u64* offset;
    const u32* length;
    const u64* keys;
    const u32* ids;
    const u32* index;
    u64 count;
};

// Group heads (the first position of each distinct key): head[g], the
// catalog id of the value (or kNewValue, then (position << 32 | g) joins
// the new list), with the bytes checked against the catalog's value.
static __global__ void string_heads_kernel(const u64* sorted_pairs, u64 ns, const u64* sorted_keys, const u64* tokens,
                                           const unsigned char* text, StringTable cat, u32* head, u32* id_of,
                                           u32* is_new, u64* new_list, unsigned long long* new_count, u32* err) {
    const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
    for (u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; i < ns; i += stride) {
        const u32 g = static_cast<u32>(sorted_pairs[i] >> 32);
        if (i > 0 && static_cast<u32>(sorted_pairs[i - 1] >> 32) == g) continue;
        const u32 pos = static_cast<u32>(sorted_pairs[i]);
        head[g] = pos;
        const u64 key = sorted_keys[g];
        const u64 c = lower_bound_u64(cat.keys, cat.count, key);
        if (c < cat.count && cat.keys[c] == key) {
            const u64 t = tokens[pos];
            const u32 si = cat.index[c];
            if (cat.length[si] != token_length(t) ||
                !same_bytes(cat.arena + cat.offset[si], text + token_offset(t), token_length(t)))
                atomicOr(err, kErrHashCollision);
            id_of[g] = cat.ids[c];
        } else {
            id_of[g] = kNewValue;
            is_new[g] = 1;
            new_list[atomicAdd(new_count, 1ull)] = (static_cast<u64>(pos) << 32) | g;
        }
    }
}

// The joint list of new values: U32 heads (position << 32 | value) and
// string heads (position << 32 | group) as (position << 33 | sort << 32 |
// payload), which sorts by first position.
static __global__ void joint_entries_kernel(const u64* ulist, u64 mu, const u64* slist, u64 ms, u64* out) {
    const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
    for (u64 k = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; k < mu + ms; k += stride) {
        const u64 e = k < mu ? ulist[k] : slist[k - mu];
        const u64 pos = e >> 32;
        out[k] = (pos << 33) | (static_cast<u64>(k < mu ? 0 : 1) << 32) | static_cast<u32>(e);
    }
}

// ids[k], index[k] of each sorted new key, fetched through its group (the
// first index of the key among the batch's sorted keys).
static __global__ void keyed_payload_kernel(const u64* keys, u64 m, const u64* sorted_keys, u64 ns, const u32* id_of,
                                            const u32* si_of, u32* ids, u32* index) {
    const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
    for (u64 k = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; k < m; k += stride) {
        const u64 g = lower_bound_u64(sorted_keys, ns, keys[k]);
        ids[k] = id_of[g];
        index[k] = si_of[g];
    }
}

// Every grouped value has its head's bytes (else two different values share
// a key).
static __global__ void verify_groups_kernel(const u64* sorted_pairs, u64 ns, const u32* head, const u64* tokens,
                                            const unsigned char* text, u32* err) {
    const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
    for (u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; i < ns; i += stride) {
        const u32 g = static_cast<u32>(sorted_pairs[i] >> 32);
        const u32 pos = static_cast<u32>(sorted_pairs[i]);
        const u32 h = head[g];
        if (h == pos) continue;
        const u64 a = tokens[pos], b = tokens[h];
        if (token_length(a) != token_length(b) ||
            !same_bytes(text + token_offset(a), text + token_offset(b), token_length(a)))
            atomicOr(err, kErrHashCollision);
    }
}

// New values of both sorts in first-position order: entry (position << 33 |
// sort << 32 | payload), payload the U32 value (sort 0) or the group (sort
// 1). Rank r gets id base + r. A U32 joins (value << 32 | id) for the U32
// index; a string gets string index str_base + (its rank among strings,
// counted by atomics) and its raw bytes are reserved in the arena.
static __global__ void assign_joint_ids_kernel(const u64* sorted, u64 m, u64 base, u64 str_base, u32* dict,
                                               u32* kinds, u64* upairs, unsigned long long* ucount, u32* id_of,
                                               u32* si_of, const u32* head, const u64* tokens, u64* str_offset,
                                               u32* str_length, unsigned long long* arena_used, u32* str_src,
                                               unsigned long long* scount) {
    const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
    for (u64 r = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; r < m; r += stride) {
        const u64 e = sorted[r];
        const u32 payload = static_cast<u32>(e);
        const u32 id = static_cast<u32>(base + r);
        if (((e >> 32) & 1u) == 0) {
            upairs[atomicAdd(ucount, 1ull)] = (static_cast<u64>(payload) << 32) | id;
            dict[id] = payload;
            kinds[id] = 0;
        } else {
            const u32 g = payload;
            const u64 t = tokens[head[g]];
            const u64 si = str_base + atomicAdd(scount, 1ull);
            id_of[g] = id;
            si_of[g] = static_cast<u32>(si);
            dict[id] = static_cast<u32>(si);
            kinds[id] = token_kind(t);
            str_length[si] = token_length(t);
            str_offset[si] = atomicAdd(arena_used, static_cast<unsigned long long>(token_length(t)));
            str_src[si - str_base] = head[g];
        }
    }
}

// One warp per new string: its raw bytes from the text into the arena.
static __global__ void copy_strings_kernel(const u32* str_src, u64 count, u64 str_base, const u64* tokens,
                                           const unsigned char* text, const u64* str_offset, unsigned char* arena) {
    const u64 warps = static_cast<u64>(gridDim.x) * (blockDim.x / kWarp);
    for (u64 k = (static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x) / kWarp; k < count; k += warps) {
        const u64 t = tokens[str_src[k]];
        const unsigned char* src = text + token_offset(t);
        unsigned char* dst = arena + str_offset[str_base + k];
        for (u32 b = lane_id(); b < token_length(t); b += kWarp) dst[b] = src[b];
    }
}

// The new strings' keys (in group order, which is key order) for the
// catalog's index, with their ids and string indices.
static __global__ void new_string_keys_kernel(const u64* sorted_keys, u64 ns, const u32* id_of, const u32* si_of,
                                              const u32* group_is_new, u64* keys, u32* ids, u32* index,
                                              unsigned long long* count) {
    const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
    for (u64 g = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; g < ns; g += stride) {
        if (!group_is_new[g]) continue;
        const unsigned long long k = atomicAdd(count, 1ull);
        keys[k] = sorted_keys[g];
        ids[k] = id_of[g];
        index[k] = si_of[g];
    }
}

// Merge of two key-sorted (key, id, index) lists with distinct keys: each
// element's output position is its own index plus its rank in the other list.
static __global__ void merge_keyed_kernel(const u64* ak, const u32* ai, const u32* ax, u64 na, const u64* bk,
                                          const u32* bi, const u32* bx, u64 nb, u64* ok, u32* oi, u32* ox) {
    const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
    for (u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; i < na + nb; i += stride) {
        u64 key, o;
        u32 id, x;
        if (i < na) {
            key = ak[i];
            id = ai[i];
            x = ax[i];
            o = i + lower_bound_u64(bk, nb, key);
        } else {
            const u64 j = i - na;
            key = bk[j];
            id = bi[j];
            x = bx[j];
            o = j + lower_bound_u64(ak, na, key);
        }
        ok[o] = key;
        oi[o] = id;
        ox[o] = x;
    }
}

// ids[position] of every String/Symbol value from its group.
static __global__ void string_ids_kernel(const u64* sorted_pairs, u64 ns, const u32* id_of, u32* ids) {
    const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
    for (u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; i < ns; i += stride)
        ids[static_cast<u32>(sorted_pairs[i])] = id_of[static_cast<u32>(sorted_pairs[i] >> 32)];
}

// Row r of the relation: (ids[2r], ids[2r + 1]).
static __global__ void split_rows_kernel(const u32* ids, u64 rows, u32* c0, u32* c1) {
    const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
    for (u64 r = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; r < rows; r += stride) {
        c0[r] = ids[2 * r];
        c1[r] = ids[2 * r + 1];
    }
}

}  // namespace spk
