// Fused join -> order for rules whose join output starts with DELTA's first
// column (the transitive-closure shape path(x, z) :- path(x, y), edge(y, z)):
// the candidate rows of a round reach HBM only once, already sorted.
//
// DELTA is sorted by (first, second), and the join emits DELTA-row-major, so
// the join output is already ordered by its first column x. A tile takes a
// range of DELTA rows aligned to x boundaries, so its join output is a set of
// complete x-runs: ordering the tile's output in shared memory orders it
// globally (x-runs of different tiles never interleave). Within an x-run the
// rows are placed by rank (a row's position is the number of smaller rows of
// its run, ties broken by emission order) when every run is short, else the
// tile is sorted by (run, second column) with a stable LSD radix sort in
// shared memory over only the bits that vary. Tiles are placed with a
// decoupled look-back in tile order, which is x order; a tile publishes its
// size as soon as its join count is known, so the wait overlaps its ordering
// work. Equal rows stay adjacent: the anti-join against FULL that consumes
// this output keeps the first of each run of equal rows (BinaryDistinct).
//
// A tile whose x-run is longer than the tile's row capacity, or whose output
// exceeds the shared-memory capacity, sets *fallback; the host then redoes
// the round with the general kernels (join, radix sort, anti-join).
#pragma once

#include "spk_common.cuh"
#include "spk_engine_kernels.cuh"
#include "spk_join.cuh"
#include "spk_setops.cuh"

namespace spk {

struct FusedRoundArgs {
    const u64* delta;
    u64 delta_rows;
    const u64* delta_rows_ptr;  // when set, the DELTA row count is read here (device-driven rounds)
    u32 rows_per_tile;        // nominal DELTA rows per tile (x boundaries move it)
    u32 left_key;             // DELTA column joined on the right relation's key
    // Index of the right relation on the join key (DELTA's second column).
    const u32* dense_offsets;
    u64 dense_keys;
    const u32* bucket_dir;
    u32 bucket_shift;
    u64 buckets;
    const u32* keys32;
    const u32* rows;          // null: identity
    const u64* right;
    // The right relation's second column alone (identity index on column 0,
    // projecting that column): the gathers read 4-byte values from an array
    // half the size of the rows, which L2 holds more of.
    const u32* right_values;
    // Compact form of that index (with right_values): 4-bit match counts,
    // eight keys to a word (15: read the offsets), and a word per key holding
    // its single match, else its first offset into right_values. Keys without
    // matches then cost a probe of the count words only, which L2 holds.
    const u32* key_class;
    const u32* key_word;
    u32 v1_side;              // 0: DELTA column, 1: right column
    u32 v1_col;
    u32 v1_bits;              // significant bits of the second output column
    u64* out;                 // sorted distinct join output
    u64* out_count;
    unsigned long long* join_rows;  // total join output rows (statistics)
    u64* status;
    u32* tile_counter;
    u32 epoch;
    u32* err;
    u32* fallback;
};

__device__ __forceinline__ void index_lookup(const FusedRoundArgs& a, u32 key, u32* begin, u32* count) {
    *begin = 0;
    *count = 0;
    if (a.dense_offsets) {
        if (key < a.dense_keys) {
            *begin = a.dense_offsets[key];
            *count = a.dense_offsets[key + 1] - *begin;
        }
        return;
    }
    const u64 b = static_cast<u64>(key) >> a.bucket_shift;
    if (b >= a.buckets) return;
    u64 lo = a.bucket_dir[b], hi = a.bucket_dir[b + 1];
    while (lo < hi) {
        const u64 mid = (lo + hi) >> 1;
        if (a.keys32[mid] < key) lo = mid + 1;
        else hi = mid;
    }
    u64 up = lo, top = a.bucket_dir[b + 1];
    while (up < top) {
        const u64 mid = (up + top) >> 1;
        if (a.keys32[mid] <= key) up = mid + 1;
        else top = mid;
    }
    *begin = static_cast<u32>(lo);
    *count = static_cast<u32>(up - lo);
}

// Shared-memory layout of one CTA (dynamic shared memory).
template <int THREADS, int CAP, int ROWCAP>
struct FusedLayout {
    static constexpr int kWarps = THREADS / kWarp;
    static constexpr size_t kKeysA = 0;                                        // u64[CAP]
    static constexpr size_t kKeysB = kKeysA + CAP * sizeof(u64);               // u64[CAP]
    static constexpr size_t kRangeLo = kKeysB + CAP * sizeof(u64);             // u32[ROWCAP]
    static constexpr size_t kRangeHi = kRangeLo + ROWCAP * sizeof(u32);        // u32[ROWCAP]
    static constexpr size_t kRunX = kRangeHi + ROWCAP * sizeof(u32);           // u32[ROWCAP]
    static constexpr size_t kRunOff = kRunX + ROWCAP * sizeof(u32);            // u32[ROWCAP + 4]
    static constexpr size_t kRank = kRunOff + (ROWCAP + 4) * sizeof(u32);      // u16[CAP]
    // The radix sort's counters reuse the index ranges' bytes: the ranges are
    // dead once the matches are emitted, before any sort.
    static constexpr size_t kWarpCount = kRangeLo;                              // u16[kWarps][256]
    static constexpr size_t kDigitStart = kWarpCount + kWarps * 256 * sizeof(unsigned short);  // u32[256]
    static_assert(kWarps * 256 * sizeof(unsigned short) + 256 * sizeof(u32) <= 2 * ROWCAP * sizeof(u32),
                  "sort counters fit the index ranges");
    static constexpr size_t kBytes = kRank + CAP * sizeof(unsigned short);
};

// Stable LSD radix sort of n <= CAP keys in shared memory over the 8-bit
// digits at `shifts`. Keys start in *src; on return *src points at the
// sorted keys (the buffers alternate). Must be called by all threads.
template <int THREADS, int CAP>
__device__ void smem_radix_sort(u64** src, u64** dst, u32 n, const int* shifts, int passes, unsigned short* rank,
                                unsigned short* warp_count, u32* digit_start, u32* scan_scratch) {
    constexpr int kWarps = THREADS / kWarp;
    constexpr int kDigits = THREADS >= 256 ? 1 : 256 / THREADS;
    static_assert(THREADS >= 256 || 256 % THREADS == 0, "digits split evenly over threads");
    const u32 lane = lane_id(), warp = warp_id();
    const u32 chunk = ((n + kWarps - 1) / kWarps + kWarp - 1) / kWarp * kWarp;  // per-warp run, multiple of 32
    for (int p = 0; p < passes; ++p) {
        const int sh = shifts[p];
        u64* a = *src;
        u64* b = *dst;
        for (int i = threadIdx.x; i < kWarps * 256; i += THREADS) warp_count[i] = 0;
        __syncthreads();
        const u32 w0 = warp * chunk;
        for (u32 j = 0; j < chunk; j += kWarp) {
            const u32 pos = w0 + j + lane;
            const bool valid = pos < n;
            const u32 d = valid ? static_cast<u32>((a[pos] >> sh) & 255) : 256u;
            const u32 peers = __match_any_sync(0xffffffffu, d);
            const u32 before = __popc(peers & lanemask_lt());
            u32 base = 0;
            if (valid) base = warp_count[warp * 256 + d];
            __syncwarp();
            if (valid && before == 0) warp_count[warp * 256 + d] = static_cast<unsigned short>(base + __popc(peers));
            __syncwarp();
            if (valid) rank[pos] = static_cast<unsigned short>(base + before);
        }
        __syncthreads();
        // Each thread owns kDigits consecutive digits: exclusive prefix of a
        // digit over warps, then over digits.
        u32 digit_total[kDigits];
        u32 thread_sum = 0;
#pragma unroll
        for (int j = 0; j < kDigits; ++j) {
            const u32 d = threadIdx.x * kDigits + j;
            u32 running = 0;
            if (d < 256) {
                for (int w = 0; w < kWarps; ++w) {
                    const u32 c = warp_count[w * 256 + d];
                    warp_count[w * 256 + d] = static_cast<unsigned short>(running);
                    running += c;
                }
            }
            digit_total[j] = running;
            thread_sum += running;
        }
        u32 total;
        u32 start = block_exclusive_scan<THREADS>(thread_sum, scan_scratch, &total);
#pragma unroll
        for (int j = 0; j < kDigits; ++j) {
            const u32 d = threadIdx.x * kDigits + j;
            if (d < 256) digit_start[d] = start;
            start += digit_total[j];
        }
        __syncthreads();
        for (u32 pos = threadIdx.x; pos < n; pos += THREADS) {
            const u64 k = a[pos];
            const u32 d = static_cast<u32>((k >> sh) & 255);
            b[digit_start[d] + warp_count[(pos / chunk) * 256 + d] + rank[pos]] = k;
        }
        __syncthreads();
        *src = b;
        *dst = a;
    }
}

// Shared-memory radix passes for a tile: the digits of the second column's
// significant bits, then those of the x-run rank.
__device__ __forceinline__ int fused_sort_shifts(u32 v1_bits, u32 runs, int* shifts) {
    int passes = 0;
    for (int b = 0; b < static_cast<int>(v1_bits); b += 8) shifts[passes++] = b;
    const int rbits = runs > 1 ? 32 - __clz(runs - 1) : 0;  // one x-run: nothing to sort on
    for (int b = 0; b < rbits; b += 8) shifts[passes++] = 32 + b;
    return passes;
}

// Runs with at most this many output rows are placed by rank.
constexpr u32 kRankRun = 48;

// DELTA rows a tile's window reaches past its nominal end, so that the x
// boundary that ends the tile is usually found in shared memory.
constexpr u64 kWindowExtra = 128;

// Packed per-thread scan value: match count in the low kCountBits, x-run
// starts above (a tile has fewer than 2048 rows, so starts fit in 11 bits).
constexpr int kCountBits = 52;
constexpr u64 kCountMask = (1ull << kCountBits) - 1;

template <int THREADS, int CAP, int ROWCAP>
__device__ __forceinline__ void fused_round(const FusedRoundArgs& a) {
    using L = FusedLayout<THREADS, CAP, ROWCAP>;
    constexpr int kRowItems = ROWCAP / THREADS;
    static_assert(ROWCAP % THREADS == 0, "rows split evenly over threads");
    static_assert(ROWCAP < 2048 && CAP < 65536, "11-bit run starts, 16-bit ranks and counts");
    static_assert(ROWCAP <= CAP, "DELTA rows are staged in the second key buffer");
    extern __shared__ __align__(16) unsigned char smem[];
    u64* keys_a = reinterpret_cast<u64*>(smem + L::kKeysA);
    u64* keys_b = reinterpret_cast<u64*>(smem + L::kKeysB);
    u32* range_lo = reinterpret_cast<u32*>(smem + L::kRangeLo);
    u32* range_hi = reinterpret_cast<u32*>(smem + L::kRangeHi);
    u32* run_x = reinterpret_cast<u32*>(smem + L::kRunX);
    u32* run_off = reinterpret_cast<u32*>(smem + L::kRunOff);
    unsigned short* rank = reinterpret_cast<unsigned short*>(smem + L::kRank);
    unsigned short* warp_count = reinterpret_cast<unsigned short*>(smem + L::kWarpCount);
    u32* digit_start = reinterpret_cast<u32*>(smem + L::kDigitStart);
    __shared__ u64 scan_scratch[THREADS / kWarp + 1];
    __shared__ u32 scan_scratch32[THREADS / kWarp + 1];
    __shared__ u64 bounds[2];
    __shared__ u64 tile_shared, out_base;

    const u64 n = a.delta_rows_ptr ? *a.delta_rows_ptr : a.delta_rows;
    const u64 R = a.rows_per_tile;
    const u64 num_tiles = (n + R - 1) / R;
    if (num_tiles == 0) {
        if (blockIdx.x == 0 && threadIdx.x == 0) *a.out_count = 0;
        return;
    }
    // Join rows of this CTA's tiles (thread 0), added to the total once at
    // the end: an atomic per tile on the one counter serialised the tiles.
    unsigned long long join_tally = 0;
    for (;;) {
        if (threadIdx.x == 0) tile_shared = atomicAdd(a.tile_counter, 1u);
        __syncthreads();
        const u64 tile = tile_shared;
        if (tile >= num_tiles) break;

        // 1. Rows [B(tile), B(tile + 1)): the first x boundary at or after each
        // nominal start. The window [p0 - 1, p1 + extra) of DELTA rows comes
        // into shared memory first (keys_b is free until the emitted keys are
        // ordered) and both boundaries are found there (warp 0: begin, warp 1:
        // end); only an x-run that reaches past the window sends a warp on to
        // scan global memory, up to ROWCAP rows.
        const u64 p0 = tile * R;
        const u64 p1 = p0 + R < n ? p0 + R : n;
        const u64 w0 = p0 > 0 ? p0 - 1 : 0;
        const u64 extra = R + 1 + kWindowExtra <= static_cast<u64>(CAP) ? kWindowExtra
                          : static_cast<u64>(CAP) > R + 1 ? CAP - 1 - R : 0;
        const u64 w1 = p1 + extra < n ? p1 + extra : n;
        u64* win = keys_b;
        for (u32 r = threadIdx.x; r < w1 - w0; r += THREADS) cp_async_8(win + r, a.delta + w0 + r);
        cp_async_commit();
        cp_async_wait<0>();
        __syncthreads();
        if (warp_id() < 2) {
            const u64 p = warp_id() == 0 ? p0 : p1;
            u64 found = ~0ull;
            if (p == 0) {
                found = 0;
            } else if (p >= n) {
                found = n;
            } else {
                // p - 1 >= w0, so every row compared here lies in the window.
                for (u64 base = p; base <= w1 && found == ~0ull; base += kWarp) {
                    const u64 q = base + lane_id();
                    const bool boundary = q < w1 ? (win[q - w0] >> 32) != (win[q - 1 - w0] >> 32) : (q == w1 && w1 == n);
                    const u32 m = __ballot_sync(0xffffffffu, boundary);
                    if (m) found = base + (__ffs(m) - 1);
                }
                for (u64 base = w1; base < p + ROWCAP && found == ~0ull; base += kWarp) {
                    const u64 q = base + lane_id();
                    const bool boundary = q >= n || (a.delta[q] >> 32) != (a.delta[q - 1] >> 32);
                    const u32 m = __ballot_sync(0xffffffffu, boundary);
                    if (m) found = base + (__ffs(m) - 1);
                }
                if (found != ~0ull && found > n) found = n;
            }
            if (lane_id() == 0) bounds[warp_id()] = found;
        }
        __syncthreads();
        const u64 row0 = bounds[0], row1 = bounds[1];
        const bool rows_ok = row0 != ~0ull && row1 != ~0ull && row1 - row0 <= static_cast<u64>(ROWCAP);
        const u32 nrows = rows_ok ? static_cast<u32>(row1 - row0) : 0u;

        // 2. The tile's DELTA rows: in the window already unless an x-run
        // reached past it (then reloaded into keys_b). Then every row's index
        // range, gathered with asynchronous copies (each thread issues all of
        // its gathers, then waits once).
        u64* trow = rows_ok ? win + (row0 - w0) : win;
        if (rows_ok && row1 > w1) {
            trow = keys_b;
            for (u32 r = threadIdx.x; r < nrows; r += THREADS) cp_async_8(trow + r, a.delta + row0 + r);
            cp_async_commit();
            cp_async_wait<0>();
            __syncthreads();
        }
        if (a.key_class) {
            // Each thread probes its own rows (the ones it scans below): the
            // counts first, then the words of the keys that have matches,
            // still in flight during the scan.
            const u32 r0 = threadIdx.x * kRowItems;
            u32 key[kRowItems], cls[kRowItems];
#pragma unroll
            for (int i = 0; i < kRowItems; ++i) {
                const u32 r = r0 + i;
                key[i] = r < nrows ? pair_col(trow[r], a.left_key) : 0u;
                cls[i] = (r < nrows && key[i] < a.dense_keys) ? __ldg(a.key_class + (key[i] >> 3)) : 0u;
            }
#pragma unroll
            for (int i = 0; i < kRowItems; ++i) {
                const u32 r = r0 + i;
                if (r < nrows) {
                    u32 c = (cls[i] >> ((key[i] & 7u) * 4u)) & 15u;
                    if (c == 15u) c = a.dense_offsets[key[i] + 1] - a.dense_offsets[key[i]];
                    range_hi[r] = c;
                    if (c) cp_async_4(range_lo + r, a.key_word + key[i]);
                }
            }
            cp_async_commit();
        } else if (a.dense_offsets) {
            for (u32 r = threadIdx.x; r < nrows; r += THREADS) {
                const u32 key = pair_col(trow[r], a.left_key);
                if (key < a.dense_keys) {
                    cp_async_4(range_lo + r, a.dense_offsets + key);
                    cp_async_4(range_hi + r, a.dense_offsets + key + 1);
                } else {
                    range_lo[r] = range_hi[r] = 0;
                }
            }
            cp_async_commit();
            cp_async_wait<0>();
        } else {
            for (u32 r = threadIdx.x; r < nrows; r += THREADS) {
                u32 f, c;
                index_lookup(a, pair_col(trow[r], a.left_key), &f, &c);
                range_lo[r] = f;
                range_hi[r] = f + c;
            }
        }
        __syncthreads();

        // 3. One scan of (x-run starts, match counts) over the rows (each
        // thread owns kRowItems consecutive rows), then every thread emits
        // its rows' matches: the run's rank per output and the right row (or
        // DELTA row) gathered into keys_a.
        const u32 local0 = threadIdx.x * kRowItems;
        u64 packed = 0;
#pragma unroll
        for (int i = 0; i < kRowItems; ++i) {
            const u32 r = local0 + i;
            if (r < nrows) {
                const u64 start = (r == 0 || (trow[r] >> 32) != (trow[r - 1] >> 32)) ? 1u : 0u;
                packed += (start << kCountBits) + (a.key_class ? range_hi[r] : range_hi[r] - range_lo[r]);
            }
        }
        u64 packed_total;
        const u64 packed_excl = block_exclusive_scan<THREADS>(packed, scan_scratch, &packed_total);
        const u64 total64 = packed_total & kCountMask;
        const u32 runs = static_cast<u32>(packed_total >> kCountBits);
        const bool ok = rows_ok && total64 <= static_cast<u64>(CAP);
        const u32 total = ok ? static_cast<u32>(total64) : 0u;
        u32* match_row = reinterpret_cast<u32*>(keys_a) + CAP;  // row ids of an indexed right relation
        if (a.key_class) cp_async_wait<0>();  // this thread's key words
        if (ok) {
            u32 off = static_cast<u32>(packed_excl & kCountMask);
            u32 rk = static_cast<u32>(packed_excl >> kCountBits);
#pragma unroll
            for (int i = 0; i < kRowItems; ++i) {
                const u32 r = local0 + i;
                if (r < nrows) {
                    const u64 row = trow[r];
                    if (r == 0 || (row >> 32) != (trow[r - 1] >> 32)) {
                        run_x[rk] = static_cast<u32>(row >> 32);
                        run_off[rk] = off;
                        ++rk;
                    }
                    const u32 first = range_lo[r];
                    const u32 count = a.key_class ? range_hi[r] : range_hi[r] - first;
                    for (u32 k = 0; k < count; ++k) {
                        const u32 o = off + k;
                        rank[o] = static_cast<unsigned short>(rk - 1);
                        if (a.v1_side != 1) keys_a[o] = row;
                        else if (a.rows) cp_async_4(match_row + o, a.rows + first + k);
                        else if (a.key_class && count == 1) match_row[o] = first;
                        else if (a.right_values) cp_async_4(match_row + o, a.right_values + first + k);
                        else cp_async_8(keys_a + o, a.right + first + k);
                    }
                    off += count;
                }
            }
        }
        if (threadIdx.x == 0) {
            run_off[runs < ROWCAP ? runs : ROWCAP] = total;
            if (ok) join_tally += total;
            if (!ok) atomicOr(a.fallback, 1u);
            // Publish the tile's output size now: successors resolve their
            // offsets while this tile still orders its rows.
            lookback_publish(a.status, tile, total, a.epoch);
        }
        cp_async_commit();
        cp_async_wait<0>();
        __syncthreads();
        if (a.v1_side == 1 && a.rows) {
            // Indexed right relation: the row ids arrived, now the rows (into
            // keys_b; the DELTA rows are no longer needed).
            for (u32 o = threadIdx.x; o < total; o += THREADS) cp_async_8(keys_b + o, a.right + match_row[o]);
            cp_async_commit();
            cp_async_wait<0>();
            __syncthreads();
        }
        int long_run = 0;
        if (a.v1_side == 1 && !a.rows && a.right_values) {
            // The gathered values share keys_a's bytes: every thread reads
            // its values before any thread writes a key.
            constexpr int kPer = (CAP + THREADS - 1) / THREADS;
            u32 vals[kPer];
#pragma unroll
            for (int i = 0; i < kPer; ++i) {
                const u32 o = threadIdx.x + i * THREADS;
                vals[i] = o < total ? match_row[o] : 0u;
            }
            __syncthreads();
#pragma unroll
            for (int i = 0; i < kPer; ++i) {
                const u32 o = threadIdx.x + i * THREADS;
                if (o < total) keys_a[o] = (static_cast<u64>(rank[o]) << 32) | vals[i];
            }
            for (u32 r = threadIdx.x; r < (ok ? runs : 0u); r += THREADS)
                long_run |= run_off[r + 1] - run_off[r] > kRankRun ? 1 : 0;
        } else {
            const u64* raw = (a.v1_side == 1 && a.rows) ? keys_b : keys_a;
            for (u32 o = threadIdx.x; o < total; o += THREADS)
                keys_a[o] = (static_cast<u64>(rank[o]) << 32) | pair_col(raw[o], a.v1_col);
            for (u32 r = threadIdx.x; r < (ok ? runs : 0u); r += THREADS)
                long_run |= run_off[r + 1] - run_off[r] > kRankRun ? 1 : 0;
        }
        long_run = __syncthreads_or(long_run);

        // 4. Order the tile by (x, second column) into `sorted`.
        u64* sorted;
        if (!long_run) {
            // Rank placement within each (short) x-run; equal rows keep
            // their emission order, so every output slot is written once.
            for (u32 o = threadIdx.x; o < total; o += THREADS) {
                const u64 k = keys_a[o];
                const u32 r = static_cast<u32>(k >> 32), v = static_cast<u32>(k);
                const u32 s0 = run_off[r], s1 = run_off[r + 1];
                u32 before = 0;
                for (u32 j = s0; j < s1; ++j) {
                    const u32 w = static_cast<u32>(keys_a[j]);
                    before += (w < v || (w == v && j < o)) ? 1u : 0u;
                }
                keys_b[s0 + before] = (static_cast<u64>(run_x[r]) << 32) | v;
            }
            sorted = keys_b;
        } else {
            int shifts[8];
            const int passes = fused_sort_shifts(a.v1_bits, runs, shifts);
            u64* src = keys_a;
            u64* dst = keys_b;
            smem_radix_sort<THREADS, CAP>(&src, &dst, total, shifts, passes, rank, warp_count, digit_start,
                                          scan_scratch32);
            for (u32 o = threadIdx.x; o < total; o += THREADS) {
                const u64 k = src[o];
                src[o] = (static_cast<u64>(run_x[k >> 32]) << 32) | static_cast<u32>(k);
            }
            sorted = src;
        }

        // 5. The tile's offset (its predecessors have mostly published by
        // now), then the ordered rows out, coalesced. Duplicates stay: the
        // anti-join that consumes this output drops adjacent equal rows.
        if (warp_id() == 0) {
            const u64 g = warp_lookback_resolve(a.status, tile, total, a.epoch, a.err);
            if (lane_id() == 0) out_base = g;
        }
        __syncthreads();
        const u64 base = out_base;
        for (u32 o = threadIdx.x; o < total; o += THREADS) a.out[base + o] = sorted[o];
        if (tile == num_tiles - 1 && threadIdx.x == 0) *a.out_count = base + total;
        __syncthreads();
    }
    if (threadIdx.x == 0 && join_tally) atomicAdd(a.join_rows, join_tally);
}

template <int THREADS, int CAP, int ROWCAP>
__global__ void __launch_bounds__(THREADS, 1024 / THREADS) fused_join_distinct_kernel(FusedRoundArgs a) {
    fused_round<THREADS, CAP, ROWCAP>(a);
}

}  // namespace spk
