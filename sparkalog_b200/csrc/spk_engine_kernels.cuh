// Kernels of the device-resident fixpoint engine (packed u64 relations).
//
// FULL of a recursive relation is kept as up to kMaxLevels sorted, mutually
// disjoint runs ("levels": BASE, MID, TAIL). The reference rewrites FULL with
// a merge every round (TargetRuntime::apply, crates/sparkalog-recursion/src/
// generic.rs:360-397); keeping small recent runs apart and merging them into
// larger ones geometrically gives the same set while each round moves only
// the recent rows. The logical FULL is the union of the levels, and it is
// materialised by merging them whenever a single sorted array is needed.
#pragma once

#include "spk_common.cuh"
#include "spk_setops.cuh"

namespace spk {

constexpr int kMaxLevels = 4;

// A level's bucket directory: dir[b] = first row whose key >> shift >= b, for
// b in [0, buckets]; about 64 rows per bucket. It turns a search over a level
// of n rows into two loads of a small (L2-resident) array plus a search over
// one bucket, instead of a log2(n)-long chain of dependent DRAM loads.
struct Levels {
    const u64* keys[kMaxLevels];
    u64 count[kMaxLevels];
    const u32* dir[kMaxLevels];
    u32 shift[kMaxLevels];
    u64 buckets[kMaxLevels];
    int n;
};

// lower_bound of `key` in level l through its directory.
__device__ __forceinline__ void dir_range(const Levels& lv, int l, u64 key, u64* lo, u64* hi) {
    const u64 b = key >> lv.shift[l];
    if (b >= lv.buckets[l]) {
        *lo = *hi = lv.count[l];
        return;
    }
    *lo = lv.dir[l][b];
    *hi = lv.dir[l][b + 1];
}

__device__ __forceinline__ u64 dir_lower_bound(const Levels& lv, int l, u64 key) {
    u64 lo, hi;
    dir_range(lv, l, key, &lo, &hi);
    return lower_bound_keys(PackedKeys{lv.keys[l]}, lo, hi, key);
}

// Builds a level's bucket directory: one independent binary search per
// bucket boundary (all in parallel, so no thread walks a long gap of empty
// buckets). `buckets` must exceed the largest key >> shift.
static __global__ void level_directory_kernel(const u64* keys, u64 n, u32 shift, u64 buckets, u32* dir) {
    const PackedKeys k{keys};
    const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
    for (u64 b = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; b <= buckets; b += stride)
        dir[b] = static_cast<u32>(b == buckets ? n : lower_bound_keys(k, 0, n, b << shift));
}

// NEWT = unique(sorted candidates) - FULL, where FULL is the union of the
// levels. This fuses the reference's BinaryDistinct unique step with
// SortedBinaryAntiJoin (crates/sparkalog-operators/src/lib.rs, the sorted
// anti-join over packed rows).
//
// Per tile of candidates and per level, the slice of the level that can hold
// the tile's keys is read off the level's directory (the bucket of the first
// key to the bucket of the last: two loads, no search). A slice of up to
// STAGE * kStreamChunks rows is streamed through shared memory in chunks of
// STAGE rows (asynchronous copies, double-buffered: the next chunk is in
// flight while the current one is searched), and each thread searches its
// sorted candidates in the chunk that spans them; a larger slice (a sparse
// tile against a big level) is searched per candidate from its directory
// bucket, all ITEMS candidates in lock step. Kept rows are compacted with a
// decoupled look-back, so NEWT stays sorted.
constexpr u64 kStreamChunks = 2;

// The rows kept after the unique step (BinaryDistinct's output size): each
// thread sums its own over all its tiles, and when the kernel ends every
// warp adds its sum to *unique_count (when given) with one atomic. (One
// atomic per warp per tile on the single counter serialised whole launches.)
// Called by every thread.
__device__ __forceinline__ void flush_unique(u32 tally, unsigned long long* unique_count) {
    if (!unique_count) return;
    const u32 c = __reduce_add_sync(0xffffffffu, tally);
    if (lane_id() == 0 && c) atomicAdd(unique_count, static_cast<unsigned long long>(c));
}

// Directory bounds of a tile's keys [first, last] in every level: the rows of
// first's bucket through last's bucket (threads 0 .. 2 * levels.n - 1).
__device__ __forceinline__ void level_slices(const Levels& levels, u64 first, u64 last, u64* range_lo, u64* range_hi) {
    const int l = static_cast<int>(threadIdx.x >> 1);
    if (l < levels.n) {
        u64 lo, hi;
        if ((threadIdx.x & 1) == 0) {
            dir_range(levels, l, first, &lo, &hi);
            range_lo[l] = lo;
        } else {
            dir_range(levels, l, last, &lo, &hi);
            range_hi[l] = hi;
        }
    }
}

template <int THREADS, int ITEMS, int STAGE>
__global__ void __launch_bounds__(THREADS) anti_join_levels_kernel(const u64* buf_a, const u64* buf_b,
                                                                   const u32* final_sel, const u64* n_ptr,
                                                                   Levels levels, u64* out, u64* out_count,
                                                                   u64* status, u32* tile_counter, u32 epoch,
                                                                   u32* err, unsigned long long* unique_count) {
    constexpr int kTile = THREADS * ITEMS;
    static_assert(STAGE >= kTile, "the output stage reuses the level stage");
    __shared__ CompactShared<THREADS> cs;
    __shared__ __align__(16) u64 stage[2 * STAGE];
    __shared__ u64 range_lo[kMaxLevels], range_hi[kMaxLevels];
    const u64* keys = (final_sel && *final_sel) ? buf_b : buf_a;
    const u64 n = *n_ptr;
    const u64 num_tiles = (n + kTile - 1) / kTile;
    if (num_tiles == 0) {
        if (blockIdx.x == 0 && threadIdx.x == 0) *out_count = 0;
        return;
    }
    u32 unique_tally = 0;
    for (;;) {
        if (threadIdx.x == 0) cs.tile = atomicAdd(tile_counter, 1u);
        __syncthreads();
        const u64 tile = cs.tile;
        if (tile >= num_tiles) break;
        const u64 tile_begin = tile * kTile;
        const u64 tile_end = tile_begin + kTile < n ? tile_begin + kTile : n;
        if (threadIdx.x < 2u * levels.n) level_slices(levels, keys[tile_begin], keys[tile_end - 1], range_lo, range_hi);
        const u64 base = tile_begin + static_cast<u64>(threadIdx.x) * ITEMS;
        u64 v[ITEMS];
        u32 keep = 0;
        u64 prev = (base > 0 && base - 1 < n) ? keys[base - 1] : 0;
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
            const u64 idx = base + i;
            v[i] = 0;
            if (idx < n) {
                const u64 k = keys[idx];
                v[i] = k;
                if (idx == 0 || k != prev) keep |= 1u << i;
                prev = k;
            }
        }
        unique_tally += __popc(keep);
        __syncthreads();
        for (int l = 0; l < levels.n; ++l) {
            const u64 lo = range_lo[l];
            const u64 hi = range_hi[l];
            const PackedKeys lv{levels.keys[l]};
            if (hi - lo <= static_cast<u64>(STAGE) * kStreamChunks) {
                const u32 chunks = static_cast<u32>((hi - lo + STAGE - 1) / STAGE);
                const u64* level_keys = levels.keys[l];
                auto issue = [&](u32 c) {
                    const u64 c0 = lo + static_cast<u64>(c) * STAGE;
                    const u32 clen = static_cast<u32>(hi - c0 < static_cast<u64>(STAGE) ? hi - c0 : STAGE);
                    u64* buf = stage + (c & 1) * STAGE;
                    for (u32 t = threadIdx.x; t < clen; t += THREADS) cp_async_8(buf + t, level_keys + c0 + t);
                    cp_async_commit();
                };
                if (chunks) issue(0);
                for (u32 c = 0; c < chunks; ++c) {
                    if (c + 1 < chunks) {
                        issue(c + 1);
                        cp_async_wait<1>();
                    } else {
                        cp_async_wait<0>();
                    }
                    __syncthreads();
                    const u64 c0 = lo + static_cast<u64>(c) * STAGE;
                    const u32 clen = static_cast<u32>(hi - c0 < static_cast<u64>(STAGE) ? hi - c0 : STAGE);
                    const u64* buf = stage + (c & 1) * STAGE;
                    const u64 first = buf[0], last = buf[clen - 1];
                    if (keep && v[0] <= last) {
                        const SmemKeys sk{buf};
                        u64 cur = 0;
#pragma unroll
                        for (int i = 0; i < ITEMS; ++i) {
                            if ((keep & (1u << i)) && v[i] >= first && v[i] <= last) {
                                cur = gallop_lower_bound(sk, cur, clen, v[i]);
                                if (cur < clen && buf[cur] == v[i]) keep &= ~(1u << i);
                            }
                        }
                    }
                    __syncthreads();
                }
            } else if (keep) {
                // Sparse tile against a large slice: each candidate's search
                // starts from its directory bucket (two loads of a small
                // array), then the bucket searches of all ITEMS candidates
                // run branch-free in lock step, so every step issues ITEMS
                // independent loads instead of one dependent chain.
                u64 pos[ITEMS], span[ITEMS], end[ITEMS];
                u64 max_span = 0;
#pragma unroll
                for (int i = 0; i < ITEMS; ++i) {
                    span[i] = 0;
                    pos[i] = end[i] = 0;
                    if (keep & (1u << i)) {
                        dir_range(levels, l, v[i], &pos[i], &end[i]);
                        span[i] = end[i] - pos[i];
                        max_span = span[i] > max_span ? span[i] : max_span;
                    }
                }
                while (max_span > 1) {
#pragma unroll
                    for (int i = 0; i < ITEMS; ++i) {
                        if (span[i] > 1) {
                            const u64 half = span[i] >> 1;
                            pos[i] = lv(pos[i] + half - 1) < v[i] ? pos[i] + half : pos[i];
                            span[i] -= half;
                        }
                    }
                    max_span -= max_span >> 1;
                }
#pragma unroll
                for (int i = 0; i < ITEMS; ++i) {
                    if ((keep & (1u << i)) && end[i] > pos[i]) {
                        const u64 p = pos[i] + (lv(pos[i]) < v[i] ? 1 : 0);
                        if (p < end[i] && lv(p) == v[i]) keep &= ~(1u << i);
                    }
                }
            }
        }
        u32 excl, total;
        const u64 off = compact_offsets<THREADS>(__popc(keep), &excl, &total, tile, status, epoch, err, cs);
        u32 wpos = excl;
#pragma unroll
        for (int i = 0; i < ITEMS; ++i)
            if (keep & (1u << i)) stage[wpos++] = v[i];
        __syncthreads();
        for (u32 j = threadIdx.x; j < total; j += THREADS) out[off + j] = stage[j];
        if (tile == num_tiles - 1 && threadIdx.x == 0) *out_count = off + total;
        __syncthreads();
    }
    flush_unique(unique_tally, unique_count);
}

// The same anti-join for small candidate sets, whose keys lie far apart in
// every level (the tail rounds of a fixpoint): each thread looks its ITEMS
// candidates up in all levels at once, so a tile's dependent chain is one
// bucket search long instead of one per level. LV (>= levels.n) sizes the
// per-level search state: three levels instead of four, or fewer items per
// thread, need fewer registers, so more CTAs share an SM.
template <int THREADS, int ITEMS, int LV = kMaxLevels>
__global__ void __launch_bounds__(THREADS) anti_join_levels_sparse_kernel(const u64* buf_a, const u64* buf_b,
                                                                          const u32* final_sel, const u64* n_ptr,
                                                                          Levels levels, u64* out, u64* out_count,
                                                                          u64* status, u32* tile_counter, u32 epoch,
                                                                          u32* err, unsigned long long* unique_count) {
    constexpr int kTile = THREADS * ITEMS;
    __shared__ DeferredShared<THREADS, kTile> ds;
    const u64* keys = (final_sel && *final_sel) ? buf_b : buf_a;
    const u64 n = *n_ptr;
    const u64 num_tiles = (n + kTile - 1) / kTile;
    if (num_tiles == 0) {
        if (blockIdx.x == 0 && threadIdx.x == 0) *out_count = 0;
        return;
    }
    u32 unique_tally = 0;
    // A tile whose look-back meets an unpublished predecessor waits while the
    // CTA searches its next tile (deferred compaction).
    DeferredState st;
    for (;;) {
        if (threadIdx.x == 0) ds.cs.tile = atomicAdd(tile_counter, 1u);
        __syncthreads();
        const u64 tile = ds.cs.tile;
        if (tile >= num_tiles) break;
        const u64 base = tile * kTile + static_cast<u64>(threadIdx.x) * ITEMS;
        u64 v[ITEMS];
        u32 keep = 0;
        u64 prev = (base > 0 && base - 1 < n) ? keys[base - 1] : 0;
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
            const u64 idx = base + i;
            v[i] = 0;
            if (idx < n) {
                const u64 k = keys[idx];
                v[i] = k;
                if (idx == 0 || k != prev) keep |= 1u << i;
                prev = k;
            }
        }
        unique_tally += __popc(keep);
        u64 pos[LV][ITEMS];
        u32 span[LV][ITEMS], bucket[LV][ITEMS];
        u32 max_span = 0;
#pragma unroll
        for (int l = 0; l < LV; ++l) {
#pragma unroll
            for (int i = 0; i < ITEMS; ++i) {
                pos[l][i] = 0;
                span[l][i] = bucket[l][i] = 0;
                if (l < levels.n && (keep & (1u << i))) {
                    u64 lo, hi;
                    dir_range(levels, l, v[i], &lo, &hi);
                    pos[l][i] = lo;
                    span[l][i] = bucket[l][i] = static_cast<u32>(hi - lo);
                    max_span = span[l][i] > max_span ? span[l][i] : max_span;
                }
            }
        }
        while (max_span > 1) {
#pragma unroll
            for (int l = 0; l < LV; ++l) {
#pragma unroll
                for (int i = 0; i < ITEMS; ++i) {
                    if (span[l][i] > 1) {
                        const u32 half = span[l][i] >> 1;
                        pos[l][i] = levels.keys[l][pos[l][i] + half - 1] < v[i] ? pos[l][i] + half : pos[l][i];
                        span[l][i] -= half;
                    }
                }
            }
            max_span -= max_span >> 1;
        }
#pragma unroll
        for (int l = 0; l < LV; ++l) {
#pragma unroll
            for (int i = 0; i < ITEMS; ++i) {
                if (bucket[l][i] > 0) {
                    // The lower bound is pos or pos + 1; past the bucket's end
                    // the keys belong to later buckets and cannot equal v.
                    const u64 p = pos[l][i] + (levels.keys[l][pos[l][i]] < v[i] ? 1 : 0);
                    if (p < levels.count[l] && levels.keys[l][p] == v[i]) keep &= ~(1u << i);
                }
            }
        }
        u32 total;
        u32 wpos = deferred_scan<THREADS, kTile>(static_cast<u32>(__popc(keep)), &total, tile, status, epoch, ds);
#pragma unroll
        for (int i = 0; i < ITEMS; ++i)
            if (keep & (1u << i)) ds.stage[st.cur][wpos++] = v[i];
        deferred_flush<THREADS, kTile>(st, num_tiles, status, epoch, err, out, out_count, ds);
        deferred_try<THREADS, kTile>(st, tile, total, num_tiles, status, epoch, out, out_count, ds);
    }
    deferred_flush<THREADS, kTile>(st, num_tiles, status, epoch, err, out, out_count, ds);
    flush_unique(unique_tally, unique_count);
}

// The same anti-join for a handful of candidates (the last rounds of a
// fixpoint), where a lookup's latency, not the loads' bandwidth, sets the
// time: G lanes search one candidate together. Each step loads G pivots of
// the candidate's bucket in every level at once and keeps the gap between the
// two pivots that bracket the key, so a bucket of S rows takes
// log_{G+1}(S) steps instead of log_2(S) dependent loads. A tile is
// THREADS / G candidates, one per group.
template <int THREADS, int G>
__device__ __forceinline__ void anti_join_group(const u64* buf_a, const u64* buf_b, const u32* final_sel,
                                                const u64* n_ptr, const Levels& levels, u64* out, u64* out_count,
                                                u64* status, u32* tile_counter, u32 epoch, u32* err,
                                                unsigned long long* unique_count) {
    static_assert(G >= 2 && G <= 32 && 32 % G == 0 && THREADS % 32 == 0, "groups tile the warp");
    constexpr int kTile = THREADS / G;
    // Each step shrinks a window of S > G rows to at most S / (G + 1) + 1;
    // 64 steps cover any u32 row range.
    constexpr int kMaxSteps = 64;
    __shared__ DeferredShared<THREADS, kTile> ds;
    const u64* keys = (final_sel && *final_sel) ? buf_b : buf_a;
    const u64 n = *n_ptr;
    const u64 num_tiles = (n + kTile - 1) / kTile;
    if (num_tiles == 0) {
        if (blockIdx.x == 0 && threadIdx.x == 0) *out_count = 0;
        return;
    }
    const u32 lane = threadIdx.x % G;
    const u32 group_mask = (G == 32 ? 0xffffffffu : ((1u << G) - 1u)) << (lane_id() / G * G);
    u32 unique_tally = 0;
    DeferredState st;
    for (;;) {
        if (threadIdx.x == 0) ds.cs.tile = atomicAdd(tile_counter, 1u);
        __syncthreads();
        const u64 tile = ds.cs.tile;
        if (tile >= num_tiles) break;
        const u64 idx = tile * kTile + threadIdx.x / G;
        u64 v = 0;
        bool keep = false;
        if (idx < n) {
            v = keys[idx];
            keep = idx == 0 || keys[idx - 1] != v;
        }
        unique_tally += (lane == 0 && keep) ? 1u : 0u;
        // [lo, hi): the rows of v's bucket in each level; a row equal to v
        // can only lie there.
        u64 lo[kMaxLevels], hi[kMaxLevels];
#pragma unroll
        for (int l = 0; l < kMaxLevels; ++l) {
            lo[l] = hi[l] = 0;
            if (keep && l < levels.n) dir_range(levels, l, v, &lo[l], &hi[l]);
        }
        bool wide = false;
#pragma unroll
        for (int l = 0; l < kMaxLevels; ++l) wide |= hi[l] - lo[l] > static_cast<u64>(G);
        for (int step = 0; step < kMaxSteps && __any_sync(0xffffffffu, wide); ++step) {
            u64 pivot[kMaxLevels];
            bool below[kMaxLevels];
#pragma unroll
            for (int l = 0; l < kMaxLevels; ++l) {
                const u64 span = hi[l] - lo[l];
                below[l] = false;
                pivot[l] = lo[l] + (span * (lane + 1)) / (G + 1);
                if (span > static_cast<u64>(G)) below[l] = levels.keys[l][pivot[l]] < v;
            }
            wide = false;
#pragma unroll
            for (int l = 0; l < kMaxLevels; ++l) {
                const u64 span = hi[l] - lo[l];
                // Pivots ascend with the lane, so the lanes below v form a prefix.
                const u32 c = __popc(__ballot_sync(0xffffffffu, below[l]) & group_mask);
                if (span > static_cast<u64>(G)) {
                    const u64 p_lo = lo[l] + (span * c) / (G + 1);          // pivot c - 1
                    const u64 p_hi = lo[l] + (span * (c + 1)) / (G + 1);    // pivot c
                    const u64 nlo = c > 0 ? p_lo + 1 : lo[l];
                    const u64 nhi = c < static_cast<u32>(G) ? p_hi + 1 : hi[l];
                    lo[l] = nlo;
                    hi[l] = nhi;
                }
                wide |= hi[l] - lo[l] > static_cast<u64>(G);
            }
        }
        if (wide) atomicOr(err, kErrIndexRange);  // cannot happen: the windows shrink every step
        bool found = false;
#pragma unroll
        for (int l = 0; l < kMaxLevels; ++l)
            if (lane < hi[l] - lo[l] && levels.keys[l][lo[l] + lane] == v) found = true;
        found = (__ballot_sync(0xffffffffu, found) & group_mask) != 0;
        keep = keep && !found;
        u32 total;
        const u32 excl = deferred_scan<THREADS, kTile>(lane == 0 && keep ? 1u : 0u, &total, tile, status, epoch, ds);
        if (lane == 0 && keep) ds.stage[st.cur][excl] = v;
        deferred_flush<THREADS, kTile>(st, num_tiles, status, epoch, err, out, out_count, ds);
        deferred_try<THREADS, kTile>(st, tile, total, num_tiles, status, epoch, out, out_count, ds);
    }
    deferred_flush<THREADS, kTile>(st, num_tiles, status, epoch, err, out, out_count, ds);
    flush_unique(unique_tally, unique_count);
}

template <int THREADS, int G>
__global__ void __launch_bounds__(THREADS) anti_join_levels_wide_kernel(const u64* buf_a, const u64* buf_b,
                                                                        const u32* final_sel, const u64* n_ptr,
                                                                        Levels levels, u64* out, u64* out_count,
                                                                        u64* status, u32* tile_counter, u32 epoch,
                                                                        u32* err, unsigned long long* unique_count) {
    anti_join_group<THREADS, G>(buf_a, buf_b, final_sel, n_ptr, levels, out, out_count, status, tile_counter, epoch,
                                err, unique_count);
}

// Per-segment activity of one round's NEWT rows (sorted, so a segment's rows
// are contiguous): seen[seg] = max(seen[seg], round1), new_rows[seg] += rows.
// Lanes holding the same segment are grouped with match.any and one lane per
// group updates the counters.
__device__ __forceinline__ void segment_activity(const u64* rows, u64 n, u32 shift, u32 count, u32 round1,
                                                 u32* seen, unsigned long long* new_rows) {
    const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
    const u64 rounds = (n + stride - 1) / stride;
    for (u64 r = 0; r < rounds; ++r) {
        const u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x + r * stride;
        u32 seg = 0xffffffffu;
        if (i < n) {
            const u32 s = static_cast<u32>(rows[i] >> 32) >> shift;
            seg = s < count ? s : 0xffffffffu;
        }
        const u32 peers = __match_any_sync(0xffffffffu, seg);
        if (seg != 0xffffffffu && (peers & lanemask_lt()) == 0) {
            atomicMax(&seen[seg], round1);
            atomicAdd(&new_rows[seg], static_cast<unsigned long long>(__popc(peers)));
        }
    }
}

static __global__ void segment_activity_kernel(const u64* rows, u64 n, u32 shift, u32 count, u32 round1,
                                               u32* seen, unsigned long long* new_rows) {
    segment_activity(rows, n, shift, count, round1, seen, new_rows);
}

// Row range of one key interval [lo_key, hi_key) in every level: out[2l] and
// out[2l + 1] are the lower bounds of lo_key and hi_key in level l.
static __global__ void level_bounds_kernel(Levels levels, u64 lo_key, u64 hi_key, u64* out) {
    const int l = static_cast<int>(threadIdx.x);
    if (l >= levels.n) return;
    const PackedKeys k{levels.keys[l]};
    out[2 * l] = lower_bound_keys(k, 0, levels.count[l], lo_key);
    out[2 * l + 1] = lower_bound_keys(k, 0, levels.count[l], hi_key);
}

// Compaction that drops every row whose segment (first column >> shift) is
// set in the `dead` bitmap; order is kept (decoupled look-back offsets).
template <int THREADS, int ITEMS>
__global__ void __launch_bounds__(THREADS) filter_segments_kernel(const u64* in, u64 n, u32 shift, const u32* dead,
                                                                  u64* out, u64* out_count, u64* status,
                                                                  u32* tile_counter, u32 epoch, u32* err) {
    constexpr int kTile = THREADS * ITEMS;
    __shared__ CompactShared<THREADS> cs;
    __shared__ u64 stage[kTile];
    const u64 num_tiles = (n + kTile - 1) / kTile;
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
        u64 v[ITEMS];
        u32 keep = 0;
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
            const u64 idx = base + i;
            v[i] = 0;
            if (idx < n) {
                v[i] = in[idx];
                const u32 seg = static_cast<u32>(v[i] >> 32) >> shift;
                if (!((dead[seg >> 5] >> (seg & 31)) & 1u)) keep |= 1u << i;
            }
        }
        u32 excl, total;
        const u64 off = compact_offsets<THREADS>(__popc(keep), &excl, &total, tile, status, epoch, err, cs);
        u32 w = excl;
#pragma unroll
        for (int i = 0; i < ITEMS; ++i)
            if (keep & (1u << i)) stage[w++] = v[i];
        __syncthreads();
        for (u32 j = threadIdx.x; j < total; j += THREADS) out[off + j] = stage[j];
        if (tile == num_tiles - 1 && threadIdx.x == 0) *out_count = off + total;
        __syncthreads();
    }
}

// Selection and projection of packed rows (an atom with constants or a
// repeated variable, and a clause head with constants): a row is kept when
// every set bit of where_mask holds (bit 0: first == where_value[0], bit 1:
// second == where_value[1], bit 2: first == second), and leaves as the pair
// (out column 0, out column 1), each an input column (source 0 or 1) or a
// constant (source 2). Compacted in order with a decoupled look-back.
struct SelectSpec {
    u32 where_mask;
    u32 where_value[2];
    u32 out_source[2];
    u32 out_value[2];
};

__device__ __forceinline__ u32 select_column(u64 row, u32 source, u32 value) {
    return source == 0 ? static_cast<u32>(row >> 32) : (source == 1 ? static_cast<u32>(row) : value);
}

template <int THREADS, int ITEMS>
__global__ void __launch_bounds__(THREADS) select_rows_kernel(const u64* in, u64 n, SelectSpec sp, u64* out,
                                                              u64* out_count, u64* status, u32* tile_counter,
                                                              u32 epoch, u32* err) {
    constexpr int kTile = THREADS * ITEMS;
    __shared__ CompactShared<THREADS> cs;
    __shared__ u64 stage[kTile];
    const u64 num_tiles = (n + kTile - 1) / kTile;
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
        u64 v[ITEMS];
        u32 keep = 0;
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
            const u64 idx = base + i;
            v[i] = 0;
            if (idx < n) {
                const u64 row = in[idx];
                const u32 c0 = static_cast<u32>(row >> 32), c1 = static_cast<u32>(row);
                const bool ok = (!(sp.where_mask & 1u) || c0 == sp.where_value[0]) &&
                                (!(sp.where_mask & 2u) || c1 == sp.where_value[1]) &&
                                (!(sp.where_mask & 4u) || c0 == c1);
                if (ok) {
                    keep |= 1u << i;
                    v[i] = pack2(select_column(row, sp.out_source[0], sp.out_value[0]),
                                 select_column(row, sp.out_source[1], sp.out_value[1]));
                }
            }
        }
        u32 excl, total;
        const u64 off = compact_offsets<THREADS>(__popc(keep), &excl, &total, tile, status, epoch, err, cs);
        u32 w = excl;
#pragma unroll
        for (int i = 0; i < ITEMS; ++i)
            if (keep & (1u << i)) stage[w++] = v[i];
        __syncthreads();
        for (u32 j = threadIdx.x; j < total; j += THREADS) out[off + j] = stage[j];
        if (tile == num_tiles - 1 && threadIdx.x == 0) *out_count = off + total;
        __syncthreads();
    }
}

// Longest run of equal first-column keys in sorted rows (the index's largest
// match count, which bounds a join's output).
static __global__ void max_run_kernel(const u64* sorted, u64 n, u32* max_degree) {
    const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
    u32 local_max = 0;
    for (u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const u32 key = static_cast<u32>(sorted[i] >> 32);
        if (i == 0 || static_cast<u32>(sorted[i - 1] >> 32) != key) {
            u64 j = i + 1;
            while (j < n && static_cast<u32>(sorted[j] >> 32) == key) ++j;
            const u32 len = static_cast<u32>(j - i);
            local_max = len > local_max ? len : local_max;
        }
    }
    atomicMax(max_degree, local_max);
}

// First-column keys of an index (high words of packed rows or pairs).
static __global__ void high_words_kernel(const u64* in, u64 n, u32* out) {
    const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
    for (u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
        out[i] = static_cast<u32>(in[i] >> 32);
}

// Bucket directory over sorted u32 keys: dir[b] = lower bound of b << shift.
static __global__ void key_directory_kernel(const u32* keys, u64 n, u32 shift, u64 buckets, u32* dir) {
    const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
    for (u64 b = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; b <= buckets; b += stride) {
        if (b == buckets) {
            dir[b] = static_cast<u32>(n);
            continue;
        }
        const u64 key = b << shift;
        u64 lo = 0, hi = n;
        while (lo < hi) {
            const u64 mid = (lo + hi) >> 1;
            if (static_cast<u64>(keys[mid]) < key) lo = mid + 1;
            else hi = mid;
        }
        dir[b] = static_cast<u32>(lo);
    }
}

// Directory of a merge's output, written by the merge itself (see Levels):
// dir[b] = first output row whose key >> shift >= b, for b in [0, buckets].
struct MergeDirectory {
    u32* dir;  // null: no directory
    u32 shift;
    u64 buckets;
};

// Diagonal splits for merge_bulk_kernel: splits[t] = number of `a` rows among
// the first min(t * tile, na + nb) merged rows (ties put a's row first), for
// t in [0, tiles]. One warp per diagonal: each step its 32 lanes test 32
// evenly spaced candidates at once, so a split over n rows costs about
// log32(n) dependent loads instead of log2(n).
__device__ __forceinline__ void merge_splits(const u64* a, u64 na, const u64* b, u64 nb, u32 tile, u64 tiles,
                                             u64* splits) {
    const u32 lane = lane_id();
    const u64 warps = static_cast<u64>(gridDim.x) * (blockDim.x / kWarp);
    const u64 total = na + nb;
    for (u64 t = static_cast<u64>(blockIdx.x) * (blockDim.x / kWarp) + warp_id(); t <= tiles; t += warps) {
        const u64 d = t * tile < total ? t * tile : total;
        // The split is the smallest i in [lo, hi] with a[i] > b[d - 1 - i];
        // "b[d - 1 - i] >= a[i]" holds exactly for the i below it.
        u64 lo = d > nb ? d - nb : 0;
        u64 hi = d < na ? d : na;
        while (hi - lo > kWarp) {
            const u64 step = (hi - lo + kWarp - 1) / kWarp;
            const u64 pos = lo + (static_cast<u64>(lane) + 1) * step - 1;
            const bool below = pos < hi && b[d - 1 - pos] >= a[pos];
            const u32 c = __popc(__ballot_sync(0xffffffffu, below));
            const u64 nlo = lo + c * step;
            const u64 nhi = lo + (static_cast<u64>(c) + 1) * step;
            lo = nlo < hi ? nlo : hi;
            hi = nhi < hi ? nhi : hi;
        }
        const u64 pos = lo + lane;
        const bool below = pos < hi && b[d - 1 - pos] >= a[pos];
        const u64 split = lo + __popc(__ballot_sync(0xffffffffu, below));
        if (lane == 0) splits[t] = split;
    }
}

static __global__ void merge_split_kernel(const u64* a, u64 na, const u64* b, u64 nb, u32 tile, u64 tiles,
                                          u64* splits) {
    merge_splits(a, na, b, nb, tile, tiles, splits);
}

// The same splits with one thread per diagonal and a plain binary search:
// more dependent loads per diagonal than the warp search, but one sector per
// step instead of 32, which wins once there are tens of thousands of
// diagonals (a large merge) and the searches' sector traffic dominates.
static __global__ void merge_split_thread_kernel(const u64* a, u64 na, const u64* b, u64 nb, u32 tile, u64 tiles,
                                                 u64* splits) {
    const u64 total = na + nb;
    const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
    for (u64 t = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; t <= tiles; t += stride) {
        const u64 d = t * tile < total ? t * tile : total;
        u64 lo = d > nb ? d - nb : 0, hi = d < na ? d : na;
        while (lo < hi) {
            const u64 mid = (lo + hi) >> 1;
            if (b[d - 1 - mid] >= a[mid]) lo = mid + 1;
            else hi = mid;
        }
        splits[t] = lo;
    }
}

// Shared-memory layout of merge_bulk_kernel: two input stages (a's slice,
// then b's slice at the next 16-byte boundary, each with up to one leading
// row of alignment slack), the output tile, per-stage slice bounds and the
// stages' barriers.
template <int THREADS, int ITEMS>
struct MergeBulkLayout {
    static constexpr int kTile = THREADS * ITEMS;
    static constexpr int kInRows = kTile + 4;
    static constexpr size_t kIn = static_cast<size_t>(kInRows) * sizeof(u64);
    static constexpr size_t kOut = 2 * kIn;
    static constexpr size_t kMeta = kOut + static_cast<size_t>(kTile) * sizeof(u64);
    static constexpr size_t kBars = kMeta + 2 * 8 * sizeof(u64);
    static constexpr size_t kBytes = kBars + 2 * sizeof(unsigned long long);
};

// Merge of two sorted, mutually disjoint runs (FULL's levels are disjoint by
// construction: NEWT excludes FULL) into `out`, with the output's directory
// written on the way.
//
// Each CTA takes a contiguous chunk of output tiles (THREADS * ITEMS rows
// each). A tile's two input slices, bounded by the diagonal splits, arrive
// in shared memory by two bulk copies that one thread issues, completed on
// the stage's mbarrier; the next tile's copies are in flight while the
// current tile is merged (two stages). Each thread finds its diagonal by a
// merge-path search in shared memory and merges ITEMS rows; ITEMS is odd, so
// the lanes' walks (ITEMS rows apart) fall on different banks without
// padding. The merged tile leaves by one bulk store. Every output row that
// starts a directory bucket (or a run of empty ones) writes the entries up
// to its bucket. Waits are capped: on expiry the kernel sets
// kErrBarrierTimeout, waits once more for its copies, and returns.
template <int THREADS, int ITEMS>
__device__ __forceinline__ void merge_bulk(const u64* a, u64 na, const u64* b, u64 nb, const u64* splits, u64 chunk,
                                           u64* out, const MergeDirectory& md, u32* err) {
    static_assert(ITEMS % 2 == 1, "odd rows per thread keep the merge walks on distinct banks");
    using L = MergeBulkLayout<THREADS, ITEMS>;
    constexpr int kTile = L::kTile;
    extern __shared__ __align__(16) unsigned char smem[];
    auto in_s = [&](int st) { return reinterpret_cast<u64*>(smem + st * L::kIn); };
    u64* out_s = reinterpret_cast<u64*>(smem + L::kOut);
    u64* meta = reinterpret_cast<u64*>(smem + L::kMeta);  // per stage: i0, i1, j0, j1, a_lead, a_rows, b_lead
    unsigned long long* bars = reinterpret_cast<unsigned long long*>(smem + L::kBars);
    __shared__ u64 before_tile;
    __shared__ int failed;

    const u64 total = na + nb;
    const u64 num_tiles = (total + kTile - 1) / kTile;
    // Bulk stores need a 16-byte aligned destination (tiles are an even
    // number of rows); otherwise the tile leaves by plain stores.
    const bool out16 = (reinterpret_cast<uintptr_t>(out) & 15) == 0;
    const u64 t_begin = static_cast<u64>(blockIdx.x) * chunk;
    const u64 t_end = t_begin + chunk < num_tiles ? t_begin + chunk : num_tiles;
    if (t_begin >= t_end) return;
    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_fence_init();
        failed = 0;
    }
    __syncthreads();

    // Thread 0: the bulk copies of tile t into stage `st`.
    auto issue = [&](u64 t, int st) {
        const u64 i0 = splits[t], i1 = splits[t + 1];
        const u64 d0 = t * kTile;
        const u64 d1 = d0 + kTile < total ? d0 + kTile : total;
        const u64 j0 = d0 - i0, j1 = d1 - i1;
        // A slice starts on the 16-byte boundary at or before its first row
        // (one leading row when that row is not aligned; inputs may be
        // slices of a larger array) and ends on the next 16-byte boundary,
        // which stays inside the allocation because allocations are
        // 16-byte multiples.
        const u64 a_lead = (reinterpret_cast<uintptr_t>(a + i0) >> 3) & 1;
        const u64 b_lead = (reinterpret_cast<uintptr_t>(b + j0) >> 3) & 1;
        const u32 a_rows = i1 > i0 ? static_cast<u32>((a_lead + i1 - i0 + 1) & ~1ull) : 0u;
        const u32 b_rows = j1 > j0 ? static_cast<u32>((b_lead + j1 - j0 + 1) & ~1ull) : 0u;
        u64* m = meta + st * 8;
        m[0] = i0; m[1] = i1; m[2] = j0; m[3] = j1; m[4] = a_lead; m[5] = a_rows; m[6] = b_lead;
        mbar_arrive_expect_tx(&bars[st], (a_rows + b_rows) * 8u);
        if (a_rows) bulk_load(in_s(st), a + (i0 - a_lead), a_rows * 8u, &bars[st]);
        if (b_rows) bulk_load(in_s(st) + a_rows, b + (j0 - b_lead), b_rows * 8u, &bars[st]);
    };

    if (threadIdx.x == 0) {
        issue(t_begin, 0);
        // The row before the chunk's first output row (the directory needs
        // its bucket); each later tile takes its predecessor's last row.
        if (md.dir && t_begin > 0) {
            const u64 i0 = splits[t_begin], j0 = t_begin * kTile - i0;
            const u64 pa = i0 > 0 ? a[i0 - 1] : 0, pb = j0 > 0 ? b[j0 - 1] : 0;
            before_tile = i0 == 0 ? pb : (j0 == 0 ? pa : (pa > pb ? pa : pb));
        }
    }
    u32 parity = 0;   // bit st: the phase parity stage st waits for next
    u32 pending = 1;  // bit st: stage st's copies were issued and not yet waited for
    for (u64 t = t_begin, k = 0; t < t_end; ++t, ++k) {
        const int st = static_cast<int>(k & 1);
        if (t + 1 < t_end) {
            if (threadIdx.x == 0) issue(t + 1, st ^ 1);
            pending |= 1u << (st ^ 1);
        }
        if (mbar_wait(&bars[st], (parity >> st) & 1u)) {
            pending &= ~(1u << st);
            parity ^= 1u << st;
        } else {
            atomicOr(err, kErrBarrierTimeout);
            failed = 1;
        }
        const u64 d0 = t * kTile;
        const u64 d1 = d0 + kTile < total ? d0 + kTile : total;
        const u32 len = static_cast<u32>(d1 - d0);
        const u64* m = meta + st * 8;
        const u64 i0 = m[0], j0 = m[2];
        const u32 sa_n = static_cast<u32>(m[1] - i0), sb_n = static_cast<u32>(m[3] - j0);
        const SmemKeys sa{in_s(st) + m[4]}, sb{in_s(st) + m[5] + m[6]};
        const u32 diag = threadIdx.x * ITEMS;
        u64 v[ITEMS];
        if (diag < len) {
            u32 ia = static_cast<u32>(merge_path(sa, sa_n, sb, sb_n, diag));
            u32 ib = diag - ia;
#pragma unroll
            for (int i = 0; i < ITEMS; ++i) {
                if (diag + i < len) {
                    if (ib >= sb_n || (ia < sa_n && sa(ia) <= sb(ib))) v[i] = sa(ia++);
                    else v[i] = sb(ib++);
                }
            }
        }
        // The previous tile's bulk store must have read out_s before it is
        // overwritten.
        if (threadIdx.x == 0) bulk_wait_read();
        __syncthreads();
#pragma unroll
        for (int i = 0; i < ITEMS; ++i)
            if (diag + i < len) out_s[diag + i] = v[i];
        fence_async_shared();
        __syncthreads();
        if (out16) {
            const u32 even = len & ~1u;
            if (threadIdx.x == 0 && even) {
                bulk_store(out + d0, out_s, even * 8u);
                bulk_commit();
            }
            if (threadIdx.x == 1 && (len & 1u)) out[d0 + even] = out_s[even];
        } else {
            for (u32 j = threadIdx.x; j < len; j += THREADS) out[d0 + j] = out_s[j];
        }
        if (md.dir) {
            // The directory entries of the buckets that start in this tile:
            // those after the previous row's bucket up to the last row's.
            // Each is the tile position of the bucket's first key (a binary
            // search in the staged tile), one bucket per thread.
            const u64 b_lo = d0 == 0 ? 0 : (before_tile >> md.shift) + 1;
            const u64 b_hi = out_s[len - 1] >> md.shift;
            const SmemKeys ok{out_s};
            for (u64 b = b_lo + threadIdx.x; b <= b_hi && b <= md.buckets; b += THREADS)
                md.dir[b] = static_cast<u32>(d0 + lower_bound_keys(ok, 0, len, b << md.shift));
            if (d0 + len == total)
                for (u64 b = b_hi + 1 + threadIdx.x; b <= md.buckets; b += THREADS) md.dir[b] = static_cast<u32>(total);
        }
        __syncthreads();
        if (md.dir && threadIdx.x == 0) before_tile = out_s[len - 1];
        if (failed) break;
    }
    if (threadIdx.x == 0) {
        // After a timeout, copies may still be in flight into shared memory:
        // wait once more (capped) for every issued stage before the CTA exits.
        for (int st = 0; st < 2; ++st)
            if ((pending >> st) & 1u) mbar_wait(&bars[st], (parity >> st) & 1u);
        bulk_wait_all();
    }
}

template <int THREADS, int ITEMS>
__global__ void __launch_bounds__(THREADS) merge_bulk_kernel(const u64* a, u64 na, const u64* b, u64 nb,
                                                             const u64* splits, u64 chunk, u64* out,
                                                             MergeDirectory md, u32* err) {
    merge_bulk<THREADS, ITEMS>(a, na, b, nb, splits, chunk, out, md, err);
}

// Packs SoA columns (c0, c1) into u64 rows and flags whether the rows are
// sorted (non-decreasing) and whether adjacent duplicates exist.
static __global__ void pack_rows_kernel(const u32* c0, const u32* c1, u64 n, u64* out, u32* flags) {
    const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
    bool unsorted = false, dup = false;
    u32 max_value = 0;
    for (u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const u64 k = pack2(c0[i], c1[i]);
        out[i] = k;
        max_value = max(max_value, max(c0[i], c1[i]));
        if (i > 0) {
            const u64 p = pack2(c0[i - 1], c1[i - 1]);
            unsorted |= p > k;
            dup |= p == k;
        }
    }
    if (__any_sync(0xffffffffu, unsorted) && lane_id() == 0) atomicOr(flags, 1u);
    if (__any_sync(0xffffffffu, dup) && lane_id() == 0) atomicOr(flags, 2u);
    // flags[1]: the largest value in either column (bounds every key the
    // pipeline can derive, since derived rows only project stored values).
    max_value = __reduce_max_sync(0xffffffffu, max_value);
    if (lane_id() == 0) atomicMax(flags + 1, max_value);
}

// Packed rows back to two columns; mask0/mask1 keep the given bits of each
// column (all ones for a plain read, the low bits to drop a segment tag).
static __global__ void unpack_rows_kernel(const u64* in, u64 n, u32* c0, u32* c1, u32 mask0 = ~0u,
                                          u32 mask1 = ~0u) {
    const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
    for (u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const u64 k = in[i];
        c0[i] = static_cast<u32>(k >> 32) & mask0;
        c1[i] = static_cast<u32>(k) & mask1;
    }
}

// Keys (key << 32 | row) for an index on an unsorted key column.
static __global__ void key_row_pairs_kernel(const u64* rows, u64 n, u32 key_col, u64* out) {
    const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
    for (u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const u64 k = rows[i];
        const u32 key = key_col == 0 ? static_cast<u32>(k >> 32) : static_cast<u32>(k);
        out[i] = pack2(key, static_cast<u32>(i));
    }
}

static __global__ void low_words_kernel(const u64* in, u64 n, u32* out) {
    const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
    for (u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
        out[i] = static_cast<u32>(in[i]);
}

// Dense CSR offsets over key values [0, num_keys]: offsets[k] is the first
// position whose key is >= k (the keys are the high words of `sorted`, which
// is sorted by them). Each segment start fills the gap of absent keys before
// it, so every offset is written exactly once. Also records the maximum
// segment length (the largest out-degree) in *max_degree.
static __global__ void dense_offsets_kernel(const u64* sorted, u64 n, u64 num_keys, u32* offsets, u32* max_degree) {
    const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
    u32 local_max = 0;
    for (u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const u32 key = static_cast<u32>(sorted[i] >> 32);
        const long long prev = i == 0 ? -1 : static_cast<long long>(sorted[i - 1] >> 32);
        if (static_cast<long long>(key) != prev) {
            for (long long k = prev + 1; k <= static_cast<long long>(key); ++k) offsets[k] = static_cast<u32>(i);
            // Segment length: scan forward to the next key change.
            u64 j = i + 1;
            while (j < n && static_cast<u32>(sorted[j] >> 32) == key) ++j;
            const u32 len = static_cast<u32>(j - i);
            local_max = len > local_max ? len : local_max;
        }
        if (i == n - 1) {
            for (u64 k = static_cast<u64>(key) + 1; k <= num_keys; ++k) offsets[k] = static_cast<u32>(n);
        }
    }
    if (n == 0 && blockIdx.x == 0) {
        for (u64 k = threadIdx.x; k <= num_keys; k += blockDim.x) offsets[k] = 0;
    }
    atomicMax(max_degree, local_max);
}

// Compact form of a dense identity index, for joins that gather the right
// relation's second column: per key a 4-bit match count (15 stands for
// fifteen or more; the offsets then give the count), eight keys to a word,
// and one 32-bit word per key that holds the key's single match when it has
// one, else its first offset into `values`. A probe of a key without matches
// reads only its count word (0.5 bytes per key: the count array stays in L2),
// a key with one match one more word, and only keys with two or more matches
// read `values`. Launched with blockDim a multiple of 32: each warp covers 32
// consecutive keys, so groups of eight lanes pack one count word.
static __global__ void compact_index_kernel(const u32* offsets, const u32* values, u64 num_keys, u32* key_class,
                                            u32* key_word) {
    const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
    const u32 lane = lane_id();
    for (u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; i - lane < num_keys; i += stride) {
        u32 nib = 0;
        if (i < num_keys) {
            const u32 lo = offsets[i], hi = offsets[i + 1];
            const u32 deg = hi - lo;
            nib = deg < 15u ? deg : 15u;
            key_word[i] = deg == 1 ? values[lo] : lo;
        }
        u32 v = nib << ((lane & 7) * 4);
        v |= __shfl_xor_sync(0xffffffffu, v, 1);
        v |= __shfl_xor_sync(0xffffffffu, v, 2);
        v |= __shfl_xor_sync(0xffffffffu, v, 4);
        if ((lane & 7) == 0 && i < num_keys) key_class[i >> 3] = v;
    }
}

}  // namespace spk
