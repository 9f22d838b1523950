// Single-key equality join DELTA |x| right with a binary projected output.
//
// Reference operator replaced: BinaryEqualityJoin on the GPU,
// column_ops.cu:74-135 (count_join_u32, finish_join_count, emit_join_u32) and
// the CUB exclusive scan between them (:348-354,388-394).
//
// Output order is the reference's: left-row-major, and the matches of one
// left row in index order (the right rows sorted by (key, row)).
//
// Emission is load balanced inside a tile: a tile's rows are scanned in the
// block, then the tile's outputs are dealt out round-robin to the threads,
// each finding its row by a binary search over the tile's row offsets in
// shared memory, so a hub key with many matches does not serialise one thread
// and every warp store covers consecutive output rows.
#pragma once

#include "spk_common.cuh"
#include "spk_setops.cuh"

namespace spk {

// Binary search in the unique keys of a U32RangeIndex (column_ops.cu:53-72).
__device__ __forceinline__ long long find_index_key(const u32* keys, u64 unique_keys, u32 key) {
    u64 lo = 0, hi = unique_keys;
    while (lo < hi) {
        const u64 mid = (lo + hi) >> 1;
        if (keys[mid] < key) lo = mid + 1;
        else hi = mid;
    }
    return (lo < unique_keys && keys[lo] == key) ? static_cast<long long>(lo) : -1;
}

template <int THREADS, int ITEMS>
struct JoinTileShared {
    static constexpr int kTile = THREADS * ITEMS;
    u32 row_offset[kTile + 1];  // tile-local exclusive output offsets of each row
    u32 match_begin[kTile];     // first index position of each row's matches
    u32 scan_scratch[THREADS / kWarp + 1];
    u64 tile_offset;
    u64 tile;
};

// ---------------------------------------------------------------------------
// Reference-layout count + scan: counts[r], offsets[r] (exclusive) and total.
// ---------------------------------------------------------------------------
template <int THREADS, int ITEMS>
__global__ void __launch_bounds__(THREADS) join_count_scan_kernel(const u32* left_keys, u64 left_rows,
                                                                  const u32* index_keys, const u32* index_starts,
                                                                  u64 unique_keys, u64* counts, u64* offsets,
                                                                  u64* total, u64* status, u32* tile_counter,
                                                                  u32 epoch, u32* err) {
    constexpr int kTile = THREADS * ITEMS;
    __shared__ u32 scan_scratch[THREADS / kWarp + 1];
    __shared__ u64 scan64[THREADS / kWarp + 1];
    __shared__ u64 tile_off;
    __shared__ u64 tile_id;
    const u64 num_tiles = (left_rows + kTile - 1) / kTile;
    (void)scan_scratch;
    for (;;) {
        if (threadIdx.x == 0) tile_id = atomicAdd(tile_counter, 1u);
        __syncthreads();
        const u64 tile = tile_id;
        if (tile >= num_tiles) break;
        const u64 base = tile * kTile + static_cast<u64>(threadIdx.x) * ITEMS;
        u64 c[ITEMS];
        u64 sum = 0;
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
            const u64 r = base + i;
            c[i] = 0;
            if (r < left_rows) {
                const long long idx = find_index_key(index_keys, unique_keys, left_keys[r]);
                c[i] = idx < 0 ? 0 : static_cast<u64>(index_starts[idx + 1] - index_starts[idx]);
                counts[r] = c[i];
            }
            sum += c[i];
        }
        u64 tile_total;
        const u64 excl = block_exclusive_scan<THREADS, u64>(sum, scan64, &tile_total);
        if (warp_id() == 0) {
            const u64 g = warp_lookback_exclusive(status, tile, tile_total, epoch, err);
            if (lane_id() == 0) tile_off = g;
        }
        __syncthreads();
        u64 run = tile_off + excl;
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
            const u64 r = base + i;
            if (r < left_rows) offsets[r] = run;
            run += c[i];
        }
        if (tile == num_tiles - 1 && threadIdx.x == 0) *total = tile_off + tile_total;
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Reference-layout emit (sparkalog_join_u32_emit): the tile's output base is
// offsets[first row of the tile]; rows are re-searched as in the reference.
// ---------------------------------------------------------------------------
template <int THREADS, int ITEMS>
__global__ void __launch_bounds__(THREADS) join_emit_kernel(const u32* left_keys, u64 left_rows,
                                                            const u32* index_keys, const u32* index_starts,
                                                            const u32* index_rows, u64 unique_keys,
                                                            const u32* projection0, u32 side0,
                                                            const u32* projection1, u32 side1, const u64* offsets,
                                                            u32* output0, u32* output1) {
    using Shared = JoinTileShared<THREADS, ITEMS>;
    constexpr int kTile = Shared::kTile;
    __shared__ Shared sh;
    const u64 num_tiles = (left_rows + kTile - 1) / kTile;
    for (u64 tile = blockIdx.x; tile < num_tiles; tile += gridDim.x) {
        const u64 tile_begin = tile * kTile;
        const u32 local0 = threadIdx.x * ITEMS;
        u32 cnt[ITEMS];
        u32 sum = 0;
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
            const u64 r = tile_begin + local0 + i;
            cnt[i] = 0;
            u32 begin = 0;
            if (r < left_rows) {
                const long long idx = find_index_key(index_keys, unique_keys, left_keys[r]);
                if (idx >= 0) {
                    begin = index_starts[idx];
                    cnt[i] = index_starts[idx + 1] - begin;
                }
            }
            sh.match_begin[local0 + i] = begin;
            sum += cnt[i];
        }
        u32 tile_total;
        u32 run = block_exclusive_scan<THREADS>(sum, sh.scan_scratch, &tile_total);
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
            sh.row_offset[local0 + i] = run;
            run += cnt[i];
        }
        if (threadIdx.x == 0) {
            sh.row_offset[kTile] = tile_total;
            sh.tile_offset = offsets[tile_begin];
        }
        __syncthreads();
        const u64 out_base = sh.tile_offset;
        for (u32 o = threadIdx.x; o < tile_total; o += THREADS) {
            // Row owning output o: last row whose offset is <= o.
            u32 lo = 0, hi = kTile;
            while (hi - lo > 1) {
                const u32 mid = (lo + hi) >> 1;
                if (sh.row_offset[mid] <= o) lo = mid;
                else hi = mid;
            }
            const u64 left_row = tile_begin + lo;
            const u32 m = sh.match_begin[lo] + (o - sh.row_offset[lo]);
            const u32 right_row = index_rows[m];
            output0[out_base + o] = side0 == 0 ? projection0[left_row] : projection0[right_row];
            output1[out_base + o] = side1 == 0 ? projection1[left_row] : projection1[right_row];
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Fused join for the device-resident fixpoint: DELTA and the right relation
// are packed (first << 32 | second) u64 rows, the output is packed too.
// Count, scan (decoupled look-back) and emit happen in one pass; the left row
// count and the output base come from device memory, so the launch needs no
// host synchronisation. Rows that would land beyond `capacity` are not
// written; the true total is still published so the host can grow the buffer.
// ---------------------------------------------------------------------------
struct FusedJoinArgs {
    const u64* delta;
    const u64* delta_count;
    u32 left_key;             // 0: first column of DELTA, 1: second
    const u32* dense_offsets; // dense CSR over key values [0, dense_keys], or null
    u64 dense_keys;
    const u32* keys;          // sparse U32RangeIndex (keys/starts), or the bucketed index's sorted keys
    const u32* starts;
    u64 unique_keys;
    const u32* bucket_dir;    // bucketed index: dir[b] = first position whose key >> bucket_shift >= b
    u32 bucket_shift;
    u64 buckets;
    const u32* rows;          // index rows; null means identity (index built on a sorted column)
    const u64* right;         // packed right relation rows
    u32 side[2];              // 0: left, 1: right
    u32 col[2];
    u64* out;
    u64 capacity;
    const u64* count_in;      // output rows already present (earlier rules of the same target)
    u64* count_out;
    u64* status;
    u32* tile_counter;
    const u32* epoch_ptr;
    u32 epoch_add;
    u32* err;
};

__device__ __forceinline__ u32 pair_col(u64 key, u32 col) {
    return col == 0 ? static_cast<u32>(key >> 32) : static_cast<u32>(key);
}

template <int THREADS, int ITEMS>
__global__ void __launch_bounds__(THREADS) join_fused_kernel(FusedJoinArgs a) {
    using Shared = JoinTileShared<THREADS, ITEMS>;
    constexpr int kTile = Shared::kTile;
    __shared__ Shared sh;
    __shared__ u64 left_key_stage[kTile];
    const u64 n = *a.delta_count;
    const u64 base_in = *a.count_in;
    const u64 num_tiles = (n + kTile - 1) / kTile;
    const u32 epoch = (a.epoch_ptr ? *a.epoch_ptr : 0u) + a.epoch_add;
    if (num_tiles == 0) {
        if (blockIdx.x == 0 && threadIdx.x == 0) *a.count_out = base_in < a.capacity ? base_in : a.capacity;
        return;
    }
    for (;;) {
        if (threadIdx.x == 0) sh.tile = atomicAdd(a.tile_counter, 1u);
        __syncthreads();
        const u64 tile = sh.tile;
        if (tile >= num_tiles) break;
        const u64 tile_begin = tile * kTile;
        const u32 local0 = threadIdx.x * ITEMS;
        u32 cnt[ITEMS];
        u32 sum = 0;
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
            const u64 r = tile_begin + local0 + i;
            cnt[i] = 0;
            u32 begin = 0;
            u64 lk = 0;
            if (r < n) {
                lk = a.delta[r];
                const u32 key = pair_col(lk, a.left_key);
                if (a.dense_offsets) {
                    if (key < a.dense_keys) {
                        begin = a.dense_offsets[key];
                        cnt[i] = a.dense_offsets[key + 1] - begin;
                    }
                } else if (a.bucket_dir) {
                    // Sparse key domain: the key's bucket bounds a short search
                    // for the first and one-past-last position of the key.
                    const u64 b = static_cast<u64>(key) >> a.bucket_shift;
                    if (b < a.buckets) {
                        u64 lo = a.bucket_dir[b], hi = a.bucket_dir[b + 1];
                        while (lo < hi) {
                            const u64 mid = (lo + hi) >> 1;
                            if (a.keys[mid] < key) lo = mid + 1;
                            else hi = mid;
                        }
                        u64 up = lo, top = a.bucket_dir[b + 1];
                        while (up < top) {
                            const u64 mid = (up + top) >> 1;
                            if (a.keys[mid] <= key) up = mid + 1;
                            else top = mid;
                        }
                        begin = static_cast<u32>(lo);
                        cnt[i] = static_cast<u32>(up - lo);
                    }
                } else {
                    const long long idx = find_index_key(a.keys, a.unique_keys, key);
                    if (idx >= 0) {
                        begin = a.starts[idx];
                        cnt[i] = a.starts[idx + 1] - begin;
                    }
                }
            }
            left_key_stage[local0 + i] = lk;
            sh.match_begin[local0 + i] = begin;
            sum += cnt[i];
        }
        u32 tile_total;
        u32 run = block_exclusive_scan<THREADS>(sum, sh.scan_scratch, &tile_total);
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
            sh.row_offset[local0 + i] = run;
            run += cnt[i];
        }
        if (threadIdx.x == 0) sh.row_offset[kTile] = tile_total;
        if (warp_id() == 0) {
            const u64 g = warp_lookback_exclusive(a.status, tile, tile_total, epoch, a.err);
            if (lane_id() == 0) sh.tile_offset = g;
        }
        __syncthreads();
        const u64 out_base = base_in + sh.tile_offset;
        for (u32 o = threadIdx.x; o < tile_total; o += THREADS) {
            u32 lo = 0, hi = kTile;
            while (hi - lo > 1) {
                const u32 mid = (lo + hi) >> 1;
                if (sh.row_offset[mid] <= o) lo = mid;
                else hi = mid;
            }
            const u32 m = sh.match_begin[lo] + (o - sh.row_offset[lo]);
            const u32 right_row = a.rows ? a.rows[m] : m;
            const u64 lk = left_key_stage[lo];
            u64 rk = 0;
            if (a.side[0] == 1 || a.side[1] == 1) rk = a.right[right_row];
            const u32 v0 = a.side[0] == 0 ? pair_col(lk, a.col[0]) : pair_col(rk, a.col[0]);
            const u32 v1 = a.side[1] == 0 ? pair_col(lk, a.col[1]) : pair_col(rk, a.col[1]);
            const u64 pos = out_base + o;
            if (pos < a.capacity) a.out[pos] = pack2(v0, v1);
        }
        if (tile == num_tiles - 1 && threadIdx.x == 0) {
            // The published count is clamped to the buffer so that later
            // kernels never read past it; the capacity bit tells the host to
            // grow the buffer and redo the round.
            const u64 total = out_base + tile_total;
            *a.count_out = total < a.capacity ? total : a.capacity;
            if (total > a.capacity) atomicOr(a.err, kErrCapacity);
        }
        __syncthreads();
    }
}

}  // namespace spk
