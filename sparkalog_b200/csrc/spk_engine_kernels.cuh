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

constexpr int kMaxLevels = 3;

struct Levels {
    const u64* keys[kMaxLevels];
    u64 count[kMaxLevels];
    int n;
};

// NEWT = unique(sorted candidates) - FULL, where FULL is the union of the
// levels. Candidates come from the radix sort's final buffer. This fuses the
// reference's BinaryDistinct unique step with SortedBinaryAntiJoin.
template <int THREADS, int ITEMS>
__global__ void __launch_bounds__(THREADS) anti_join_levels_kernel(const u64* buf_a, const u64* buf_b,
                                                                   const u32* final_sel, const u64* n_ptr,
                                                                   Levels levels, u64* out, u64* out_count,
                                                                   u64* status, u32* tile_counter, u32 epoch,
                                                                   u32* err) {
    constexpr int kTile = THREADS * ITEMS;
    __shared__ CompactShared<THREADS> cs;
    __shared__ u64 stage[kTile];
    __shared__ u64 range_lo[kMaxLevels], range_hi[kMaxLevels];
    const u64* keys = (final_sel && *final_sel) ? buf_b : buf_a;
    const u64 n = *n_ptr;
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
        const u64 tile_begin = tile * kTile;
        const u64 tile_end = tile_begin + kTile < n ? tile_begin + kTile : n;
        // Narrow every level to the tile's key span (one warp per level).
        const int w = static_cast<int>(warp_id());
        if (w < levels.n && lane_id() == 0) {
            const PackedKeys lv{levels.keys[w]};
            const u64 c = levels.count[w];
            range_lo[w] = lower_bound_keys(lv, 0, c, keys[tile_begin]);
            const u64 hi = lower_bound_keys(lv, 0, c, keys[tile_end - 1]);
            range_hi[w] = hi < c ? hi + 1 : c;
        }
        __syncthreads();
        const u64 base = tile_begin + static_cast<u64>(threadIdx.x) * ITEMS;
        u64 v[ITEMS];
        u32 keep = 0, count = 0;
        u64 cursor[kMaxLevels];
#pragma unroll
        for (int l = 0; l < kMaxLevels; ++l) cursor[l] = l < levels.n ? range_lo[l] : 0;
        u64 prev = (base > 0 && base - 1 < n) ? keys[base - 1] : 0;
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
            const u64 idx = base + i;
            v[i] = 0;
            if (idx < n) {
                const u64 k = keys[idx];
                v[i] = k;
                bool kept = (idx == 0 || k != prev);
                prev = k;
                if (kept) {
#pragma unroll
                    for (int l = 0; l < kMaxLevels; ++l) {
                        if (l < levels.n) {
                            const PackedKeys lv{levels.keys[l]};
                            cursor[l] = gallop_lower_bound(lv, cursor[l], range_hi[l], k);
                            if (cursor[l] < range_hi[l] && lv(cursor[l]) == k) kept = false;
                        }
                    }
                }
                if (kept) {
                    keep |= 1u << i;
                    ++count;
                }
            }
        }
        u32 excl, total;
        const u64 off = compact_offsets<THREADS>(count, &excl, &total, tile, status, epoch, err, cs);
        u32 wpos = excl;
#pragma unroll
        for (int i = 0; i < ITEMS; ++i)
            if (keep & (1u << i)) stage[wpos++] = v[i];
        __syncthreads();
        for (u32 j = threadIdx.x; j < total; j += THREADS) out[off + j] = stage[j];
        if (tile == num_tiles - 1 && threadIdx.x == 0) *out_count = off + total;
        __syncthreads();
    }
}

// Merge of two sorted, mutually disjoint runs (levels are disjoint by
// construction: NEWT excludes FULL). Output position = merge diagonal, so no
// compaction or look-back is needed: pure streaming at HBM rate.
template <int THREADS, int ITEMS>
__global__ void __launch_bounds__(THREADS) merge_disjoint_kernel(const u64* a, u64 na, const u64* b, u64 nb,
                                                                 u64* out) {
    constexpr int kTile = THREADS * ITEMS;
    __shared__ u64 sm[kTile];
    __shared__ u64 split[2];
    const PackedKeys ka{a}, kb{b};
    const u64 total = na + nb;
    const u64 num_tiles = (total + kTile - 1) / kTile;
    for (u64 tile = blockIdx.x; tile < num_tiles; tile += gridDim.x) {
        const u64 d0 = tile * kTile;
        const u64 d1 = d0 + kTile < total ? d0 + kTile : total;
        if (threadIdx.x == 0) split[0] = merge_path(ka, na, kb, nb, d0);
        if (threadIdx.x == kWarp) split[1] = merge_path(ka, na, kb, nb, d1);
        __syncthreads();
        const u64 i0 = split[0], i1 = split[1];
        const u64 j0 = d0 - i0, j1 = d1 - i1;
        const u32 sa_n = static_cast<u32>(i1 - i0), sb_n = static_cast<u32>(j1 - j0);
        for (u32 t = threadIdx.x; t < sa_n; t += THREADS) sm[t] = a[i0 + t];
        for (u32 t = threadIdx.x; t < sb_n; t += THREADS) sm[sa_n + t] = b[j0 + t];
        __syncthreads();
        const SmemKeys sa{sm}, sb{sm + sa_n};
        const u32 diag = threadIdx.x * ITEMS;
        const u32 len = static_cast<u32>(d1 - d0);
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
        __syncthreads();
#pragma unroll
        for (int i = 0; i < ITEMS; ++i)
            if (diag + i < len) sm[diag + i] = v[i];
        __syncthreads();
        for (u32 j = threadIdx.x; j < len; j += THREADS) out[d0 + j] = sm[j];
        __syncthreads();
    }
}

// Packs SoA columns (c0, c1) into u64 rows and flags whether the rows are
// sorted (non-decreasing) and whether adjacent duplicates exist.
static __global__ void pack_rows_kernel(const u32* c0, const u32* c1, u64 n, u64* out, u32* flags) {
    const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
    bool unsorted = false, dup = false;
    for (u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const u64 k = pack2(c0[i], c1[i]);
        out[i] = k;
        if (i > 0) {
            const u64 p = pack2(c0[i - 1], c1[i - 1]);
            unsorted |= p > k;
            dup |= p == k;
        }
    }
    if (__any_sync(0xffffffffu, unsorted) && lane_id() == 0) atomicOr(flags, 1u);
    if (__any_sync(0xffffffffu, dup) && lane_id() == 0) atomicOr(flags, 2u);
}

static __global__ void unpack_rows_kernel(const u64* in, u64 n, u32* c0, u32* c1) {
    const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
    for (u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const u64 k = in[i];
        c0[i] = static_cast<u32>(k >> 32);
        c1[i] = static_cast<u32>(k);
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

}  // namespace spk
