// LSD radix sort of packed 64-bit (first << 32 | second) keys.
//
// Replaces cub::DeviceRadixSort::SortKeys in the reference's distinct
// (crates/sparkalog-execution/native/column_ops.cu:461-469,522-530).
//
// Structure (one launch each, all on one stream, no host synchronisation):
//   1. radix_histogram: one read of the keys builds the 256-bin histogram of
//      every pass at once, with warp-aggregated (match.any) shared-memory
//      atomics, then one global atomic per bin per CTA.
//   2. radix_plan: exclusive scan of each histogram into global bin offsets.
//      A pass whose digit is the same for every key is an identity
//      permutation and is marked inactive, so keys whose high bits are zero
//      (24-bit node ids in a 64-bit key) skip those passes.
//   3. radix_pass (once per active pass): tiles of TILE keys are taken in
//      atomic-counter order; each tile is staged in shared memory with 128-bit
//      loads, ranked stably per digit with match.any warp multi-split, its
//      global offsets come from a per-digit decoupled look-back, the tile is
//      reordered in shared memory and written out so that keys of one digit
//      go to consecutive addresses (coalesced stores, two keys of one digit
//      per 128-bit store where the destination is aligned).
// Buffer ping-pong is decided on the device (RadixPlan::src_sel/final_sel),
// because skipped passes are only known after the histogram.
#pragma once

#include "spk_common.cuh"

namespace spk {

constexpr int kRadixBits = 8;
constexpr int kRadix = 1 << kRadixBits;
constexpr int kMaxPasses = 8;

struct RadixPlan {
    u32 hist[kMaxPasses][kRadix];
    u32 tile_counter[kMaxPasses];
    u32 bin_offset[kMaxPasses][kRadix];
    u32 active[kMaxPasses];
    u32 src_sel[kMaxPasses];  // 0: keys live in buffer A, 1: buffer B
    u32 final_sel;
    u32 n;                    // key count seen by the plan kernel
};
// Bytes of RadixPlan that must be zero before radix_histogram runs.
constexpr size_t kRadixPlanClearBytes = sizeof(u32) * (kMaxPasses * kRadix + kMaxPasses);

// Warp-aggregated histogram update: d == kRadix marks an inactive lane.
// A digit shared by the whole warp (constant high bits, or the sorted high
// bits of a join output) costs one shared atomic; otherwise lanes with equal
// digits are grouped with match.any and each group's leader adds its size.
__device__ __forceinline__ void warp_histogram_add(u32* hist, u32 d) {
    const u32 d0 = __shfl_sync(0xffffffffu, d, 0);
    if (__all_sync(0xffffffffu, d == d0)) {
        if (lane_id() == 0 && d0 < static_cast<u32>(kRadix)) atomicAdd(&hist[d0], static_cast<u32>(kWarp));
        return;
    }
    const u32 peers = __match_any_sync(0xffffffffu, d);
    if (d < static_cast<u32>(kRadix) && (peers & lanemask_lt()) == 0) atomicAdd(&hist[d], __popc(peers));
}

template <int THREADS>
__global__ void __launch_bounds__(THREADS) radix_histogram(const u64* __restrict__ keys, const u64* n_ptr,
                                                           u64 n_host, RadixPlan* plan, int begin_bit,
                                                           int passes) {
    __shared__ u32 sh[kMaxPasses][kRadix];
    for (int i = threadIdx.x; i < kMaxPasses * kRadix; i += THREADS) (&sh[0][0])[i] = 0;
    __syncthreads();
    const u64 n = n_ptr ? *n_ptr : n_host;
    const u64 stride = static_cast<u64>(gridDim.x) * THREADS;
    // Iterate in whole-warp steps so that match.any always sees 32 lanes.
    const u64 first = static_cast<u64>(blockIdx.x) * THREADS + threadIdx.x;
    const u64 rounds = (n + stride - 1) / stride;
    for (u64 r = 0; r < rounds; ++r) {
        const u64 i = first + r * stride;
        const bool valid = i < n;
        const u64 k = valid ? keys[i] : 0;
        for (int p = 0; p < passes; ++p) {
            const u32 d = valid ? static_cast<u32>((k >> (begin_bit + p * kRadixBits)) & (kRadix - 1)) : kRadix;
            warp_histogram_add(sh[p], d);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * kRadix; i += THREADS) {
        const u32 c = (&sh[0][0])[i];
        if (c) atomicAdd(&plan->hist[0][0] + i, c);
    }
}

// One CTA of kRadix threads.
static __global__ void __launch_bounds__(kRadix) radix_plan(RadixPlan* plan, const u64* n_ptr, u64 n_host, int passes) {
    __shared__ u32 scratch[kRadix / kWarp + 1];
    __shared__ u32 any_full;
    const u64 n = n_ptr ? *n_ptr : n_host;
    for (int p = 0; p < passes; ++p) {
        if (threadIdx.x == 0) any_full = 0;
        __syncthreads();
        const u32 c = plan->hist[p][threadIdx.x];
        if (static_cast<u64>(c) == n) any_full = 1;
        u32 total;
        const u32 off = block_exclusive_scan<kRadix>(c, scratch, &total);
        plan->bin_offset[p][threadIdx.x] = off;
        __syncthreads();
        if (threadIdx.x == 0) plan->active[p] = (n > 0 && !any_full) ? 1u : 0u;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        u32 cur = 0;
        for (int p = 0; p < passes; ++p) {
            plan->src_sel[p] = cur;
            if (plan->active[p]) cur ^= 1u;
        }
        for (int p = passes; p < kMaxPasses; ++p) {
            plan->active[p] = 0;
            plan->src_sel[p] = cur;
        }
        plan->final_sel = cur;
        plan->n = static_cast<u32>(n);
    }
}

template <int THREADS, int ITEMS>
struct RadixPassShared {
    static constexpr int kTile = THREADS * ITEMS;
    static constexpr int kWarps = THREADS / kWarp;
    u64 keys[kTile];
    u32 warp_count[kWarps][kRadix];
    u32 tile_start[kRadix];
    u64 global_base[kRadix];
    u32 scan_scratch[kRadix / kWarp + 1];
    u32 tile;
};

template <int THREADS, int ITEMS>
__global__ void __launch_bounds__(THREADS) radix_pass(u64* buf_a, u64* buf_b, const RadixPlan* __restrict__ plan,
                                                      RadixPlan* plan_rw, int pass, int shift, u64* status,
                                                      const u32* epoch_ptr, u32 epoch_add, u32* err) {
    static_assert(THREADS == kRadix, "one digit per thread in the look-back");
    using Shared = RadixPassShared<THREADS, ITEMS>;
    constexpr int kTile = Shared::kTile;
    __shared__ __align__(16) Shared sh;
    if (!plan->active[pass]) return;
    const u64* __restrict__ src = plan->src_sel[pass] ? buf_b : buf_a;
    u64* __restrict__ dst = plan->src_sel[pass] ? buf_a : buf_b;
    const u64 n = plan->n;
    const u64 num_tiles = (n + kTile - 1) / kTile;
    const u32 epoch = (epoch_ptr ? *epoch_ptr : 0u) + epoch_add;
    const u32 lane = lane_id(), warp = warp_id();
    const bool aligned16 = ((reinterpret_cast<uintptr_t>(src) & 15) == 0);

    for (;;) {
        if (threadIdx.x == 0) sh.tile = atomicAdd(&plan_rw->tile_counter[pass], 1u);
        __syncthreads();
        const u64 tile = sh.tile;
        if (tile >= num_tiles) break;
        const u64 tile_base = tile * kTile;
        const u32 valid_count = static_cast<u32>(n - tile_base < static_cast<u64>(kTile) ? n - tile_base : kTile);

        // Stage the tile in shared memory (128-bit loads when aligned and full).
        if (aligned16 && valid_count == kTile) {
            const ulonglong2* s2 = reinterpret_cast<const ulonglong2*>(src + tile_base);
            ulonglong2* d2 = reinterpret_cast<ulonglong2*>(sh.keys);
#pragma unroll
            for (int i = 0; i < ITEMS / 2; ++i) d2[threadIdx.x + i * THREADS] = s2[threadIdx.x + i * THREADS];
        } else {
            for (u32 i = threadIdx.x; i < valid_count; i += THREADS) sh.keys[i] = src[tile_base + i];
        }
        for (int i = threadIdx.x; i < Shared::kWarps * kRadix; i += THREADS) (&sh.warp_count[0][0])[i] = 0;
        __syncthreads();

        // Stable warp multi-split ranking: warp w owns tile positions
        // [w*32*ITEMS, (w+1)*32*ITEMS), visited item-major then lane order.
        u64 key[ITEMS];
        u32 digit[ITEMS];
        u32 rank[ITEMS];
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
            const u32 pos = warp * (kWarp * ITEMS) + i * kWarp + lane;
            const bool valid = pos < valid_count;
            key[i] = valid ? sh.keys[pos] : 0;
            const u32 d = valid ? static_cast<u32>((key[i] >> shift) & (kRadix - 1)) : kRadix;
            digit[i] = d;
            const u32 peers = __match_any_sync(0xffffffffu, d);
            const u32 before = __popc(peers & lanemask_lt());
            u32 base = 0;
            if (valid) base = sh.warp_count[warp][d];
            __syncwarp();
            if (valid && before == 0) sh.warp_count[warp][d] = base + __popc(peers);
            __syncwarp();
            rank[i] = base + before;
        }
        __syncthreads();

        // Per digit (thread t owns digit t): warp prefix, tile count, tile start.
        u32 running = 0;
#pragma unroll
        for (int w = 0; w < Shared::kWarps; ++w) {
            const u32 c = sh.warp_count[w][threadIdx.x];
            sh.warp_count[w][threadIdx.x] = running;
            running += c;
        }
        u32 tile_total;
        const u32 start = block_exclusive_scan<THREADS>(running, sh.scan_scratch, &tile_total);
        sh.tile_start[threadIdx.x] = start;
        const u64 excl = lookback_exclusive(status + threadIdx.x, kRadix, tile, running, epoch, err);
        sh.global_base[threadIdx.x] = static_cast<u64>(plan->bin_offset[pass][threadIdx.x]) + excl;
        __syncthreads();

        // Reorder the tile by digit in shared memory.
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
            if (digit[i] < static_cast<u32>(kRadix)) {
                const u32 pos = sh.tile_start[digit[i]] + sh.warp_count[warp][digit[i]] + rank[i];
                sh.keys[pos] = key[i];
            }
        }
        __syncthreads();

        // Write out: consecutive positions of one digit are consecutive
        // addresses. Each thread takes two neighbouring positions; when both
        // hold the same digit and the first lands on a 16-byte boundary they
        // leave as one 128-bit store (a warp then writes 512 contiguous
        // bytes), otherwise as two 64-bit stores.
        const bool dst16 = (reinterpret_cast<uintptr_t>(dst) & 15) == 0;
        for (u32 j = 2 * threadIdx.x; j < valid_count; j += 2 * THREADS) {
            const u64 k0 = sh.keys[j];
            const u32 d0 = static_cast<u32>((k0 >> shift) & (kRadix - 1));
            const u64 o0 = sh.global_base[d0] + (j - sh.tile_start[d0]);
            if (j + 1 < valid_count) {
                const u64 k1 = sh.keys[j + 1];
                const u32 d1 = static_cast<u32>((k1 >> shift) & (kRadix - 1));
                if (d1 == d0 && dst16 && (o0 & 1) == 0) {
                    *reinterpret_cast<ulonglong2*>(dst + o0) = make_ulonglong2(k0, k1);
                    continue;
                }
                dst[sh.global_base[d1] + (j + 1 - sh.tile_start[d1])] = k1;
            }
            dst[o0] = k0;
        }
        __syncthreads();
    }
}

// Host-side launcher. Sorts `n` keys (n_ptr == nullptr) or a device-resident
// count (*n_ptr, n_host is then an upper bound used only for nothing but
// documentation) over bits [begin_bit, end_bit). After it, the sorted keys
// are in buffer A if plan->final_sel == 0 else in buffer B.
struct RadixSortConfig {
    static constexpr int kThreads = 256;
    static constexpr int kItems = 16;
    static constexpr int kTile = kThreads * kItems;
};

inline size_t radix_status_words(u64 max_keys) {
    return static_cast<size_t>((max_keys + RadixSortConfig::kTile - 1) / RadixSortConfig::kTile + 1) * kRadix;
}

}  // namespace spk
