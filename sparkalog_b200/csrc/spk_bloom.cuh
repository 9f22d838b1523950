// A blocked Bloom filter of a recursive relation's FULL, for the anti-join.
//
// SortedBinaryAntiJoin (crates/sparkalog-execution/native/column_ops.cu:
// 167-227, 551-641) keeps the candidates absent from FULL. Searching FULL's
// sorted levels costs every candidate a dependent chain of loads in every
// level, although in a transitive closure almost every distinct candidate
// is new (a path is rarely re-derived). The filter answers "certainly
// absent" for most candidates with one 32-byte sector: a key sets (and
// probes) three bits of one 256-bit block, the block and the bits taken
// from a 64-bit mix of the key. A candidate whose three bits are all set
// may be in FULL; only those are searched in the levels, so the result is
// exactly the reference's. Every row of FULL is in the filter (it is built
// from FULL and takes every row the anti-join adds), so there are no false
// negatives; rows removed from FULL may stay in it (that only adds false
// positives).
#pragma once

#include "spk_common.cuh"
#include "spk_engine_kernels.cuh"

namespace spk {

constexpr int kBloomBlockWords = 8;  // 256 bits: one 32-byte sector

struct Bloom {
    u32* words;      // blocks * kBloomBlockWords
    u64 block_mask;  // blocks - 1 (blocks is a power of two)
};

__device__ __forceinline__ u64 bloom_mix(u64 x) {
    // The splitmix64 finaliser (Steele, Lea, Flood 2014).
    x ^= x >> 30;
    x *= 0xBF58476D1CE4E5B9ull;
    x ^= x >> 27;
    x *= 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// The key's block and its three (word, bit) positions in it.
__device__ __forceinline__ u64 bloom_slot(u64 key, u64 block_mask, u32* word, u32* bit) {
    const u64 h = bloom_mix(key);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const u32 v = static_cast<u32>(h >> (40 + 8 * i)) & 0xffu;
        word[i] = v >> 5;
        bit[i] = v & 31u;
    }
    return h & block_mask;
}

__device__ __forceinline__ bool bloom_maybe(const Bloom& bf, u64 key) {
    u32 w[3], b[3];
    const u64 block = bloom_slot(key, bf.block_mask, w, b);
    const uint4* p = reinterpret_cast<const uint4*>(bf.words + block * kBloomBlockWords);
    const uint4 lo = p[0], hi = p[1];
    const u32 words[8] = {lo.x, lo.y, lo.z, lo.w, hi.x, hi.y, hi.z, hi.w};
    bool all = true;
#pragma unroll
    for (int i = 0; i < 3; ++i) all = all && ((words[w[i]] >> b[i]) & 1u);
    return all;
}

__device__ __forceinline__ void bloom_insert(const Bloom& bf, u64 key) {
    u32 w[3], b[3];
    const u64 block = bloom_slot(key, bf.block_mask, w, b);
    u32* p = bf.words + block * kBloomBlockWords;
#pragma unroll
    for (int i = 0; i < 3; ++i) atomicOr(p + w[i], 1u << b[i]);
}

static __global__ void bloom_insert_kernel(const u64* rows, u64 n, Bloom bf) {
    const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
    for (u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) bloom_insert(bf, rows[i]);
}

// NEWT = unique(sorted candidates) - FULL with the filter in front of the
// level search: each thread takes ITEMS consecutive candidates, keeps the
// first of each run of equal ones (BinaryDistinct), probes the filter, and
// searches the levels (all at once, in lock step, as the sparse anti-join
// does) only for the candidates the filter cannot rule out. The kept rows
// are compacted in order with a decoupled look-back and added to the filter.
template <int THREADS, int ITEMS>
__device__ __forceinline__ void anti_join_bloom(const u64* buf_a, const u64* buf_b, const u32* final_sel,
                                                const u64* n_ptr, const Levels& levels, const Bloom& bf, u64* out,
                                                u64* out_count, u64* status, u32* tile_counter, u32 epoch, u32* err,
                                                unsigned long long* unique_count) {
    constexpr int kTile = THREADS * ITEMS;
    __shared__ CompactShared<THREADS> cs;
    __shared__ u64 stage[kTile];
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
        u32 maybe = 0;
#pragma unroll
        for (int i = 0; i < ITEMS; ++i)
            if ((keep & (1u << i)) && bloom_maybe(bf, v[i])) maybe |= 1u << i;
        if (maybe) {
            u64 pos[kMaxLevels][ITEMS];
            u32 span[kMaxLevels][ITEMS];
            u32 max_span = 0;
#pragma unroll
            for (int l = 0; l < kMaxLevels; ++l) {
#pragma unroll
                for (int i = 0; i < ITEMS; ++i) {
                    pos[l][i] = 0;
                    span[l][i] = 0;
                    if (l < levels.n && (maybe & (1u << i))) {
                        u64 lo, hi;
                        dir_range(levels, l, v[i], &lo, &hi);
                        pos[l][i] = lo;
                        span[l][i] = static_cast<u32>(hi - lo);
                        max_span = span[l][i] > max_span ? span[l][i] : max_span;
                    }
                }
            }
            // Lower bound of v in each bucket: the window shrinks to one row.
            u32 bucket[kMaxLevels][ITEMS];
#pragma unroll
            for (int l = 0; l < kMaxLevels; ++l)
#pragma unroll
                for (int i = 0; i < ITEMS; ++i) bucket[l][i] = span[l][i];
            while (max_span > 1) {
#pragma unroll
                for (int l = 0; l < kMaxLevels; ++l) {
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
            for (int l = 0; l < kMaxLevels; ++l) {
#pragma unroll
                for (int i = 0; i < ITEMS; ++i) {
                    if (bucket[l][i] > 0) {
                        const u64 p = pos[l][i] + (levels.keys[l][pos[l][i]] < v[i] ? 1 : 0);
                        if (p < levels.count[l] && levels.keys[l][p] == v[i]) keep &= ~(1u << i);
                    }
                }
            }
        }
        u32 excl, total;
        const u64 off = compact_offsets<THREADS>(__popc(keep), &excl, &total, tile, status, epoch, err, cs);
        u32 wpos = excl;
#pragma unroll
        for (int i = 0; i < ITEMS; ++i)
            if (keep & (1u << i)) {
                stage[wpos++] = v[i];
                bloom_insert(bf, v[i]);
            }
        __syncthreads();
        for (u32 j = threadIdx.x; j < total; j += THREADS) out[off + j] = stage[j];
        if (tile == num_tiles - 1 && threadIdx.x == 0) *out_count = off + total;
        __syncthreads();
    }
    flush_unique(unique_tally, unique_count);
}

template <int THREADS, int ITEMS>
__global__ void __launch_bounds__(THREADS) anti_join_bloom_kernel(const u64* buf_a, const u64* buf_b,
                                                                  const u32* final_sel, const u64* n_ptr,
                                                                  Levels levels, Bloom bf, u64* out, u64* out_count,
                                                                  u64* status, u32* tile_counter, u32 epoch, u32* err,
                                                                  unsigned long long* unique_count) {
    anti_join_bloom<THREADS, ITEMS>(buf_a, buf_b, final_sel, n_ptr, levels, bf, out, out_count, status, tile_counter,
                                    epoch, err, unique_count);
}

}  // namespace spk
