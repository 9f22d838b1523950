// FULL membership as a device hash set of packed rows.
//
// The reference's SortedBinaryAntiJoin (crates/sparkalog-operators/src/lib.rs,
// anti_join over sorted pairs) answers "is this candidate already in FULL?"
// by searching the sorted FULL. Here a recursive relation can also keep FULL
// in an open-addressing hash set next to its sorted levels: a candidate costs
// one 32-byte sector read (a group of four slots) instead of a dependent
// search per level, and the sorted levels are still maintained for output and
// for every operation that needs order.
//
// Layout: groups of four u64 slots (one 32-byte sector, 32-byte aligned);
// kEmptySlot marks a free slot. Group index = mix(row) & group_mask, then
// linear probing over groups. Slots only ever go from empty to a row, so a
// probe that meets a group with a free slot has seen every place the row
// could be. The row equal to kEmptySlot (both columns 0xffffffff) is kept in
// a separate flag word. The set is read-only while it is queried; rows are
// inserted by a separate launch (compare-and-swap into the first free slot).
// The host keeps the load at most one half (one sixteenth right after a
// build), so a query almost always ends in its first group.
#pragma once

#include "spk_common.cuh"
#include "spk_engine_kernels.cuh"
#include "spk_setops.cuh"

namespace spk {

constexpr u64 kEmptySlot = ~0ull;

struct MemberSet {
    u64* slots;        // 4 * (group_mask + 1) slots
    u64 group_mask;
    u32* has_empty_key;  // 1 when the row kEmptySlot is a member
};

// MurmurHash3's 64-bit finaliser (fmix64), a published bijective mixer.
__device__ __forceinline__ u64 member_mix(u64 k) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ull;
    k ^= k >> 33;
    return k;
}

// 0: absent, 1: present, 2: the group is full (probe further).
__device__ __forceinline__ int member_group_test(ulonglong2 a, ulonglong2 b, u64 key) {
    if (a.x == key || a.y == key || b.x == key || b.y == key) return 1;
    if (a.x == kEmptySlot || a.y == kEmptySlot || b.x == kEmptySlot || b.y == kEmptySlot) return 0;
    return 2;
}

__device__ __forceinline__ bool member_contains_from(const MemberSet& set, u64 key, u64 group, u32* err) {
    for (u64 p = 0; p <= set.group_mask; ++p) {
        const ulonglong2* q = reinterpret_cast<const ulonglong2*>(set.slots + 4 * group);
        const int r = member_group_test(__ldg(q), __ldg(q + 1), key);
        if (r != 2) return r == 1;
        group = (group + 1) & set.group_mask;
    }
    atomicOr(err, kErrMemberProbe);
    return false;
}

// Inserts rows[0, n) (distinct from each other and from the members): one
// read of the row's group, then a compare-and-swap into its first free slot
// (the next free one if another row took it first), group after group.
static __global__ void member_insert_kernel(const u64* rows, u64 n, MemberSet set, u32* err) {
    const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
    for (u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const u64 key = rows[i];
        if (key == kEmptySlot) {
            atomicOr(set.has_empty_key, 1u);
            continue;
        }
        u64 group = member_mix(key) & set.group_mask;
        bool done = false;
        for (u64 p = 0; p <= set.group_mask && !done; ++p) {
            const ulonglong2* q = reinterpret_cast<const ulonglong2*>(set.slots + 4 * group);
            const ulonglong2 a = __ldcg(q), b = __ldcg(q + 1);
            u64 slot[4] = {a.x, a.y, b.x, b.y};
            unsigned long long* g = reinterpret_cast<unsigned long long*>(set.slots + 4 * group);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (done) break;
                if (slot[j] == key) {
                    done = true;
                } else if (slot[j] == kEmptySlot) {
                    const u64 old = atomicCAS(g + j, static_cast<unsigned long long>(kEmptySlot),
                                              static_cast<unsigned long long>(key));
                    done = old == kEmptySlot || old == key;
                }
            }
            group = (group + 1) & set.group_mask;
        }
        if (!done) atomicOr(err, kErrMemberProbe);
    }
}

// NEWT = unique(sorted candidates) - FULL with FULL's membership from the
// hash set: each thread's ITEMS candidates issue their first-group loads
// together, and the rare full group continues on its own. Kept rows are
// compacted in order with a decoupled look-back, so NEWT stays sorted.
template <int THREADS, int ITEMS>
__global__ void __launch_bounds__(THREADS) anti_join_member_kernel(const u64* buf_a, const u64* buf_b,
                                                                   const u32* final_sel, const u64* n_ptr,
                                                                   MemberSet set, u64* out, u64* out_count,
                                                                   u64* status, u32* tile_counter, u32 epoch,
                                                                   u32* err, unsigned long long* unique_count) {
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
    const bool empty_key_member = *set.has_empty_key != 0;
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
        ulonglong2 lo[ITEMS], hi[ITEMS];
        u64 group[ITEMS];
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
            group[i] = 0;
            lo[i] = hi[i] = make_ulonglong2(kEmptySlot, kEmptySlot);
            if ((keep & (1u << i)) && v[i] != kEmptySlot) {
                group[i] = member_mix(v[i]) & set.group_mask;
                const ulonglong2* q = reinterpret_cast<const ulonglong2*>(set.slots + 4 * group[i]);
                lo[i] = __ldg(q);
                hi[i] = __ldg(q + 1);
            }
        }
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
            if (!(keep & (1u << i))) continue;
            bool present;
            if (v[i] == kEmptySlot) {
                present = empty_key_member;
            } else {
                const int r = member_group_test(lo[i], hi[i], v[i]);
                present = r == 2 ? member_contains_from(set, v[i], (group[i] + 1) & set.group_mask, err) : r == 1;
            }
            if (present) keep &= ~(1u << i);
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

}  // namespace spk
