// Sorted-set kernels over lexicographic (first, second) u32 pairs:
// unique compaction, anti-join (left - right), union (merge + dedup) and the
// disjoint merge used by the device-resident fixpoint.
//
// Reference operators replaced:
//   distinct's unique + unpack  column_ops.cu:474-481,149-165
//   anti-join mark/select/gather column_ops.cu:167-227,551-641
//   union merge/unique/unpack    column_ops.cu:643-775
//
// Every output-compacting kernel takes tiles in atomic-counter order, scans
// its keep flags in the block, gets its global offset from a warp-parallel
// decoupled look-back, stages the kept rows in shared memory and writes them
// with coalesced stores. The last tile publishes the output count.
#pragma once

#include "spk_common.cuh"

namespace spk {

__device__ __forceinline__ u64 pack2(u32 a, u32 b) { return (static_cast<u64>(a) << 32) | b; }

// Number of elements of `a` in the first `diag` merged elements of (a, b),
// when ties put a's element first: the smallest i with a[i] > b[diag-1-i].
template <class A, class B>
__device__ __forceinline__ u64 merge_path(const A& a, u64 na, const B& b, u64 nb, u64 diag) {
    u64 lo = diag > nb ? diag - nb : 0;
    u64 hi = diag < na ? diag : na;
    while (lo < hi) {
        const u64 mid = (lo + hi) >> 1;
        if (b(diag - 1 - mid) >= a(mid)) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

struct SoaKeys {
    const u32* first;
    const u32* second;
    __device__ __forceinline__ u64 operator()(u64 i) const { return pack2(first[i], second[i]); }
};
struct PackedKeys {
    const u64* keys;
    __device__ __forceinline__ u64 operator()(u64 i) const { return keys[i]; }
};
struct SmemKeys {
    const u64* keys;
    __device__ __forceinline__ u64 operator()(u64 i) const { return keys[i]; }
};

// lower_bound over [lo, hi) of a sorted accessor.
template <class A>
__device__ __forceinline__ u64 lower_bound_keys(const A& a, u64 lo, u64 hi, u64 key) {
    while (lo < hi) {
        const u64 mid = (lo + hi) >> 1;
        if (a(mid) < key) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Galloping lower_bound starting at `from` (known: a(from - 1) < key or from == lo).
template <class A>
__device__ __forceinline__ u64 gallop_lower_bound(const A& a, u64 from, u64 hi, u64 key) {
    u64 step = 1, lo = from, probe = from;
    while (probe < hi && a(probe) < key) {
        lo = probe + 1;
        probe = from + step;
        step <<= 1;
    }
    return lower_bound_keys(a, lo, probe < hi ? probe : hi, key);
}

// Warp-cooperative lower_bound over [lo, hi): each step the 32 lanes probe 32
// evenly spaced positions and the ballot of "probe < key" (a prefix, since
// the input is sorted) cuts the range 32-fold, so a search over n keys costs
// about log32(n) dependent loads instead of log2(n). All 32 lanes must call
// it with the same arguments; all get the result.
template <class A>
__device__ __forceinline__ u64 warp_lower_bound(const A& a, u64 lo, u64 hi, u64 key) {
    const u32 lane = lane_id();
    while (hi - lo > kWarp) {
        const u64 step = (hi - lo + kWarp - 1) / kWarp;
        const u64 pos = lo + (static_cast<u64>(lane) + 1) * step - 1;
        const bool less = pos < hi && a(pos) < key;
        const u32 c = __popc(__ballot_sync(0xffffffffu, less));
        const u64 nlo = lo + c * step;
        const u64 nhi = lo + (static_cast<u64>(c) + 1) * step;
        lo = nlo < hi ? nlo : hi;
        hi = nhi < hi ? nhi : hi;
    }
    const u64 pos = lo + lane;
    const bool less = pos < hi && a(pos) < key;
    return lo + __popc(__ballot_sync(0xffffffffu, less));
}

template <int THREADS>
struct CompactShared {
    u32 scan_scratch[THREADS / kWarp + 1];
    u64 tile_offset;
    u64 tile;
};

// Block scan of per-thread keep counts plus look-back. All threads return
// the tile's global output offset; *thread_excl gets the thread's prefix and
// *tile_total the tile's kept count.
template <int THREADS>
__device__ __forceinline__ u64 compact_offsets(u32 thread_count, u32* thread_excl, u32* tile_total, u64 tile,
                                               u64* status, u32 epoch, u32* err, CompactShared<THREADS>& cs) {
    u32 total;
    const u32 excl = block_exclusive_scan<THREADS>(thread_count, cs.scan_scratch, &total);
    if (warp_id() == 0) {
        const u64 g = warp_lookback_exclusive(status, tile, total, epoch, err);
        if (lane_id() == 0) cs.tile_offset = g;
    }
    __syncthreads();
    *thread_excl = excl;
    *tile_total = total;
    return cs.tile_offset;
}

// Ordered compaction whose tiles do not wait on slow predecessors. A tile
// publishes its kept count, stages its kept rows, and tries its look-back
// without waiting; if a predecessor has not published yet, the tile stays in
// the other stage buffer, with its walk's state, while the CTA works on its
// next tile, and is finished and written after that tile's rows are staged.
// A CTA publishes its current tile's count before it waits on its waiting
// tile, so every wait ends: a claimed tile's count never depends on a wait.
template <int THREADS, int TILE>
struct DeferredShared {
    CompactShared<THREADS> cs;
    u64 stage[2][TILE];
    long long walk_base;
    u64 walk_excl;
    int walk_done;
};

struct DeferredState {
    bool pending = false;
    u64 tile = 0;
    u32 total = 0;
    long long base = 0;
    u64 excl = 0;
    int cur = 0;
};

// Block scan of the per-thread keep counts; publishes the tile's count and
// returns the thread's offset within the tile (rows go to stage[st.cur]).
template <int THREADS, int TILE>
__device__ __forceinline__ u32 deferred_scan(u32 thread_count, u32* tile_total, u64 tile, u64* status, u32 epoch,
                                             DeferredShared<THREADS, TILE>& ds) {
    const u32 excl = block_exclusive_scan<THREADS>(thread_count, ds.cs.scan_scratch, tile_total);
    if (threadIdx.x == 0) lookback_publish(status, tile, *tile_total, epoch);
    return excl;
}

// Finishes and writes the waiting tile, if any. All threads.
template <int THREADS, int TILE>
__device__ __forceinline__ void deferred_flush(DeferredState& st, u64 num_tiles, u64* status, u32 epoch, u32* err,
                                               u64* out, u64* out_count, DeferredShared<THREADS, TILE>& ds) {
    if (!st.pending) return;
    if (warp_id() == 0) {
        warp_lookback_finish(status, st.tile, st.total, epoch, &st.base, &st.excl, err);
        if (lane_id() == 0) ds.cs.tile_offset = st.excl;
    }
    __syncthreads();
    const u64 off = ds.cs.tile_offset;
    const u64* rows = ds.stage[st.cur ^ 1];
    for (u32 j = threadIdx.x; j < st.total; j += THREADS) out[off + j] = rows[j];
    if (st.tile == num_tiles - 1 && threadIdx.x == 0) *out_count = off + st.total;
    st.pending = false;
}

// Tries the current tile's look-back once: writes it now, or leaves it
// waiting. Call after deferred_flush; ends with a barrier. All threads.
template <int THREADS, int TILE>
__device__ __forceinline__ void deferred_try(DeferredState& st, u64 tile, u32 total, u64 num_tiles, u64* status,
                                             u32 epoch, u64* out, u64* out_count,
                                             DeferredShared<THREADS, TILE>& ds) {
    if (warp_id() == 0) {
        long long base = static_cast<long long>(tile) - 1;
        u64 excl = 0;
        const bool done = warp_lookback_try(status, tile, total, epoch, &base, &excl);
        if (lane_id() == 0) {
            ds.walk_done = done ? 1 : 0;
            ds.walk_base = base;
            ds.walk_excl = excl;
        }
    }
    __syncthreads();
    if (ds.walk_done) {
        const u64 off = ds.walk_excl;
        const u64* rows = ds.stage[st.cur];
        for (u32 j = threadIdx.x; j < total; j += THREADS) out[off + j] = rows[j];
        if (tile == num_tiles - 1 && threadIdx.x == 0) *out_count = off + total;
    } else {
        st.pending = true;
        st.tile = tile;
        st.total = total;
        st.base = ds.walk_base;
        st.excl = ds.walk_excl;
        st.cur ^= 1;
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// Unique + unpack of sorted packed keys (the end of distinct).
// ---------------------------------------------------------------------------
template <int THREADS, int ITEMS>
__global__ void __launch_bounds__(THREADS) unique_unpack_kernel(const u64* buf_a, const u64* buf_b,
                                                                const u32* final_sel, u64 n, u32* out_first,
                                                                u32* out_second, u64* out_count, u64* status,
                                                                u32* tile_counter, u32 epoch, u32* err) {
    constexpr int kTile = THREADS * ITEMS;
    __shared__ CompactShared<THREADS> cs;
    __shared__ u64 stage[kTile];
    const u64* keys = (final_sel && *final_sel) ? buf_b : buf_a;
    const u64 num_tiles = (n + kTile - 1) / kTile;
    for (;;) {
        if (threadIdx.x == 0) cs.tile = atomicAdd(tile_counter, 1u);
        __syncthreads();
        const u64 tile = cs.tile;
        if (tile >= num_tiles) break;
        const u64 base = tile * kTile + static_cast<u64>(threadIdx.x) * ITEMS;
        u64 v[ITEMS];
        u32 keep = 0, count = 0;
        u64 prev = (base > 0 && base - 1 < n) ? keys[base - 1] : 0;
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
            const u64 idx = base + i;
            const bool valid = idx < n;
            v[i] = valid ? keys[idx] : 0;
            const bool k = valid && (idx == 0 || v[i] != prev);
            prev = v[i];
            keep |= (k ? 1u : 0u) << i;
            count += k;
        }
        u32 excl, total;
        const u64 off = compact_offsets<THREADS>(count, &excl, &total, tile, status, epoch, err, cs);
        u32 w = excl;
#pragma unroll
        for (int i = 0; i < ITEMS; ++i)
            if (keep & (1u << i)) stage[w++] = v[i];
        __syncthreads();
        for (u32 j = threadIdx.x; j < total; j += THREADS) {
            const u64 k = stage[j];
            out_first[off + j] = static_cast<u32>(k >> 32);
            out_second[off + j] = static_cast<u32>(k);
        }
        if (tile == num_tiles - 1 && threadIdx.x == 0) *out_count = off + total;
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Anti-join over SoA columns: stable left - right (the reference's
// SortedBinaryAntiJoin), with the reference's side outputs: flags[row] is 1
// for kept rows, selected[] lists kept row ids, *selected_rows their count.
// ---------------------------------------------------------------------------
template <int THREADS, int ITEMS>
__global__ void __launch_bounds__(THREADS) anti_join_soa_kernel(const u32* lf, const u32* ls, u64 ln, const u32* rf,
                                                                const u32* rs, u64 rn, u32* flags, u32* selected,
                                                                u32* selected_rows, u32* out_first, u32* out_second,
                                                                u64* status, u32* tile_counter, u32 epoch, u32* err) {
    constexpr int kTile = THREADS * ITEMS;
    __shared__ CompactShared<THREADS> cs;
    __shared__ u32 stage_row[kTile];
    __shared__ u64 range[2];
    const SoaKeys right{rf, rs};
    const u64 num_tiles = (ln + kTile - 1) / kTile;
    for (;;) {
        if (threadIdx.x == 0) cs.tile = atomicAdd(tile_counter, 1u);
        __syncthreads();
        const u64 tile = cs.tile;
        if (tile >= num_tiles) break;
        const u64 tile_begin = tile * kTile;
        const u64 tile_end = tile_begin + kTile < ln ? tile_begin + kTile : ln;
        // Narrow the right range once per tile: [lb(first), lb(last)+1 bound).
        if (warp_id() == 0) {
            const u64 lo = warp_lower_bound(right, 0, rn, pack2(lf[tile_begin], ls[tile_begin]));
            if (lane_id() == 0) range[0] = lo;
        } else if (warp_id() == 1) {
            const u64 hi = warp_lower_bound(right, 0, rn, pack2(lf[tile_end - 1], ls[tile_end - 1]));
            if (lane_id() == 0) range[1] = hi < rn ? hi + 1 : rn;
        }
        __syncthreads();
        // lower_bound is monotone in the key, so any key between the tile's
        // first and last keys has its lower bound inside [r_lo, r_hi); keys
        // outside that span (an unsorted left input, which the reference's
        // per-row binary search also accepts) search the whole right input.
        const u64 r_lo = range[0], r_hi = range[1] > range[0] ? range[1] : range[0];
        const u64 t_first = pack2(lf[tile_begin], ls[tile_begin]);
        const u64 t_last = pack2(lf[tile_end - 1], ls[tile_end - 1]);
        const u64 base = tile_begin + static_cast<u64>(threadIdx.x) * ITEMS;
        u32 keep = 0, count = 0;
        u64 cursor = r_lo, prev_key = 0;
        bool have_cursor = false;
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
            const u64 idx = base + i;
            if (idx < ln) {
                const u64 key = pack2(lf[idx], ls[idx]);
                u64 hi_bound = rn;
                if (key >= t_first && key <= t_last) {
                    hi_bound = r_hi;
                    cursor = (have_cursor && key >= prev_key) ? gallop_lower_bound(right, cursor, r_hi, key)
                                                              : lower_bound_keys(right, r_lo, r_hi, key);
                    have_cursor = true;
                } else {
                    cursor = lower_bound_keys(right, 0, rn, key);
                    have_cursor = false;
                }
                prev_key = key;
                const bool matched = cursor < hi_bound && right(cursor) == key;
                flags[idx] = matched ? 0u : 1u;
                if (!matched) {
                    keep |= 1u << i;
                    ++count;
                }
            }
        }
        (void)cursor;
        u32 excl, total;
        const u64 off = compact_offsets<THREADS>(count, &excl, &total, tile, status, epoch, err, cs);
        u32 w = excl;
#pragma unroll
        for (int i = 0; i < ITEMS; ++i)
            if (keep & (1u << i)) stage_row[w++] = static_cast<u32>(base + i);
        __syncthreads();
        for (u32 j = threadIdx.x; j < total; j += THREADS) {
            const u32 row = stage_row[j];
            selected[off + j] = row;
            out_first[off + j] = lf[row];
            out_second[off + j] = ls[row];
        }
        if (tile == num_tiles - 1 && threadIdx.x == 0) *selected_rows = static_cast<u32>(off + total);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Union over SoA columns: merge-path partitioned merge of two sorted inputs
// with duplicate removal, unpacked into two output columns.
// ---------------------------------------------------------------------------
template <int THREADS, int ITEMS>
__global__ void __launch_bounds__(THREADS) union_soa_kernel(const u32* lf, const u32* ls, u64 ln, const u32* rf,
                                                            const u32* rs, u64 rn, u32* out_first, u32* out_second,
                                                            u64* out_count, u64* status, u32* tile_counter, u32 epoch,
                                                            u32* err) {
    constexpr int kTile = THREADS * ITEMS;
    __shared__ CompactShared<THREADS> cs;
    __shared__ u64 sm[kTile + 2];
    __shared__ u64 split[2];
    __shared__ u64 tile_prev;
    __shared__ int has_prev;
    const SoaKeys a{lf, ls}, b{rf, rs};
    const u64 total_in = ln + rn;
    const u64 num_tiles = (total_in + kTile - 1) / kTile;
    for (;;) {
        if (threadIdx.x == 0) cs.tile = atomicAdd(tile_counter, 1u);
        __syncthreads();
        const u64 tile = cs.tile;
        if (tile >= num_tiles) break;
        const u64 d0 = tile * kTile;
        const u64 d1 = d0 + kTile < total_in ? d0 + kTile : total_in;
        if (threadIdx.x == 0) {
            const u64 i0 = merge_path(a, ln, b, rn, d0);
            split[0] = i0;
            const u64 j0 = d0 - i0;
            u64 p = 0;
            int hp = 0;
            if (i0 > 0) { p = a(i0 - 1); hp = 1; }
            if (j0 > 0) { const u64 q = b(j0 - 1); p = hp ? (q > p ? q : p) : q; hp = 1; }
            tile_prev = p;
            has_prev = hp;
        }
        if (threadIdx.x == kWarp) split[1] = merge_path(a, ln, b, rn, d1);
        __syncthreads();
        const u64 i0 = split[0], i1 = split[1];
        const u64 j0 = d0 - i0, j1 = d1 - i1;
        const u32 na = static_cast<u32>(i1 - i0), nb = static_cast<u32>(j1 - j0);
        for (u32 t = threadIdx.x; t < na; t += THREADS) sm[t] = a(i0 + t);
        for (u32 t = threadIdx.x; t < nb; t += THREADS) sm[na + t] = b(j0 + t);
        __syncthreads();
        const SmemKeys sa{sm}, sb{sm + na};
        const u32 diag = threadIdx.x * ITEMS;
        const u32 len = d1 - d0 > diag ? static_cast<u32>(d1 - d0 - diag) : 0u;
        u64 v[ITEMS];
        u32 keep = 0, count = 0;
        if (len > 0) {
            u32 ia = static_cast<u32>(merge_path(sa, na, sb, nb, diag));
            u32 ib = diag - ia;
            u64 prev;
            bool hp;
            if (diag == 0) {
                prev = tile_prev;
                hp = has_prev != 0;
            } else {
                const u64 pa = ia > 0 ? sa(ia - 1) : 0, pb = ib > 0 ? sb(ib - 1) : 0;
                prev = ia == 0 ? pb : (ib == 0 ? pa : (pa > pb ? pa : pb));
                hp = true;
            }
#pragma unroll
            for (int i = 0; i < ITEMS; ++i) {
                if (static_cast<u32>(i) < len) {
                    u64 x;
                    if (ib >= nb || (ia < na && sa(ia) <= sb(ib))) x = sa(ia++);
                    else x = sb(ib++);
                    v[i] = x;
                    const bool k = !hp || x != prev;
                    prev = x;
                    hp = true;
                    if (k) {
                        keep |= 1u << i;
                        ++count;
                    }
                } else {
                    v[i] = 0;
                }
            }
        }
        __syncthreads();  // sm is reused as the output stage
        u32 excl, total;
        const u64 off = compact_offsets<THREADS>(count, &excl, &total, tile, status, epoch, err, cs);
        u32 w = excl;
#pragma unroll
        for (int i = 0; i < ITEMS; ++i)
            if (keep & (1u << i)) sm[w++] = v[i];
        __syncthreads();
        for (u32 j = threadIdx.x; j < total; j += THREADS) {
            const u64 k = sm[j];
            out_first[off + j] = static_cast<u32>(k >> 32);
            out_second[off + j] = static_cast<u32>(k);
        }
        if (tile == num_tiles - 1 && threadIdx.x == 0) *out_count = off + total;
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Filter (the reference's sparkalog_filter_u32, column_ops.cu:20-43 and
// 283-318): row ids i, ascending, with compare(input[i], op, operand), and
// flags[i] = 1 / 0. Operation codes are the ABI's: 0 ==, 1 !=, 2 <, 3 <=,
// 4 >, 5 >=; any other code matches nothing. Kept ids are compacted in order
// with a decoupled look-back; the count is u32 like the reference's.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool filter_matches(u32 value, u32 op, u32 operand) {
    switch (op) {
        case 0: return value == operand;
        case 1: return value != operand;
        case 2: return value < operand;
        case 3: return value <= operand;
        case 4: return value > operand;
        case 5: return value >= operand;
        default: return false;
    }
}

template <int THREADS, int ITEMS>
__global__ void __launch_bounds__(THREADS) filter_select_kernel(const u32* input, u64 n, u32 op, u32 operand,
                                                                u32* flags, u32* output, u32* count, u64* status,
                                                                u32* tile_counter, u32 epoch, u32* err) {
    constexpr int kTile = THREADS * ITEMS;
    __shared__ CompactShared<THREADS> cs;
    __shared__ u32 stage[kTile];
    const u64 num_tiles = (n + kTile - 1) / kTile;
    for (;;) {
        if (threadIdx.x == 0) cs.tile = atomicAdd(tile_counter, 1u);
        __syncthreads();
        const u64 tile = cs.tile;
        if (tile >= num_tiles) break;
        const u64 base = tile * kTile + static_cast<u64>(threadIdx.x) * ITEMS;
        u32 keep = 0;
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
            const u64 idx = base + i;
            if (idx < n) {
                const bool m = filter_matches(input[idx], op, operand);
                flags[idx] = m ? 1u : 0u;
                keep |= m ? (1u << i) : 0u;
            }
        }
        u32 excl, total;
        const u64 off = compact_offsets<THREADS>(__popc(keep), &excl, &total, tile, status, epoch, err, cs);
        u32 w = excl;
#pragma unroll
        for (int i = 0; i < ITEMS; ++i)
            if (keep & (1u << i)) stage[w++] = static_cast<u32>(base + i);
        __syncthreads();
        for (u32 j = threadIdx.x; j < total; j += THREADS) output[off + j] = stage[j];
        if (tile == num_tiles - 1 && threadIdx.x == 0) *count = static_cast<u32>(off + total);
        __syncthreads();
    }
}

// output[i] = i % modulus (the reference's sparkalog_fill_mod_u32).
static __global__ void fill_mod_kernel(u32* output, u64 n, u32 modulus) {
    const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
    for (u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
        output[i] = static_cast<u32>(i % modulus);
}

// data[i] += 1 (the reference's sparkalog_add_one_i32, its workspace smoke test).
static __global__ void add_one_kernel(int* data, u64 n) {
    const u64 stride = static_cast<u64>(gridDim.x) * blockDim.x;
    for (u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) data[i] += 1;
}

}  // namespace spk
