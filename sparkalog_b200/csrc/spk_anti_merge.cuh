// Merge-form anti-join for the rounds whose candidates are dense in FULL's
// key space: NEWT = unique(sorted candidates) - FULL, FULL the union of the
// levels, replacing SortedBinaryAntiJoin (crates/sparkalog-execution/native/
// column_ops.cu:167-227, 551-641) with the reference's own merge formulation.
//
// The candidates and FULL's largest level (the partner) are cut into tiles
// of THREADS * ITEMS rows of their merged order (merge-path diagonals, the
// partner's row first on equal keys), so every tile holds a bounded number
// of rows whatever the ratio of candidates to FULL. For the other levels
// (the sides) a tile needs only their rows inside the tile's key range,
// which the plan kernel finds through their directories. A tile's partner
// slice, candidate slice and side slices arrive in shared memory by bulk
// copies on one mbarrier while the previous tile is processed (two stages);
// side slices that do not fit the stage are searched in global memory
// instead. Each thread takes ITEMS consecutive candidates, keeps the first of
// each run of equal ones (BinaryDistinct), and drops those found in a slice:
// a candidate equal to a partner row either finds it in the tile's partner
// slice or, when the row ends the previous tile, in the one partner row
// loaded ahead of the slice. Kept rows are compacted in tile order with a
// decoupled look-back (tiles are claimed in order, so the look-back only
// waits on tiles already claimed), staged in place, and stored coalesced.
#pragma once

#include "spk_common.cuh"
#include "spk_engine_kernels.cuh"
#include "spk_setops.cuh"

namespace spk {

constexpr int kAntiSides = kMaxLevels - 1;

// One tile of the plan: partner rows [i0, i1), candidates [j0, j1), and
// each side level's rows [side_lo, side_hi) with keys in the tile's range.
struct AntiTile {
    u64 i0, i1, j0, j1;
    u64 side_lo[kAntiSides], side_hi[kAntiSides];
};

// Merge-path split: the number of partner rows among the first d rows of the
// merged order (partner first on equal keys): the smallest i with
// L[i] > C[d - 1 - i].
__device__ __forceinline__ u64 anti_split(const u64* L, u64 nL, const u64* C, u64 nC, u64 d) {
    u64 lo = d > nC ? d - nC : 0, hi = d < nL ? d : nL;
    while (lo < hi) {
        const u64 mid = (lo + hi) >> 1;
        if (C[d - 1 - mid] >= L[mid]) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// The side levels of a plan: every level but the partner, in level order.
__device__ __forceinline__ int anti_side_level(int partner, int s) { return s < partner ? s : s + 1; }

// One warp per tile: lanes 0 and 1 find the tile's two diagonals and its
// first and last merged keys, then two lanes per side level bound that
// level's rows in [first, last] through its directory.
template <int TILE>
__global__ void anti_merge_plan_kernel(const u64* buf_a, const u64* buf_b, const u32* final_sel, const u64* n_ptr,
                                       Levels levels, int partner, AntiTile* plan) {
    const u64* C = (final_sel && *final_sel) ? buf_b : buf_a;
    const u64 nC = *n_ptr;
    const u64* L = levels.keys[partner];
    const u64 nL = levels.count[partner];
    const u64 total = nL + nC;
    const u64 tiles = (total + TILE - 1) / TILE;
    const u32 lane = lane_id();
    const u64 warps = static_cast<u64>(gridDim.x) * (blockDim.x / kWarp);
    for (u64 t = static_cast<u64>(blockIdx.x) * (blockDim.x / kWarp) + warp_id(); t < tiles; t += warps) {
        u64 i = 0, j = 0, key = 0;
        if (lane < 2) {
            const u64 d = (t + lane) * TILE < total ? (t + lane) * TILE : total;
            i = anti_split(L, nL, C, nC, d);
            j = d - i;
            if (lane == 0) {
                // First merged row of the tile (the tile is not empty).
                key = (i < nL && (j >= nC || L[i] <= C[j])) ? L[i] : C[j];
            } else {
                // Last merged row of the tile: the larger of the rows before d.
                const u64 a = i > 0 ? L[i - 1] : 0, c = j > 0 ? C[j - 1] : 0;
                key = i == 0 ? c : (j == 0 ? a : (a > c ? a : c));
            }
        }
        const u64 first = __shfl_sync(0xffffffffu, key, 0);
        const u64 last = __shfl_sync(0xffffffffu, key, 1);
        AntiTile& p = plan[t];
        if (lane == 0) {
            p.i0 = i;
            p.j0 = j;
        } else if (lane == 1) {
            p.i1 = i;
            p.j1 = j;
        } else if (lane < 2 + 2 * kAntiSides) {
            const int s = static_cast<int>(lane - 2) >> 1;
            const bool hi_side = ((lane - 2) & 1) != 0;
            const int l = anti_side_level(partner, s);
            u64 v = 0;
            if (l < levels.n && levels.count[l] > 0) {
                if (!hi_side) v = dir_lower_bound(levels, l, first);
                else v = last == ~0ull ? levels.count[l] : dir_lower_bound(levels, l, last + 1);
            }
            if (!hi_side) p.side_lo[s] = v;
            else p.side_hi[s] = v;
        }
    }
}

// Shared memory of anti_merge_kernel: two stages, each holding the partner
// and candidate slices (with one row ahead of each and 16-byte alignment
// slack) and up to SIDE_ROWS rows of side slices; per-stage bookkeeping;
// the stages' barriers.
template <int THREADS, int ITEMS, int SIDE_ROWS>
struct AntiMergeLayout {
    static constexpr int kTile = THREADS * ITEMS;
    static constexpr int kMainRows = kTile + 8;
    static constexpr int kSideRows = SIDE_ROWS + 2 * kAntiSides;
    static constexpr int kStageRows = kMainRows + kSideRows;
    static constexpr size_t kStage = static_cast<size_t>(kStageRows) * sizeof(u64);
    static constexpr int kMetaWords = 16;
    static constexpr size_t kMeta = 2 * kStage;
    static constexpr size_t kBars = kMeta + 2 * kMetaWords * sizeof(u64);
    static constexpr size_t kBytes = kBars + 2 * sizeof(unsigned long long);
    static_assert(kTile % 2 == 0 && kMainRows % 2 == 0, "16-byte aligned regions");
};

// Per-stage bookkeeping words.
enum : int {
    kAmTile = 0,      // tile index
    kAmLOff = 1,      // stage row of partner row i0
    kAmLCount = 2,    // i1 - i0
    kAmCOff = 3,      // stage row of candidate j0
    kAmCCount = 4,    // j1 - j0
    kAmI0 = 5,
    kAmJ0 = 6,
    kAmSideOff = 7,   // + s: stage row of the side slice, or ~0: search it in global memory
    kAmSideCount = 7 + kAntiSides,
    kAmSideLo = 7 + 2 * kAntiSides,  // + s: the slice's first row in its level
};
static_assert(kAmSideLo + kAntiSides <= 16, "bookkeeping fits 16 words");

// Pass 1 over the tiles, statically assigned (tile blockIdx.x + k *
// gridDim.x), with the next tile's copies always in flight: each tile's kept
// candidates go to scratch[j0 ..] (a tile keeps at most its j1 - j0
// candidates) and their number to counts[tile]. No tile waits on another, so
// nothing serialises the tiles; anti_merge_scan_kernel and
// anti_merge_copy_kernel then pack the kept runs in tile order.
template <int THREADS, int ITEMS, int SIDE_ROWS>
__global__ void __launch_bounds__(THREADS) anti_merge_kernel(const u64* buf_a, const u64* buf_b, const u32* final_sel,
                                                             const u64* n_ptr, Levels levels, int partner,
                                                             const AntiTile* plan, u64* scratch, u32* counts,
                                                             u32* err, unsigned long long* unique_count) {
    using Lay = AntiMergeLayout<THREADS, ITEMS, SIDE_ROWS>;
    constexpr int kTile = Lay::kTile;
    extern __shared__ __align__(16) unsigned char smem[];
    auto stage = [&](int st) { return reinterpret_cast<u64*>(smem + st * Lay::kStage); };
    u64* meta = reinterpret_cast<u64*>(smem + Lay::kMeta);
    unsigned long long* bars = reinterpret_cast<unsigned long long*>(smem + Lay::kBars);
    __shared__ u32 scan_scratch[THREADS / kWarp + 1];
    __shared__ int failed;

    const u64* C = (final_sel && *final_sel) ? buf_b : buf_a;
    const u64 nC = *n_ptr;
    const u64* L = levels.keys[partner];
    const u64 nL = levels.count[partner];
    const u64 num_tiles = (nL + nC + kTile - 1) / kTile;
    const u64 first_tile = blockIdx.x;
    if (nC == 0 || first_tile >= num_tiles) return;
    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_fence_init();
        failed = 0;
    }
    __syncthreads();

    // Thread 0: the copies of tile t (plan entry p) into stage st.
    auto issue = [&](u64 t, const AntiTile& p, int st) {
        u64* m = meta + st * Lay::kMetaWords;
        const u64 i0 = p.i0, i1 = p.i1, j0 = p.j0, j1 = p.j1;
        u64* base = stage(st);
        u32 bytes = 0;
        // Partner slice from row i0 - 1 (the row that may equal this tile's
        // first candidate), starting on a 16-byte boundary.
        const u64 ls = i0 > 0 ? i0 - 1 : 0;
        const u64 l_lead = (reinterpret_cast<uintptr_t>(L + ls) >> 3) & 1;
        const u32 l_rows = i1 > ls ? static_cast<u32>((l_lead + i1 - ls + 1) & ~1ull) : 0u;
        // Candidates from row j0 - 1 (the unique step compares with it).
        const u64 cs0 = j0 > 0 ? j0 - 1 : 0;
        const u64 c_lead = (reinterpret_cast<uintptr_t>(C + cs0) >> 3) & 1;
        const u32 c_rows = j1 > cs0 ? static_cast<u32>((c_lead + j1 - cs0 + 1) & ~1ull) : 0u;
        m[kAmTile] = t;
        m[kAmLOff] = l_lead + (i0 - ls);
        m[kAmLCount] = i1 - i0;
        m[kAmCOff] = l_rows + c_lead + (j0 - cs0);
        m[kAmCCount] = j1 - j0;
        m[kAmI0] = i0;
        m[kAmJ0] = j0;
        bytes += (l_rows + c_rows) * 8u;
        u32 side_used = 0;
        u32 side_rows[kAntiSides];
        const u64* side_src[kAntiSides];
#pragma unroll
        for (int s = 0; s < kAntiSides; ++s) {
            const int l = anti_side_level(partner, s);
            const u64 lo = p.side_lo[s], hi = p.side_hi[s];
            const u64 cnt = (l < levels.n && hi > lo) ? hi - lo : 0;
            m[kAmSideLo + s] = lo;
            m[kAmSideCount + s] = cnt;
            side_rows[s] = 0;
            side_src[s] = nullptr;
            m[kAmSideOff + s] = 0;
            if (cnt == 0) continue;
            const u64* src = levels.keys[l] + lo;
            const u64 lead = (reinterpret_cast<uintptr_t>(src) >> 3) & 1;
            const u64 rows = (lead + cnt + 1) & ~1ull;
            if (side_used + rows <= static_cast<u64>(Lay::kSideRows)) {
                m[kAmSideOff + s] = Lay::kMainRows + side_used + lead;
                side_rows[s] = static_cast<u32>(rows);
                side_src[s] = src - lead;
                side_used += static_cast<u32>(rows);
                bytes += static_cast<u32>(rows) * 8u;
            } else {
                m[kAmSideOff + s] = ~0ull;
            }
        }
        mbar_arrive_expect_tx(&bars[st], bytes);
        if (l_rows) bulk_load(base, L + (ls - l_lead), l_rows * 8u, &bars[st]);
        if (c_rows) bulk_load(base + l_rows, C + (cs0 - c_lead), c_rows * 8u, &bars[st]);
        u32 at = Lay::kMainRows;
#pragma unroll
        for (int s = 0; s < kAntiSides; ++s) {
            if (side_rows[s]) {
                bulk_load(base + at, side_src[s], side_rows[s] * 8u, &bars[st]);
                at += side_rows[s];
            }
        }
    };

    // Thread 0 fetches the plan entry of the tile after next into shared
    // memory with asynchronous copies (plan_buf[(k + 1) & 1] holds the next
    // tile's at iteration k), so the issue of the next tile never waits on a
    // plan load and no thread holds a plan entry in registers.
    const u64 stride = gridDim.x;
    __shared__ __align__(16) AntiTile plan_buf[2];
    static_assert(sizeof(AntiTile) % 16 == 0, "plan entries move in 16-byte pieces");
    auto fetch_plan = [&](u64 t, int slot) {
        const char* src = reinterpret_cast<const char*>(plan + t);
        char* dst = reinterpret_cast<char*>(&plan_buf[slot]);
#pragma unroll
        for (int i = 0; i < static_cast<int>(sizeof(AntiTile) / 16); ++i) cp_async_16(dst + 16 * i, src + 16 * i);
        cp_async_commit();
    };
    if (threadIdx.x == 0) {
        issue(first_tile, plan[first_tile], 0);
        if (first_tile + stride < num_tiles) fetch_plan(first_tile + stride, 1);
    }
    u32 parity = 0, pending = 1;
    int k = 0;
    u32 unique_tally = 0;
    for (u64 tile = first_tile; tile < num_tiles; tile += stride, ++k) {
        const int st = k & 1;
        if (threadIdx.x == 0 && tile + stride < num_tiles) {
            cp_async_wait<0>();
            issue(tile + stride, plan_buf[(k + 1) & 1], st ^ 1);
            pending |= 1u << (st ^ 1);
            if (tile + 2 * stride < num_tiles) fetch_plan(tile + 2 * stride, k & 1);
        }
        if (mbar_wait(&bars[st], (parity >> st) & 1u)) {
            parity ^= 1u << st;
            pending &= ~(1u << st);
        } else {
            atomicOr(err, kErrBarrierTimeout);
            failed = 1;
        }
        const u64* m = meta + st * Lay::kMetaWords;
        const u64* S = stage(st);
        const u32 nLs = static_cast<u32>(m[kAmLCount]), nCs = static_cast<u32>(m[kAmCCount]);
        const u64* Ls = S + m[kAmLOff];
        const u64* Cs = S + m[kAmCOff];
        const bool has_l_prev = m[kAmI0] > 0, has_c_prev = m[kAmJ0] > 0;
        const u64 j0 = m[kAmJ0];

        // Each thread walks ITEMS consecutive rows of the tile's merged order
        // (partner rows first on equal keys), from its merge-path split. A
        // candidate is a member of the partner level exactly when the last
        // partner row before it equals it, and a repeat when the last
        // candidate before it does; the rows just ahead of the tile (one of
        // each, loaded with the slices) seed both for the first thread.
        const u32 len = nLs + nCs;
        const u32 diag = threadIdx.x * ITEMS;
        u64 v[ITEMS];
        u32 keep = 0;
        if (diag < len) {
            // Merge-path split of this thread's diagonal (32-bit indices).
            u32 ia, ib;
            {
                u32 lo = diag > nCs ? diag - nCs : 0u, hi = diag < nLs ? diag : nLs;
                while (lo < hi) {
                    const u32 mid = (lo + hi) >> 1;
                    if (Cs[diag - 1 - mid] >= Ls[mid]) lo = mid + 1;
                    else hi = mid;
                }
                ia = lo;
                ib = diag - lo;
            }
            bool l_ok = ia > 0 || has_l_prev, c_ok = ib > 0 || has_c_prev;
            u64 last_l = l_ok ? Ls[static_cast<int>(ia) - 1] : 0;
            u64 last_c = c_ok ? Cs[static_cast<int>(ib) - 1] : 0;
            // The two heads stay in registers; only the side that advanced
            // is read again.
            u64 lh = ia < nLs ? Ls[ia] : 0, ch = ib < nCs ? Cs[ib] : 0;
#pragma unroll
            for (int i = 0; i < ITEMS; ++i) {
                v[i] = 0;
                if (diag + i < len) {
                    if (ib >= nCs || (ia < nLs && lh <= ch)) {
                        last_l = lh;
                        l_ok = true;
                        ++ia;
                        lh = ia < nLs ? Ls[ia] : 0;
                    } else {
                        const u64 c = ch;
                        ++ib;
                        ch = ib < nCs ? Cs[ib] : 0;
                        if (!(c_ok && c == last_c)) {
                            ++unique_tally;
                            if (!(l_ok && c == last_l)) {
                                keep |= 1u << i;
                                v[i] = c;
                            }
                        }
                        last_c = c;
                        c_ok = true;
                    }
                }
            }
        }
#pragma unroll
        for (int s = 0; s < kAntiSides; ++s) {
            const u64 cnt = m[kAmSideCount + s];
            if (!keep || cnt == 0) continue;
            const u64 off = m[kAmSideOff + s];
            // One search for the first kept candidate, galloping after it.
            if (off != ~0ull) {
                const u64* ss = S + off;
                const SmemKeys sk{ss};
                u64 cur = 0;
                bool started = false;
#pragma unroll
                for (int i = 0; i < ITEMS; ++i) {
                    if (keep & (1u << i)) {
                        cur = started ? gallop_lower_bound(sk, cur, cnt, v[i]) : lower_bound_keys(sk, 0, cnt, v[i]);
                        started = true;
                        if (cur < cnt && ss[cur] == v[i]) keep &= ~(1u << i);
                    }
                }
            } else {
                const u64 lo = m[kAmSideLo + s];
                const PackedKeys gk{levels.keys[anti_side_level(partner, s)]};
                u64 cur = lo;
                bool started = false;
#pragma unroll
                for (int i = 0; i < ITEMS; ++i) {
                    if (keep & (1u << i)) {
                        cur = started ? gallop_lower_bound(gk, cur, lo + cnt, v[i])
                                      : lower_bound_keys(gk, lo, lo + cnt, v[i]);
                        started = true;
                        if (cur < lo + cnt && gk(cur) == v[i]) keep &= ~(1u << i);
                    }
                }
            }
        }
        u32 total;
        const u32 excl = block_exclusive_scan<THREADS>(static_cast<u32>(__popc(keep)), scan_scratch, &total);
        // The block scan synchronised: every read of the stage is done.
        // Stage the kept rows in place, then store them coalesced.
        u64* outs = const_cast<u64*>(Cs);
        u32 wpos = excl;
#pragma unroll
        for (int i = 0; i < ITEMS; ++i)
            if (keep & (1u << i)) outs[wpos++] = v[i];
        __syncthreads();
        for (u32 j = threadIdx.x; j < total; j += THREADS) scratch[j0 + j] = outs[j];
        if (threadIdx.x == 0) counts[tile] = total;
        // The stage's generic accesses come before the bulk copies that refill it.
        fence_async_shared();
        __syncthreads();
        if (failed) break;
    }
    flush_unique(unique_tally, unique_count);
    if (threadIdx.x == 0) {
        // After a timeout, copies may still be in flight into shared memory.
        for (int st = 0; st < 2; ++st)
            if ((pending >> st) & 1u) mbar_wait(&bars[st], (parity >> st) & 1u);
    }
}

// Pass 2: the tiles' kept counts turned into NEWT offsets in place (an
// exclusive scan; counts[num_tiles] receives the total, which is also NEWT's
// size). One CTA: a fixpoint round has at most about a hundred thousand
// tiles, and each thread sums a contiguous run of them.
template <int THREADS, int TILE>
__global__ void __launch_bounds__(THREADS) anti_merge_scan_kernel(const u64* n_ptr, Levels levels, int partner,
                                                                  u32* counts, u64* out_count) {
    __shared__ u32 scratch[THREADS / kWarp + 1];
    const u64 nC = *n_ptr;
    const u64 num_tiles = nC == 0 ? 0 : (levels.count[partner] + nC + TILE - 1) / TILE;
    // Chunks of THREADS * 16 counts: each thread loads its 16 consecutive
    // counts at once (independent loads), the block scans the per-thread
    // sums, and a running carry joins the chunks.
    constexpr u64 kPer = 16;
    u32 carry = 0;
    for (u64 base = 0; base < num_tiles; base += THREADS * kPer) {
        const u64 b = base + threadIdx.x * kPer;
        u32 c[kPer];
        u32 sum = 0;
#pragma unroll
        for (u64 i = 0; i < kPer; ++i) {
            c[i] = b + i < num_tiles ? counts[b + i] : 0u;
            sum += c[i];
        }
        u32 total;
        u32 run = carry + block_exclusive_scan<THREADS>(sum, scratch, &total);
#pragma unroll
        for (u64 i = 0; i < kPer; ++i) {
            if (b + i < num_tiles) counts[b + i] = run;
            run += c[i];
        }
        carry += total;
        __syncthreads();  // the scan's scratch is reused by the next chunk
    }
    if (threadIdx.x == 0) {
        counts[num_tiles] = carry;
        *out_count = carry;
    }
}

// Pass 3: each tile's kept run copied to its NEWT offset (a warp per tile).
static __global__ void anti_merge_copy_kernel(const u64* n_ptr, Levels levels, int partner, u32 tile_rows,
                                              const AntiTile* plan, const u64* scratch, const u32* offsets,
                                              u64* out) {
    const u64 nC = *n_ptr;
    const u64 num_tiles = nC == 0 ? 0 : (levels.count[partner] + nC + tile_rows - 1) / tile_rows;
    const u64 warps = static_cast<u64>(gridDim.x) * (blockDim.x / kWarp);
    for (u64 t = static_cast<u64>(blockIdx.x) * (blockDim.x / kWarp) + warp_id(); t < num_tiles; t += warps) {
        const u32 o = offsets[t], n = offsets[t + 1] - o;
        const u64* src = scratch + plan[t].j0;
        u64* dst = out + o;
        // Four independent loads in flight per lane before their stores.
        for (u32 j = lane_id(); j < n; j += 4 * kWarp) {
            u64 v[4];
#pragma unroll
            for (int i = 0; i < 4; ++i)
                if (j + i * kWarp < n) v[i] = src[j + i * kWarp];
#pragma unroll
            for (int i = 0; i < 4; ++i)
                if (j + i * kWarp < n) dst[j + i * kWarp] = v[i];
        }
    }
}

}  // namespace spk
