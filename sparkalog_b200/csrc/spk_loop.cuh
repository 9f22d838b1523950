// Device-driven rounds of the semi-naive loop (RecursiveExecutor::run,
// crates/sparkalog-recursion/src/generic.rs:472-525) for the transitive-
// closure shape, run as the body of a CUDA graph WHILE node.
//
// The host-driven loop ends every round with a device-to-host copy of the
// round's counts and a stream synchronisation, then picks the next round's
// kernels and buffers from those counts. In the long tail of a fixpoint
// (rounds of a few thousand to a hundred thousand rows) that round trip and
// the launch latency around it cost about as much as the kernels. Here one
// round is a fixed sequence of kernels whose pointers and sizes live in a
// device descriptor (LoopDesc), so the same graph body serves every round:
// clear the round's counters, fused join + order, group-searched anti-join,
// diagonal splits, bulk merge of NEWT into TAIL, and the round-end kernel. The round-end kernel applies the round on the device
// (TargetRuntime::apply, generic.rs:360-397: FULL's TAIL <- TAIL u NEWT,
// DELTA <- NEWT), counts it, tests convergence, and sets the WHILE node's
// condition. It stops the loop, leaving everything to the host, when:
//   * NEWT is empty (the fixpoint: every DELTA is empty);
//   * the next round's candidate bound exceeds what the loop's buffers and
//     launch shapes were sized for;
//   * TAIL has outgrown 1/ratio of the level above it (a cascade is due);
//   * the iteration limit is reached;
//   * a kernel reported an error or a fused tile did not fit (then the round
//     is not applied, and the host redoes it with the general kernels).
#pragma once

#include "spk_bloom.cuh"
#include "spk_common.cuh"
#include "spk_engine_kernels.cuh"
#include "spk_fused.cuh"

namespace spk {

enum : u32 {
    kLoopRunning = 0,
    kLoopConverged = 1,   // NEWT was empty
    kLoopBound = 2,       // the next round's candidate bound is too large for the loop
    kLoopCascade = 3,     // TAIL must merge into the level above it
    kLoopLimit = 4,       // the iteration limit was reached
    kLoopRedo = 5,        // a fused tile overflowed or a buffer filled: round not applied
    kLoopFault = 6,       // a kernel set an error bit: round not applied
    kLoopRowLimit = 7,    // FULL would exceed 2^32 - 1 rows: round not applied
};

struct LoopTrace {
    u64 delta_rows, join_rows, unique_rows, new_rows, full_rows;
};

struct LoopDesc {
    FusedRoundArgs fused;  // delta, delta_rows_ptr (-> delta_n), out = candidates, out_count = counts + 1
    Levels lv;             // FULL's levels; entry tail_slot is TAIL
    u32 tail_slot;
    // One round's counts: [0] join rows, [1] candidates, [2] NEWT rows, [3] unique rows.
    u64* counts;
    u32* counters;         // tile counters: [0] fused, [1] anti-join
    u64* anti_status;      // look-back words of the anti-join (cleared every round)
    u32* err;              // error bits; err[8] is the fused kernel's fallback flag
    u64* delta;            // DELTA (== fused.delta)
    u64* newt;             // NEWT, the anti-join's output
    u64 delta_n;
    u64* tail;             // TAIL (== lv.keys[tail_slot])
    u64* spare;            // the merge's destination
    u64 tail_n;
    u64* splits;
    MergeDirectory md;     // TAIL's directory, written by every merge (a fixed shape)
    u64 bound;             // largest candidate bound a round of the loop may have
    u64 max_degree;        // the right index's largest match count (candidate bound = DELTA * it)
    u64 upper_n;           // rows of the level above TAIL (cascade test)
    u64 ratio;
    u64 other_rows;        // FULL rows outside TAIL
    u64 iterations;        // rounds applied by this launch
    u64 limit;             // rounds this launch may apply
    u64 total_new;
    u64 rounds_total;      // the executor's rounds before this launch
    u32 stop;
    u32 seg_shift, seg_count;
    u32* seg_seen;
    unsigned long long* seg_new;
    LoopTrace* trace;      // one record per applied round (capacity >= limit)
    Bloom bloom;           // FULL's Bloom filter (the Bloom variant of the anti-join)
};

template <int THREADS, int CAP, int ROWCAP>
__global__ void __launch_bounds__(THREADS, 1024 / THREADS) loop_fused_kernel(const LoopDesc* d) {
    const FusedRoundArgs a = d->fused;
    fused_round<THREADS, CAP, ROWCAP>(a);
}

template <int THREADS, int G>
__global__ void __launch_bounds__(THREADS) loop_anti_join_kernel(const LoopDesc* d) {
    const u64* cand = d->fused.out;
    anti_join_group<THREADS, G>(cand, cand, nullptr, d->counts + 1, d->lv, d->newt, d->counts + 2, d->anti_status,
                                d->counters + 1, 1u, d->err, reinterpret_cast<unsigned long long*>(d->counts + 3));
}

template <int THREADS, int ITEMS>
__global__ void __launch_bounds__(THREADS) loop_anti_join_bloom_kernel(const LoopDesc* d) {
    const u64* cand = d->fused.out;
    anti_join_bloom<THREADS, ITEMS>(cand, cand, nullptr, d->counts + 1, d->lv, d->bloom, d->newt, d->counts + 2,
                                    d->anti_status, d->counters + 1, 1u, d->err,
                                    reinterpret_cast<unsigned long long*>(d->counts + 3));
}

static __global__ void loop_split_kernel(const LoopDesc* d, u32 tile) {
    const u64 total = d->tail_n + d->counts[2];
    merge_splits(d->tail, d->tail_n, d->newt, d->counts[2], tile, (total + tile - 1) / tile, d->splits);
}

template <int THREADS, int ITEMS>
__global__ void __launch_bounds__(THREADS) loop_merge_kernel(const LoopDesc* d) {
    constexpr u64 kTile = static_cast<u64>(THREADS) * ITEMS;
    const u64 na = d->tail_n, nb = d->counts[2];
    const u64 tiles = (na + nb + kTile - 1) / kTile;
    const u64 chunk = (tiles + gridDim.x - 1) / gridDim.x;
    if (tiles == 0) return;
    merge_bulk<THREADS, ITEMS>(d->tail, na, d->newt, nb, d->splits, chunk, d->spare, d->md, d->err);
}

// One thread: applies the round (or refuses it) and sets the WHILE condition.
static __global__ void loop_round_end_kernel(LoopDesc* d, cudaGraphConditionalHandle handle) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const u64 joined = d->counts[0], unique = d->counts[3], newt = d->counts[2];
    const u32 bits = d->err[0];
    const bool fallback = d->err[8] != 0;
    u32 stop = kLoopRunning;
    if (fallback || (bits & kErrCapacity)) {
        stop = kLoopRedo;
    } else if (bits) {
        stop = kLoopFault;
    } else if (d->other_rows + d->tail_n + newt > 0xffffffffull) {
        stop = kLoopRowLimit;
    } else {
        // TargetRuntime::apply: the merge already wrote TAIL u NEWT (and its
        // directory) to `spare`; DELTA <- NEWT.
        LoopTrace& tr = d->trace[d->iterations];
        tr.delta_rows = d->delta_n;
        tr.join_rows = joined;
        tr.unique_rows = unique;
        tr.new_rows = newt;
        tr.full_rows = d->other_rows + d->tail_n + newt;
        u64* merged = d->spare;
        d->spare = d->tail;
        d->tail = merged;
        d->tail_n += newt;
        d->lv.keys[d->tail_slot] = merged;
        d->lv.count[d->tail_slot] = d->tail_n;
        d->lv.dir[d->tail_slot] = d->md.dir;
        d->lv.shift[d->tail_slot] = d->md.shift;
        d->lv.buckets[d->tail_slot] = d->md.buckets;
        u64* next_delta = d->newt;
        d->newt = d->delta;
        d->delta = next_delta;
        d->delta_n = newt;
        d->fused.delta = next_delta;
        d->iterations += 1;
        d->total_new += newt;
        if (newt == 0) stop = kLoopConverged;
        else if (d->iterations >= d->limit) stop = kLoopLimit;
        else if (newt * d->max_degree > d->bound) stop = kLoopBound;
        else if (d->tail_n * d->ratio > d->upper_n) stop = kLoopCascade;
    }
    d->stop = stop;
    cudaGraphSetConditional(handle, stop == kLoopRunning ? 1u : 0u);
}

// Per-segment activity of the round just applied (runs after the round-end
// kernel, so a refused round records nothing): its NEWT is now DELTA.
static __global__ void loop_segment_kernel(const LoopDesc* d) {
    const u32 stop = d->stop;
    if (stop != kLoopRunning && stop != kLoopConverged && stop != kLoopLimit && stop != kLoopBound &&
        stop != kLoopCascade)
        return;
    segment_activity(d->delta, d->delta_n, d->seg_shift, d->seg_count,
                     static_cast<u32>(d->rounds_total + d->iterations), d->seg_seen, d->seg_new);
}

}  // namespace spk
