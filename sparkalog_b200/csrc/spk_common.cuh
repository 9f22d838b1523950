// Shared device primitives for the sparkalog B200 kernels.
//
// All kernels here are integer, HBM-bound work (sort, merge, join, compaction);
// none of it is a dense contraction, so the tensor cores are not used.
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

namespace spk {

using u32 = std::uint32_t;
using u64 = std::uint64_t;

constexpr int kWarp = 32;

// Error bits written to a device error word (never a trap or an assert).
enum : u32 {
    kErrLookbackTimeout = 1u << 0,   // a decoupled look-back spin hit its cap
    kErrCapacity = 1u << 1,          // an output did not fit its buffer
    kErrIndexRange = 1u << 2,        // a key outside the dense index range
    kErrMemberProbe = 1u << 3,       // a hash-set probe walked every group (the set was full)
    kErrBarrierTimeout = 1u << 4,    // a bulk-copy barrier wait hit its cap
};

__device__ __forceinline__ u32 lanemask_lt() {
    u32 mask;
    asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(mask));
    return mask;
}

__device__ __forceinline__ u32 lane_id() { return threadIdx.x & (kWarp - 1); }

// Asynchronous 8- and 4-byte global -> shared copies (cp.async, L1-allocating), so a
// thread keeps many loads in flight without holding them in registers.
__device__ __forceinline__ void cp_async_8(void* smem, const void* gmem) {
    const u32 s = static_cast<u32>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_16(void* smem, const void* gmem) {
    const u32 s = static_cast<u32>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_4(void* smem, const void* gmem) {
    const u32 s = static_cast<u32>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}
__device__ __forceinline__ u32 warp_id() { return threadIdx.x / kWarp; }

// ---------------------------------------------------------------------------
// Bulk (TMA, one-dimensional) copies between global and shared memory
// (cp.async.bulk, sm_90+), completed on a shared-memory mbarrier for loads
// and tracked by bulk groups for stores. One thread issues a whole
// contiguous range, so staging a tile costs one instruction instead of one
// per row. Addresses and sizes must be multiples of 16 bytes. No multicast
// form is used anywhere: every copy reads this GPU's own memory.
// ---------------------------------------------------------------------------
__device__ __forceinline__ u32 smem_addr(const void* p) { return static_cast<u32>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar, u32 count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// Makes initialised barriers visible to the asynchronous (bulk copy) proxy.
__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Arrives once and announces `bytes` of bulk-copy transactions for the
// current phase.
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, u32 bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, u32 parity) {
    u32 done;
    asm volatile(
        "{\n"
        ".reg .pred p;\n"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// Spin cap of one mbarrier wait. A bulk copy of a tile from HBM completes in
// microseconds; a wait this long means something is broken, and the caller
// records an error bit instead of waiting forever.
constexpr u32 kBarrierSpinCap = 1u << 24;

// Waits for the barrier's phase `parity` to complete, at most
// kBarrierSpinCap polls; returns false when the cap was hit.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, u32 parity) {
    for (u32 spins = 0; spins < kBarrierSpinCap; ++spins) {
        if (mbar_try_wait(bar, parity)) return true;
        if (spins > 64) __nanosleep(32);
    }
    return false;
}

// Global -> shared bulk copy of `bytes` completing on `bar`.
__device__ __forceinline__ void bulk_load(void* smem_dst, const void* gmem_src, u32 bytes, unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(smem_dst)),
        "l"(gmem_src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// Orders this thread's earlier shared-memory writes before later bulk-copy
// reads of them (generic proxy -> async proxy).
__device__ __forceinline__ void fence_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Shared -> global bulk copy, tracked by the issuing thread's bulk groups.
__device__ __forceinline__ void bulk_store(void* gmem_dst, const void* smem_src, u32 bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(gmem_dst), "r"(smem_addr(smem_src)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// Waits until the issuing thread's bulk stores have finished reading shared memory.
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// Waits until the issuing thread's bulk stores are complete.
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

__device__ __forceinline__ u64 ld_volatile(const u64* p) {
    u64 v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_volatile(u64* p, u64 v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// ---------------------------------------------------------------------------
// Decoupled look-back status words.
//
// One 64-bit word per (tile, channel): [63:40] epoch, [39:38] flag, [37:0]
// value. A word whose epoch differs from the running launch's epoch reads as
// "not yet published", so a status buffer never needs clearing between
// launches as long as consecutive users of one buffer use distinct epochs.
// ---------------------------------------------------------------------------
constexpr u64 kFlagAggregate = 1;
constexpr u64 kFlagInclusive = 2;
constexpr int kValueBits = 38;
constexpr u64 kValueMask = (1ull << kValueBits) - 1;
constexpr u32 kEpochMask = (1u << 24) - 1;

__device__ __forceinline__ u64 make_status(u32 epoch, u64 flag, u64 value) {
    return (static_cast<u64>(epoch & kEpochMask) << 40) | (flag << kValueBits) | (value & kValueMask);
}

// Spin cap for one look-back wait. Predecessor tiles are always held by
// resident CTAs (tile ids come from an atomic counter in acquisition order),
// so a wait this long only happens if something is broken; the kernel then
// records kErrLookbackTimeout and continues with what it has.
constexpr u32 kSpinCap = 1u << 22;

// Sequential look-back for one channel. Returns the exclusive prefix of tile
// `tile` and publishes its inclusive prefix. `status` points at the word of
// tile 0 for this channel; consecutive tiles are `stride` words apart.
__device__ __forceinline__ u64 lookback_exclusive(u64* status, size_t stride, u64 tile, u64 aggregate,
                                                  u32 epoch, u32* err) {
    if (tile == 0) {
        st_volatile(status, make_status(epoch, kFlagInclusive, aggregate));
        return 0;
    }
    st_volatile(status + tile * stride, make_status(epoch, kFlagAggregate, aggregate));
    u64 exclusive = 0;
    long long t = static_cast<long long>(tile) - 1;
    u32 spins = 0;
    while (t >= 0) {
        u64 w = ld_volatile(status + static_cast<u64>(t) * stride);
        u32 e = static_cast<u32>(w >> 40) & kEpochMask;
        u64 flag = (w >> kValueBits) & 3;
        if (e != (epoch & kEpochMask) || flag == 0) {
            if (++spins > kSpinCap) {
                atomicOr(err, kErrLookbackTimeout);
                break;
            }
            if (spins > 64) __nanosleep(64);
            continue;
        }
        exclusive += w & kValueMask;
        if (flag == kFlagInclusive) break;
        --t;
    }
    st_volatile(status + tile * stride, make_status(epoch, kFlagInclusive, exclusive + aggregate));
    return exclusive;
}

// First half of a decoupled look-back: publishes a tile's aggregate (tile 0:
// its inclusive prefix) as soon as it is known, so successors can move on
// while this tile still works. Called by one thread.
__device__ __forceinline__ void lookback_publish(u64* status, u64 tile, u64 aggregate, u32 epoch) {
    st_volatile(status + tile, make_status(epoch, tile == 0 ? kFlagInclusive : kFlagAggregate, aggregate));
}

// Second half: the exclusive prefix from the predecessors' words (lane i
// inspects tile (tile - 1 - i), so 32 predecessors are read per step), then
// the tile's inclusive prefix is published. Must be called by all 32 lanes of
// one warp; every lane gets the result.
__device__ __forceinline__ u64 warp_lookback_resolve(u64* status, u64 tile, u64 aggregate, u32 epoch, u32* err) {
    const u32 lane = lane_id();
    if (tile == 0) return 0;
    u64 exclusive = 0;
    long long base = static_cast<long long>(tile) - 1;
    u32 spins = 0;
    while (base >= 0) {
        long long t = base - lane;
        u64 w = 0;
        bool ready = true;
        u64 flag = 0;
        if (t >= 0) {
            w = ld_volatile(status + t);
            u32 e = static_cast<u32>(w >> 40) & kEpochMask;
            flag = (w >> kValueBits) & 3;
            ready = (e == (epoch & kEpochMask)) && flag != 0;
        } else {
            flag = kFlagInclusive;  // before tile 0: acts as a zero inclusive prefix
            w = 0;
        }
        // Find the first lane (closest predecessor) that is inclusive; every
        // lane up to it must be ready.
        u32 incl = __ballot_sync(0xffffffffu, ready && flag == kFlagInclusive);
        u32 not_ready = __ballot_sync(0xffffffffu, !ready);
        u32 first_incl = incl ? (__ffs(incl) - 1) : 32;
        u32 first_wait = not_ready ? (__ffs(not_ready) - 1) : 32;
        if (first_wait < first_incl || (first_incl == 32 && first_wait < 32)) {
            if (++spins > kSpinCap) {
                if (lane == 0) atomicOr(err, kErrLookbackTimeout);
                break;
            }
            if (spins > 64) __nanosleep(64);
            continue;
        }
        u64 v = (lane <= first_incl && t >= 0) ? (w & kValueMask) : 0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        exclusive += v;
        if (first_incl < 32) break;
        base -= 32;
    }
    if (lane == 0) st_volatile(status + tile, make_status(epoch, kFlagInclusive, exclusive + aggregate));
    return exclusive;
}

// Look-back that does not wait: walks from *base (the closest predecessor not
// yet summed, adding into *exclusive) while the predecessors' words are
// published. Returns true, with the tile's inclusive prefix published, once
// it reaches an inclusive word; returns false at the first unpublished word,
// with the walk's state left in *base and *exclusive for a later call. Called
// by all 32 lanes of one warp with identical state; tile 0 starts at base -1.
__device__ __forceinline__ bool warp_lookback_try(u64* status, u64 tile, u64 aggregate, u32 epoch, long long* base,
                                                  u64* exclusive) {
    const u32 lane = lane_id();
    for (;;) {
        const long long t = *base - static_cast<long long>(lane);
        u64 w = 0;
        bool ready = true;
        u64 flag = kFlagInclusive;  // before tile 0: a zero inclusive prefix
        if (t >= 0) {
            w = ld_volatile(status + t);
            const u32 e = static_cast<u32>(w >> 40) & kEpochMask;
            flag = (w >> kValueBits) & 3;
            ready = (e == (epoch & kEpochMask)) && flag != 0;
        }
        const u32 incl = __ballot_sync(0xffffffffu, ready && flag == kFlagInclusive);
        const u32 not_ready = __ballot_sync(0xffffffffu, !ready);
        const u32 first_incl = incl ? (__ffs(incl) - 1) : 32;
        const u32 first_wait = not_ready ? (__ffs(not_ready) - 1) : 32;
        const bool blocked = first_wait < first_incl;
        const u32 take = blocked ? first_wait : (first_incl < 32 ? first_incl + 1 : 32);
        u64 v = (lane < take && t >= 0) ? (w & kValueMask) : 0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        *exclusive += v;
        if (blocked) {
            *base -= static_cast<long long>(first_wait);
            return false;
        }
        if (first_incl < 32) {
            if (lane == 0) st_volatile(status + tile, make_status(epoch, kFlagInclusive, *exclusive + aggregate));
            return true;
        }
        *base -= 32;
    }
}

// Completes a walk that warp_lookback_try left unfinished, waiting for the
// predecessors still unpublished (capped; kErrLookbackTimeout past the cap).
__device__ __forceinline__ void warp_lookback_finish(u64* status, u64 tile, u64 aggregate, u32 epoch, long long* base,
                                                     u64* exclusive, u32* err) {
    u32 spins = 0;
    while (!warp_lookback_try(status, tile, aggregate, epoch, base, exclusive)) {
        if (++spins > kSpinCap) {
            if (lane_id() == 0) atomicOr(err, kErrLookbackTimeout);
            return;
        }
        if (spins > 64) __nanosleep(64);
    }
}

// Warp-cooperative look-back for a single channel (used by compaction
// kernels): publish and resolve back to back. Must be called by all 32 lanes
// of one warp; every lane gets the result.
__device__ __forceinline__ u64 warp_lookback_exclusive(u64* status, u64 tile, u64 aggregate, u32 epoch,
                                                       u32* err) {
    if (lane_id() == 0) lookback_publish(status, tile, aggregate, epoch);
    return warp_lookback_resolve(status, tile, aggregate, epoch, err);
}

// ---------------------------------------------------------------------------
// Block-wide exclusive scan of one value per thread (THREADS % 32 == 0).
// `scratch` holds THREADS/32 + 1 words. Returns the exclusive prefix and
// writes the block total to *total. Contains __syncthreads().
// ---------------------------------------------------------------------------
template <int THREADS, typename T>
__device__ __forceinline__ T block_exclusive_scan(T value, T* scratch, T* total) {
    constexpr int kWarps = THREADS / kWarp;
    const u32 lane = lane_id(), warp = warp_id();
    T inclusive = value;
#pragma unroll
    for (int o = 1; o < kWarp; o <<= 1) {
        T n = __shfl_up_sync(0xffffffffu, inclusive, o);
        if (lane >= static_cast<u32>(o)) inclusive += n;
    }
    if (lane == kWarp - 1) scratch[warp] = inclusive;
    __syncthreads();
    if (warp == 0) {
        T w = lane < static_cast<u32>(kWarps) ? scratch[lane] : T(0);
        T wi = w;
#pragma unroll
        for (int o = 1; o < kWarp; o <<= 1) {
            T n = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= static_cast<u32>(o)) wi += n;
        }
        if (lane < static_cast<u32>(kWarps)) scratch[lane] = wi - w;
        if (lane == kWarps - 1) scratch[kWarps] = wi;
    }
    __syncthreads();
    T result = scratch[warp] + inclusive - value;
    *total = scratch[kWarps];
    return result;
}

inline unsigned int ceil_div_u(size_t a, size_t b) { return static_cast<unsigned int>((a + b - 1) / b); }

}  // namespace spk
