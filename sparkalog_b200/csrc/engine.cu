// Device-resident RelationStore / RecursiveExecutor (the Tier B C ABI).
//
// Semantics follow crates/sparkalog-recursion/src/generic.rs:
//   RelationStore            :16-121   (FULL / DELTA / NEWT per relation)
//   RuleRuntime::evaluate    :197-259  (cached right index, join, distinct)
//   TargetRuntime::combine   :299-358  (union of clause outputs, anti-join)
//   TargetRuntime::apply     :360-397  (FULL u= NEWT, DELTA <- NEWT)
//   RecursiveExecutor::run   :472-525  (loop while any DELTA is non-empty,
//                                       counting every executed round)
//
// B200 layout: every relation lives on the device as packed 64-bit rows
// (first << 32 | second), so lexicographic pair order is u64 order. One round
// of the loop is a fixed sequence of kernels on one stream:
//   join (fused count/scan/emit)  ->  radix sort of the candidates
//   ->  unique + anti-join against the FULL levels (one fused pass)  ->  NEWT
//   ->  merge NEWT into the levels  ->  DELTA <- NEWT
// with one small device-to-host copy of the round's counts per round.
//
// Clause outputs of one target are appended into one candidate buffer and
// sorted once: unique(A ++ B) equals the reference's union of the two
// distinct outputs (generic.rs:317-336).

#include "sparkalog_b200.h"
#include "spk_common.cuh"
#include "spk_engine_kernels.cuh"
#include "spk_host.h"
#include "spk_join.cuh"
#include "spk_radix.cuh"
#include "spk_fused.cuh"
#include "spk_member.cuh"
#include "spk_ingest.cuh"
#include "spk_anti_merge.cuh"
#include "spk_bloom.cuh"
#include "spk_loop.cuh"
#include "spk_setops.cuh"

#include <algorithm>
#include <mutex>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <system_error>
#include <thread>
#include <vector>

using spk::u32;
using spk::u64;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& message) {
    g_last_error = message;
    return code;
}

int cuda_fail(cudaError_t st, const char* what) {
    g_last_error = std::string(what) + " failed with CUDA error " + std::to_string(static_cast<int>(st)) + " (" +
                   cudaGetErrorString(st) + ")";
    return static_cast<int>(st);
}

// Small pinned host buffers (counts, error words) are recycled per size class
// instead of freed: cudaFreeHost synchronises the whole device and unpins
// pages, which would make every store or executor teardown a device-wide
// barrier.
std::mutex g_pinned_mu;
std::map<size_t, std::vector<void*>> g_pinned_free;

size_t pinned_class(size_t bytes) {
    size_t c = 256;
    while (c < bytes) c <<= 1;
    return c;
}

cudaError_t pinned_get(void** p, size_t bytes) {
    const size_t c = pinned_class(bytes);
    {
        std::lock_guard<std::mutex> lock(g_pinned_mu);
        auto& list = g_pinned_free[c];
        if (!list.empty()) {
            *p = list.back();
            list.pop_back();
            return cudaSuccess;
        }
    }
    return cudaMallocHost(p, c);
}

void pinned_put(void* p, size_t bytes) {
    if (!p) return;
    std::lock_guard<std::mutex> lock(g_pinned_mu);
    g_pinned_free[pinned_class(bytes)].push_back(p);
}

// Device columns into caller host memory. A page-locked destination, or a
// small copy, takes one DMA per column. For a large pageable destination the
// driver would stage every byte through its own page-locked buffer on one
// thread, page faults included (a few GB/s); instead the columns are cut into
// chunks that several host threads each DMA into a page-locked chunk of their
// own and copy out while the other threads' chunks are in flight.
constexpr size_t kHostChunk = 8u << 20;
constexpr size_t kStagedMin = 32u << 20;

cudaError_t columns_to_host(u32* first, u32* second, const u32* d0, const u32* d1, u64 n, cudaStream_t s) {
    const size_t bytes = n * 4;
    cudaPointerAttributes attr{};
    cudaError_t e = cudaPointerGetAttributes(&attr, first);
    if (e != cudaSuccess) return e;
    const bool pageable = attr.type == cudaMemoryTypeUnregistered;
    if (!pageable || bytes < kStagedMin) {
        e = cudaMemcpyAsync(first, d0, bytes, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(second, d1, bytes, cudaMemcpyDeviceToHost, s);
        return e;
    }
    struct Job {
        char* dst;
        const char* src;
        size_t len;
    };
    std::vector<Job> jobs;
    for (int c = 0; c < 2; ++c) {
        char* dst = reinterpret_cast<char*>(c ? second : first);
        const char* src = reinterpret_cast<const char*>(c ? d1 : d0);
        for (size_t off = 0; off < bytes; off += kHostChunk)
            jobs.push_back({dst + off, src + off, std::min(kHostChunk, bytes - off)});
    }
    int device = 0;
    e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t workers = std::min<size_t>({16, std::max(1u, hw / 2), jobs.size()});
    std::atomic<int> status{cudaSuccess};
    auto work = [&](size_t t) {
        cudaError_t w = cudaSetDevice(device);
        void* buf = nullptr;
        cudaEvent_t ev = nullptr;
        if (w == cudaSuccess) w = pinned_get(&buf, kHostChunk);
        if (w == cudaSuccess) w = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        for (size_t j = t; w == cudaSuccess && j < jobs.size(); j += workers) {
            if (status.load(std::memory_order_relaxed) != cudaSuccess) break;
            w = cudaMemcpyAsync(buf, jobs[j].src, jobs[j].len, cudaMemcpyDeviceToHost, s);
            if (w == cudaSuccess) w = cudaEventRecord(ev, s);
            if (w == cudaSuccess) w = cudaEventSynchronize(ev);
            if (w == cudaSuccess) std::memcpy(jobs[j].dst, buf, jobs[j].len);
        }
        if (ev) cudaEventDestroy(ev);
        if (buf) pinned_put(buf, kHostChunk);
        if (w != cudaSuccess) {
            int expect = cudaSuccess;
            status.compare_exchange_strong(expect, static_cast<int>(w));
        }
    };
    std::vector<std::thread> pool;
    size_t started = 0;
    try {
        for (; started + 1 < workers; ++started) pool.emplace_back(work, started + 1);
    } catch (const std::system_error&) {
        // Fewer threads than planned: the jobs of the missing ones run below.
    }
    work(0);
    for (auto& th : pool) th.join();
    for (size_t t = started + 1; t < workers; ++t) work(t);
    return static_cast<cudaError_t>(status.load());
}

#define SPK_CUDA(expr, what)                         \
    do {                                             \
        cudaError_t _st = (expr);                    \
        if (_st != cudaSuccess) return cuda_fail(_st, what); \
    } while (0)

constexpr int kThreads = 256;
constexpr int kSetItems = 8;
constexpr int kSetTile = kThreads * kSetItems;
constexpr int kJoinItems = 8;
constexpr int kJoinTile = kThreads * kJoinItems;
constexpr u64 kMaxRelationRows = 0xffffffffull;  // row ids are u32
constexpr size_t kCounterWords = 1024;  // per-round tile counters
constexpr int kLevelStage = 2048;  // level rows per shared-memory chunk of the anti-join (two buffers)
constexpr int kSparseThreads = 256;  // anti-join of small candidate sets
constexpr int kSparseItems = 4;
constexpr int kSparseTile = kSparseThreads * kSparseItems;
constexpr int kSparseMinTile = kSparseThreads * 2;  // the per-thread search's smallest tile (sparse_items 2)
constexpr int kAntiMergeThreads = 256;  // merge-form anti-join: 9 merged rows per thread,
constexpr int kAntiMergeItems = 9;      // 1,024 rows of side slices per stage
constexpr int kAntiMergeSide = 1024;
constexpr int kAntiMergeTile = kAntiMergeThreads * kAntiMergeItems;
constexpr int kWideThreads = 256;    // group-searched anti-join (lanes per candidate: tuning.group_lanes)
constexpr int kSortThreads = spk::RadixSortConfig::kThreads;
constexpr int kSortItems = spk::RadixSortConfig::kItems;
constexpr int kSortTile = spk::RadixSortConfig::kTile;

// Built-in tuning (sparkalog_tuning in the header). Candidate bounds up to
// group_candidates use the group-searched anti-join, whose rounds are
// latency-bound; on the 16.7M-node ER fixpoint 2^17 took 18.75 ms against
// 18.86 ms for 2^15 and 18.77 ms for 2^19 with 64-row directory buckets.
sparkalog_tuning default_tuning() {
    sparkalog_tuning t{};
    t.dir_rows_log2 = 6;
    t.group_lanes = 8;
    t.group_candidates = 1ull << 17;
    t.sparse_candidates = 1ull << 26;
    t.fused_rows_cap = 672;
    t.merge_items = 11;
    t.level_ratio = 4;
    t.levels = 3;
    t.bloom_bits = 0;
    t.merge_anti_ratio = 0;
    t.sparse_items = 2;
    t.compact_index = 1;
    return t;
}

bool tuning_valid(const sparkalog_tuning& t) {
    const bool lanes = t.group_lanes == 4 || t.group_lanes == 8 || t.group_lanes == 16;
    return t.dir_rows_log2 <= 10 && lanes && t.fused_rows_cap >= 64 && t.fused_rows_cap <= 768 &&
           (t.merge_items == 7 || t.merge_items == 11 || t.merge_items == 15) && t.level_ratio >= 2 && t.level_ratio <= 64 && t.levels >= 2 &&
           t.levels <= static_cast<u32>(spk::kMaxLevels) && t.group_candidates <= t.sparse_candidates &&
           (t.bloom_bits == 0 || (t.bloom_bits >= 4 && t.bloom_bits <= 32)) && t.merge_anti_ratio <= 1024 &&
           t.sparse_items >= 2 && t.sparse_items <= 4 && t.compact_index <= 1;
}

// A stream-ordered device allocation that only grows.
struct DevArray {
    void* ptr = nullptr;
    size_t bytes = 0;

    template <class T>
    T* as() const { return static_cast<T*>(ptr); }

    // Grows to at least `need` bytes. With keep_bytes > 0 the first keep_bytes
    // bytes are preserved.
    cudaError_t ensure(size_t need, cudaStream_t s, size_t keep_bytes = 0) {
        if (need <= bytes && ptr) return cudaSuccess;
        size_t cap = std::max<size_t>(need, 4096);
        cap = std::max(cap, bytes + bytes / 2);
        cap = spk::align_up(cap, 256);
        void* fresh = nullptr;
        cudaError_t st = cudaMallocAsync(&fresh, cap, s);
        if (st != cudaSuccess) return st;
        if (keep_bytes && ptr) {
            st = cudaMemcpyAsync(fresh, ptr, std::min(keep_bytes, bytes), cudaMemcpyDeviceToDevice, s);
            if (st != cudaSuccess) return st;
        }
        if (ptr) cudaFreeAsync(ptr, s);
        ptr = fresh;
        bytes = cap;
        return cudaSuccess;
    }

    // Like ensure(), but a fresh allocation is zero-filled. Decoupled
    // look-back status buffers must start zeroed: pool memory recycled from
    // relation rows can otherwise decode as a published status word.
    cudaError_t ensure_zeroed(size_t need, cudaStream_t s) {
        if (need <= bytes && ptr) return cudaSuccess;
        cudaError_t st = ensure(need, s);
        if (st != cudaSuccess) return st;
        return cudaMemsetAsync(ptr, 0, bytes, s);
    }

    void release(cudaStream_t s) {
        if (ptr) cudaFreeAsync(ptr, s);
        ptr = nullptr;
        bytes = 0;
    }
};

void swap_arrays(DevArray& a, DevArray& b) {
    std::swap(a.ptr, b.ptr);
    std::swap(a.bytes, b.bytes);
}

struct RelState {
    bool recursive = false;
    u64 version = 0;
    bool sorted = true;     // level[0] as inserted is non-decreasing
    bool has_dups = false;  // level[0] as inserted has adjacent duplicates
    DevArray level[spk::kMaxLevels];
    u64 level_n[spk::kMaxLevels] = {};
    // Bucket directories of the levels (see spk::Levels), rebuilt lazily
    // after a level changes.
    DevArray dir[spk::kMaxLevels];
    bool dir_valid[spk::kMaxLevels] = {};
    u32 dir_shift[spk::kMaxLevels] = {};
    u64 dir_buckets[spk::kMaxLevels] = {};
    DevArray spare;         // merge destination, swapped with a level after a merge
    DevArray delta, newt;
    u64 delta_n = 0;
    bool delta_sorted = true;  // DELTA is sorted and unique (always after a round)
    // FULL as a hash set (spk::MemberSet) for the anti-join of recursive
    // relations; built lazily from the levels, kept in step with every round's
    // NEWT, dropped when FULL changes otherwise or the load passes one half.
    DevArray member;         // 4 * member_groups u64 slots
    DevArray member_flag;    // u32: the row spk::kEmptySlot is a member
    u64 member_groups = 0;   // power of two
    u64 member_count = 0;    // rows inserted
    bool member_valid = false;
    // FULL's blocked Bloom filter (spk_bloom.cuh), when the tuning asks for
    // one: built from the levels, kept in step by the anti-join, dropped when
    // FULL changes otherwise.
    DevArray bloom;
    u64 bloom_blocks = 0;
    u64 bloom_capacity = 0;  // rows the filter was sized for
    bool bloom_valid = false;

    u64 full_rows() const {
        u64 n = 0;
        for (int l = 0; l < spk::kMaxLevels; ++l) n += level_n[l];
        return n;
    }
};

}  // namespace

struct StoreOps;

struct sparkalog_store {
    cudaStream_t stream = nullptr;
    std::map<u32, RelState> relations;
    DevArray scratch_u32[2];   // staging columns for host inserts / reads
    DevArray flags;            // device flag words
    DevArray merge_splits;     // diagonal splits of the merge pre-pass
    u32 max_value = 0;         // largest value stored in any column
    u32 dir_rows_log2 = 6;     // ~2^k rows per level-directory bucket
    u32 merge_items = 11;      // rows per thread of a merge tile
    DevArray fault;            // u32 error bits of the store's merges (read when a run ends)
    u32 levels = 3;            // sorted runs of a recursive FULL (the last executor run's tuning)
    StoreOps* ops = nullptr;   // scratch of store-level operations (anti-join, append, segments)
    u32* pinned = nullptr;     // small pinned host buffer

    RelState* find(u32 id) {
        auto it = relations.find(id);
        return it == relations.end() ? nullptr : &it->second;
    }
};

namespace {

unsigned grid_for(const void* kernel, int threads, size_t tiles) {
    return spk::persistent_grid(kernel, threads, 0, tiles);
}

unsigned simple_grid(size_t n) {
    size_t blocks = (n + 255) / 256;
    size_t cap = static_cast<size_t>(spk::device_sm_count()) * 8;
    return static_cast<unsigned>(std::max<size_t>(1, std::min(blocks, cap)));
}

// Merge of two disjoint sorted runs into `out` (capacity checked by caller):
// the diagonal splits (one warp per diagonal), then the bulk-copy merge with
// `items` rows per thread (7, 11 or 15). Returns the number of kernels
// launched through *launches. Errors of the merge's barrier waits go to *err.
// Merges of at least this many tiles find their diagonals one per thread
// (merge_split_thread_kernel); smaller ones one per warp.
constexpr u64 kThreadSplitTiles = 8192;

template <int ITEMS>
cudaError_t launch_merge_items(const u64* a, u64 na, const u64* b, u64 nb, u64* out, DevArray& splits,
                               cudaStream_t s, u32* err, spk::MergeDirectory md) {
    constexpr int kTile = kThreads * ITEMS;
    using Layout = spk::MergeBulkLayout<kThreads, ITEMS>;
    auto kernel = spk::merge_bulk_kernel<kThreads, ITEMS>;
    const u64 total = na + nb;
    const u64 tiles = (total + kTile - 1) / kTile;
    cudaError_t st = splits.ensure((tiles + 1) * 8, s);
    if (st != cudaSuccess) return st;
    {
        if (tiles >= kThreadSplitTiles) {
            const u64 blocks = std::min<u64>((tiles + 1 + 127) / 128, static_cast<u64>(spk::device_sm_count()) * 16);
            spk::merge_split_thread_kernel<<<static_cast<unsigned>(blocks), 128, 0, s>>>(a, na, b, nb, kTile, tiles,
                                                                                       splits.as<u64>());
        } else {
            const u64 warps = tiles + 1;
            const u64 blocks = std::min<u64>((warps + 7) / 8, static_cast<u64>(spk::device_sm_count()) * 8);
            spk::merge_split_kernel<<<static_cast<unsigned>(std::max<u64>(blocks, 1)), 256, 0, s>>>(
                a, na, b, nb, kTile, tiles, splits.as<u64>());
        }
        st = cudaGetLastError();
        if (st != cudaSuccess) return st;
    }
    // The shared-memory opt-in is per device.
    static std::atomic<u64> configured{0};
    int device = 0;
    st = cudaGetDevice(&device);
    if (st != cudaSuccess) return st;
    const u64 bit = 1ull << (device & 63);
    if (!(configured.load() & bit)) {
        st = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(Layout::kBytes));
        if (st != cudaSuccess) return st;
        configured.fetch_or(bit);
    }
    const u64 grid0 = spk::persistent_grid(reinterpret_cast<const void*>(kernel), kThreads, Layout::kBytes, tiles);
    const u64 chunk = (tiles + grid0 - 1) / grid0;
    const u64 grid = (tiles + chunk - 1) / chunk;
    kernel<<<static_cast<unsigned>(grid), kThreads, Layout::kBytes, s>>>(a, na, b, nb, splits.as<u64>(), chunk, out,
                                                                         md, err);
    return cudaGetLastError();
}

cudaError_t launch_merge(const u64* a, u64 na, const u64* b, u64 nb, u64* out, DevArray& splits, cudaStream_t s,
                         u32 items, u32* err, u64* launches = nullptr,
                         spk::MergeDirectory md = spk::MergeDirectory{nullptr, 0, 0}) {
    if (launches) *launches = 0;
    if (na + nb == 0) return cudaSuccess;
    if (nb == 0) return cudaMemcpyAsync(out, a, na * 8, cudaMemcpyDeviceToDevice, s);
    if (na == 0) return cudaMemcpyAsync(out, b, nb * 8, cudaMemcpyDeviceToDevice, s);
    if (launches) *launches = 2;
    if (items == 7) return launch_merge_items<7>(a, na, b, nb, out, splits, s, err, md);
    if (items == 15) return launch_merge_items<15>(a, na, b, nb, out, splits, s, err, md);
    return launch_merge_items<11>(a, na, b, nb, out, splits, s, err, md);
}

// A store's merges: its split buffer, merge shape and fault word.
cudaError_t store_merge(sparkalog_store* st, const u64* a, u64 na, const u64* b, u64 nb, u64* out,
                        u64* launches = nullptr, spk::MergeDirectory md = spk::MergeDirectory{nullptr, 0, 0}) {
    return launch_merge(a, na, b, nb, out, st->merge_splits, st->stream, st->merge_items, st->fault.as<u32>(),
                        launches, md);
}

// Reads (and clears) the store's merge fault bits; non-zero bits fail.
int check_store_fault(sparkalog_store* st) {
    cudaStream_t s = st->stream;
    SPK_CUDA(cudaMemcpyAsync(st->pinned + 2, st->fault.ptr, 4, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync");
    SPK_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    const u32 bits = st->pinned[2];
    if (bits) {
        SPK_CUDA(cudaMemsetAsync(st->fault.ptr, 0, 4, s), "cudaMemsetAsync");
        return fail(SPARKALOG_E_DEVICE_FAULT, "device error bits " + std::to_string(bits) + " (merge)");
    }
    return 0;
}

// Collapses all levels of a relation into level[0] (a single sorted run).
// Levels are disjoint sorted runs, larger towards level 0, so the smallest
// merge first: each level merges into the nearest non-empty level below it,
// from the top down, and level 0 is rewritten once.
int materialize(sparkalog_store* st, RelState& r) {
    cudaStream_t s = st->stream;
    for (int l = spk::kMaxLevels - 1; l >= 1; --l) {
        if (r.level_n[l] == 0) continue;
        int t = l - 1;
        while (t > 0 && r.level_n[t] == 0) --t;
        if (r.level_n[t] == 0) {
            swap_arrays(r.level[t], r.level[l]);
        } else {
            const u64 total = r.level_n[t] + r.level_n[l];
            SPK_CUDA(r.spare.ensure(total * 8, s), "cudaMallocAsync");
            SPK_CUDA(store_merge(st, r.level[t].as<u64>(), r.level_n[t], r.level[l].as<u64>(), r.level_n[l],
                                 r.spare.as<u64>()),
                     "merge_bulk_kernel");
            swap_arrays(r.level[t], r.spare);
        }
        r.level_n[t] += r.level_n[l];
        r.level_n[l] = 0;
        r.dir_valid[t] = r.dir_valid[l] = false;
    }
    return 0;
}

// Uploads (or adopts device) columns and packs them into `dst`.
int pack_columns(sparkalog_store* st, const u32* c0, const u32* c1, size_t rows, int location, DevArray& dst,
                 bool* sorted, bool* has_dups) {
    cudaStream_t s = st->stream;
    *sorted = true;
    *has_dups = false;
    SPK_CUDA(dst.ensure(std::max<size_t>(rows, 1) * 8, s), "cudaMallocAsync");
    if (rows == 0) return 0;
    if (c0 == nullptr || c1 == nullptr) return fail(SPARKALOG_E_INVALID_ARGUMENT, "null column pointer");
    const u32* d0 = c0;
    const u32* d1 = c1;
    if (location == SPARKALOG_HOST) {
        SPK_CUDA(st->scratch_u32[0].ensure(rows * 4, s), "cudaMallocAsync");
        SPK_CUDA(st->scratch_u32[1].ensure(rows * 4, s), "cudaMallocAsync");
        SPK_CUDA(cudaMemcpyAsync(st->scratch_u32[0].ptr, c0, rows * 4, cudaMemcpyHostToDevice, s), "cudaMemcpyAsync");
        SPK_CUDA(cudaMemcpyAsync(st->scratch_u32[1].ptr, c1, rows * 4, cudaMemcpyHostToDevice, s), "cudaMemcpyAsync");
        d0 = st->scratch_u32[0].as<u32>();
        d1 = st->scratch_u32[1].as<u32>();
    }
    u32* flags = st->flags.as<u32>();
    SPK_CUDA(cudaMemsetAsync(flags, 0, 8, s), "cudaMemsetAsync");
    spk::pack_rows_kernel<<<simple_grid(rows), 256, 0, s>>>(d0, d1, rows, dst.as<u64>(), flags);
    SPK_CUDA(cudaGetLastError(), "pack_rows_kernel");
    SPK_CUDA(cudaMemcpyAsync(st->pinned, flags, 8, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync");
    SPK_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    *sorted = (st->pinned[0] & 1u) == 0;
    *has_dups = (st->pinned[0] & 2u) != 0;
    st->max_value = std::max(st->max_value, st->pinned[1]);
    return 0;
}

// Rebuilds the bucket directory of every non-empty level whose rows changed.
// The bucket width comes from the store's largest value, which bounds every
// key: ~2^dir_rows_log2 rows per bucket.
void directory_shape(const sparkalog_store* st, u64 rows, u32* shift, u64* buckets) {
    const u64 key_max = (static_cast<u64>(st->max_value) << 32) | st->max_value;
    const int key_bits = 64 - __builtin_clzll(key_max | 1);
    const int target_bits = 64 - __builtin_clzll(std::max<u64>(rows >> st->dir_rows_log2, 1));
    *shift = static_cast<u32>(std::max(0, key_bits - target_bits));
    *buckets = (key_max >> *shift) + 1;
}

int refresh_directories(sparkalog_store* st, RelState& r, cudaStream_t s, u64* launches) {
    for (int l = 0; l < spk::kMaxLevels; ++l) {
        if (r.level_n[l] == 0 || r.dir_valid[l]) continue;
        u32 shift;
        u64 buckets;
        directory_shape(st, r.level_n[l], &shift, &buckets);
        SPK_CUDA(r.dir[l].ensure((buckets + 1) * 4, s), "cudaMallocAsync");
        spk::level_directory_kernel<<<simple_grid(buckets + 1), 256, 0, s>>>(r.level[l].as<u64>(), r.level_n[l], shift,
                                                                            buckets, r.dir[l].as<u32>());
        SPK_CUDA(cudaGetLastError(), "level_directory_kernel");
        r.dir_shift[l] = shift;
        r.dir_buckets[l] = buckets;
        r.dir_valid[l] = true;
        if (launches) *launches += 1;
    }
    return 0;
}

// Grows r.spare and level l's directory for a merged level of n rows (done
// before the merge so that allocation stays out of its timing).
int merge_buffers(sparkalog_store* st, RelState& r, int l, u64 n, cudaStream_t s) {
    u32 shift;
    u64 buckets;
    directory_shape(st, n, &shift, &buckets);
    SPK_CUDA(r.spare.ensure(n * 8, s), "cudaMallocAsync");
    SPK_CUDA(r.dir[l].ensure((buckets + 1) * 4, s), "cudaMallocAsync");
    return 0;
}

// Merges two disjoint sorted runs into level l of r (through r.spare) and
// writes the merged level's directory on the way when the merge runs a kernel.
int merge_into_level(sparkalog_store* st, RelState& r, int l, const u64* a, u64 na, const u64* b, u64 nb,
                     cudaStream_t s, u64* launches) {
    const u64 n = na + nb;
    SPK_CUDA(r.spare.ensure(n * 8, s), "cudaMallocAsync");
    u32 shift;
    u64 buckets;
    directory_shape(st, n, &shift, &buckets);
    SPK_CUDA(r.dir[l].ensure((buckets + 1) * 4, s), "cudaMallocAsync");
    u64 launched = 0;
    SPK_CUDA(store_merge(st, a, na, b, nb, r.spare.as<u64>(), &launched,
                         spk::MergeDirectory{r.dir[l].as<u32>(), shift, buckets}),
             "merge_bulk_kernel");
    swap_arrays(r.level[l], r.spare);
    r.level_n[l] = n;
    r.dir_valid[l] = launched > 0;  // a plain copy (one side empty) wrote no directory
    r.dir_shift[l] = shift;
    r.dir_buckets[l] = buckets;
    if (launches) *launches += launched;
    return 0;
}

// FULL's hash set (spk::MemberSet). The host keeps its load at most one half
// and builds it with sixteen slots per row, so a recursive FULL can grow
// eightfold before the set is rebuilt.
constexpr u64 kMemberMinGroups = 4096;

spk::MemberSet member_set(RelState& r) {
    return spk::MemberSet{r.member.as<u64>(), r.member_groups - 1, r.member_flag.as<u32>()};
}

// Builds the set from every level of FULL. Leaves member_valid false (and
// returns 0) when the device has too little free memory for it; the caller
// then searches the sorted levels instead.
int member_build(RelState& r, u32* err, cudaStream_t s, u64* launches) {
    const u64 rows = r.full_rows();
    u64 groups = kMemberMinGroups;
    while (groups < 4 * rows) groups <<= 1;
    const size_t bytes = groups * 32;
    r.member_valid = false;
    if (bytes > r.member.bytes) {
        size_t free_bytes = 0, total_bytes = 0;
        if (cudaMemGetInfo(&free_bytes, &total_bytes) != cudaSuccess) {
            cudaGetLastError();
            return 0;
        }
        if (bytes > free_bytes / 2) return 0;
    }
    SPK_CUDA(r.member.ensure(bytes, s), "cudaMallocAsync");
    SPK_CUDA(r.member_flag.ensure(256, s), "cudaMallocAsync");
    SPK_CUDA(cudaMemsetAsync(r.member.ptr, 0xff, bytes, s), "cudaMemsetAsync");
    SPK_CUDA(cudaMemsetAsync(r.member_flag.ptr, 0, 4, s), "cudaMemsetAsync");
    r.member_groups = groups;
    const spk::MemberSet set = member_set(r);
    for (int l = 0; l < spk::kMaxLevels; ++l) {
        if (r.level_n[l] == 0) continue;
        spk::member_insert_kernel<<<simple_grid(r.level_n[l]), 256, 0, s>>>(r.level[l].as<u64>(), r.level_n[l], set,
                                                                           err);
        SPK_CUDA(cudaGetLastError(), "member_insert_kernel");
        if (launches) *launches += 1;
    }
    r.member_count = rows;
    r.member_valid = true;
    return 0;
}

// Adds rows (new to FULL, distinct) to a valid set; drops the set instead
// when they would push its load past one half.
int member_add(RelState& r, const u64* rows, u64 n, u32* err, cudaStream_t s, u64* launches) {
    if (!r.member_valid || n == 0) return 0;
    if ((r.member_count + n) * 2 > r.member_groups * 4) {
        r.member_valid = false;
        return 0;
    }
    spk::member_insert_kernel<<<simple_grid(n), 256, 0, s>>>(rows, n, member_set(r), err);
    SPK_CUDA(cudaGetLastError(), "member_insert_kernel");
    if (launches) *launches += 1;
    r.member_count += n;
    return 0;
}

// FULL's Bloom filter: 2^k blocks of 256 bits, about `bits` bits per row
// for 8 times the rows FULL holds when it is built (a recursive relation
// grows several-fold), rebuilt larger once FULL outgrows that.
spk::Bloom bloom_of(RelState& r) { return spk::Bloom{r.bloom.as<u32>(), r.bloom_blocks - 1}; }

int bloom_build(RelState& r, u32 bits, cudaStream_t s, u64* launches) {
    const u64 rows = std::max<u64>(r.full_rows(), 1);
    u64 blocks = 4096;
    while (blocks * 256 < 8 * rows * bits) blocks <<= 1;
    SPK_CUDA(r.bloom.ensure(blocks * 32, s), "cudaMallocAsync");
    SPK_CUDA(cudaMemsetAsync(r.bloom.ptr, 0, blocks * 32, s), "cudaMemsetAsync");
    r.bloom_blocks = blocks;
    r.bloom_capacity = blocks * 256 / bits;
    const spk::Bloom bf = bloom_of(r);
    for (int l = 0; l < spk::kMaxLevels; ++l) {
        if (r.level_n[l] == 0) continue;
        spk::bloom_insert_kernel<<<simple_grid(r.level_n[l]), 256, 0, s>>>(r.level[l].as<u64>(), r.level_n[l], bf);
        SPK_CUDA(cudaGetLastError(), "bloom_insert_kernel");
        if (launches) *launches += 1;
    }
    r.bloom_valid = true;
    return 0;
}

// A valid filter for FULL before its anti-join (built, or rebuilt larger).
int bloom_ready(RelState& r, u32 bits, cudaStream_t s, u64* launches) {
    if (r.bloom_valid && r.full_rows() <= r.bloom_capacity) return 0;
    return bloom_build(r, bits, s, launches);
}

struct SortScratch {
    DevArray plan;     // RadixPlan
    DevArray status;   // look-back words
};

struct IndexCache {
    bool valid = false;
    u32 relation = 0;
    u64 version = 0;
    u32 column = 0;
    DevArray offsets;   // u32[num_keys + 1] (dense index)
    u32* values_ptr = nullptr;  // u32[n] inside `offsets`: the second column in row order (identity)
    // Compact form of an identity dense index (tuning.compact_index): 4-bit
    // match counts, eight keys to a word, then a word per key (its single
    // match, else its first offset), both inside `compact`.
    DevArray compact;
    u32* key_class = nullptr;
    u32* key_word = nullptr;
    DevArray rows;      // u32[n] (empty when identity)
    bool identity = true;
    u64 num_keys = 0;
    u32 max_degree = 0;
    // Bucketed index, used when the key domain is much larger than the row
    // count (tagged serving keys): sorted first-column keys plus a bucket
    // directory over them, instead of max_key + 1 dense offsets.
    bool bucketed = false;
    DevArray keys32;    // u32[n]
    DevArray bucket_dir;
    u32 bucket_shift = 0;
    u64 buckets = 0;
};

struct TargetRT {
    u32 id = 0;
    std::vector<size_t> rules;
    DevArray j_a, j_b;     // candidate buffers (sort ping-pong)
    u64 j_cap = 0;         // elements
    SortScratch sort;
    u32 fused_rows = 672;      // DELTA rows per fused tile in the next round
    u32 fused_rows_cap = 672;  // its ceiling, halved whenever a tile overflows
    bool force_generic = false;  // redo the current round with the general kernels
    bool fused_last = false;     // the round just applied ran the fused kernel
    DevArray anti_plan;          // merge-form anti-join tiles (spk::AntiTile)
    DevArray anti_scratch;       // ... each tile's kept run, at its first candidate index
    DevArray anti_counts;        // ... and its length (u32 per tile)
    double unique_per_delta = -1.0;  // last round's distinct candidates per DELTA row
};

}  // namespace

struct sparkalog_executor {
    std::vector<u32> relations;
    std::vector<sparkalog_rule_plan> rules;
    std::vector<TargetRT> targets;
    std::vector<IndexCache> index;
    DevArray counters;     // device: tile counters, error word
    DevArray status;       // shared look-back words for join / anti-join
    u64* host_counts = nullptr;  // pinned mirror of `counts`
    DevArray rule_delta;         // device: DELTA row count of each rule's delta input
    u64* host_rule_delta = nullptr;
    size_t counts_words = 0;
    u32 epoch = 1;
    SortScratch index_sort;
    DevArray index_pairs[2];
    u32* host_active = nullptr;  // pinned: radix pass activity per target (8 words each)
    // Batched runs: per-segment (instance) activity, see sparkalog_executor_track_segments.
    u32 seg_shift = 0;
    u32 seg_count = 0;
    u64 rounds_total = 0;        // rounds executed over the executor's lifetime (all run/step calls)
    DevArray seg_seen;           // u32[seg_count]
    DevArray seg_new;            // u64[seg_count]

    // Profiling: CUDA events around each kernel class on the executor's stream.
    struct Timing {
        int cls;
        cudaEvent_t a, b;
        double bytes;
        u64 launches;
    };
    bool profiling = false;
    bool fused_enabled = true;
    cudaStream_t stream = nullptr;  // the store's stream at compile time (syncs of executor-only state)
    bool device_loop = true;       // tail rounds as a CUDA graph WHILE loop (see spk_loop.cuh)
    u64 loop_launches = 0;         // graph launches of the device loop
    u64 loop_rounds = 0;           // rounds applied by the device loop
    sparkalog_tuning tuning = default_tuning();
    // `counters` holds, in this order: the per-round tile counters
    // (kCounterWords u32), the per-target counts (counts_words u64), the error
    // word and the fused kernels' fallback flags, then a few words that the
    // per-round clearing leaves alone. One memset clears a round's words and
    // one copy brings its counts and error bits to the host.
    u32* tile_counters() const { return counters.as<u32>(); }
    u64* count_words() const { return reinterpret_cast<u64*>(counters.as<u32>() + kCounterWords); }
    u32* err_words() const { return counters.as<u32>() + kCounterWords + 2 * counts_words; }
    bool member_enabled = false;  // anti-join through FULL's hash set (opt-in)
    std::vector<sparkalog_round_trace> trace;  // per-round operator cardinalities
    std::vector<cudaEvent_t> free_events;
    std::vector<Timing> timings;
    sparkalog_kernel_stats stats{};

    cudaEvent_t take_event() {
        if (free_events.empty()) {
            cudaEvent_t e = nullptr;
            cudaEventCreate(&e);
            return e;
        }
        cudaEvent_t e = free_events.back();
        free_events.pop_back();
        return e;
    }
    // Opens a timed section; returns its index or -1 when not profiling.
    int begin(int cls, cudaStream_t s) {
        if (!profiling) return -1;
        Timing t{cls, take_event(), take_event(), 0.0, 0};
        cudaEventRecord(t.a, s);
        timings.push_back(t);
        return static_cast<int>(timings.size()) - 1;
    }
    void end(int idx, cudaStream_t s, double bytes, u64 launches) {
        if (idx < 0) return;
        cudaEventRecord(timings[idx].b, s);
        timings[idx].bytes = bytes;
        timings[idx].launches = launches;
    }
    // Folds completed sections into the statistics (call after a stream sync).
    void collect() {
        for (auto& t : timings) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, t.a, t.b) == cudaSuccess) {
                stats.milliseconds[t.cls] += ms;
                stats.bytes[t.cls] += t.bytes;
                stats.launches[t.cls] += t.launches;
            }
            free_events.push_back(t.a);
            free_events.push_back(t.b);
        }
        timings.clear();
    }
};

namespace {

// Radix sort of *n_dev keys (or n_host_bound keys when n_dev is null) held in
// buffers a/b; n_host_bound sizes the grids and the look-back buffer. The
// sorted keys end in a or b as RadixPlan::final_sel says.
int radix_sort(u64* a, u64* b, const u64* n_dev, u64 n_host_bound, SortScratch& sc, sparkalog_executor* ex,
               u32* err, cudaStream_t s, int* hist_timing, int* pass_timing) {
    SPK_CUDA(sc.plan.ensure(sizeof(spk::RadixPlan), s), "cudaMallocAsync");
    SPK_CUDA(sc.status.ensure_zeroed(spk::radix_status_words(n_host_bound) * 8, s), "cudaMallocAsync");
    spk::RadixPlan* plan = sc.plan.as<spk::RadixPlan>();
    const int th = ex->begin(SPARKALOG_K_SORT_HIST, s);
    SPK_CUDA(cudaMemsetAsync(plan, 0, spk::kRadixPlanClearBytes, s), "cudaMemsetAsync");
    constexpr int kPasses = 8;
    {
        auto kernel = spk::radix_histogram<kThreads>;
        kernel<<<simple_grid(n_host_bound), kThreads, 0, s>>>(a, n_dev, n_host_bound, plan, 0, kPasses);
        SPK_CUDA(cudaGetLastError(), "radix_histogram");
    }
    spk::radix_plan<<<1, spk::kRadix, 0, s>>>(plan, n_dev, n_host_bound, kPasses);
    SPK_CUDA(cudaGetLastError(), "radix_plan");
    ex->end(th, s, 0.0, 2);
    ex->stats.total_launches += 2;
    const int tp = ex->begin(SPARKALOG_K_SORT_PASS, s);
    auto kernel = spk::radix_pass<kSortThreads, kSortItems>;
    const size_t tiles = (n_host_bound + kSortTile - 1) / kSortTile;
    const unsigned grid = grid_for(reinterpret_cast<const void*>(kernel), kSortThreads, std::max<size_t>(tiles, 1));
    for (int p = 0; p < kPasses; ++p) {
        kernel<<<grid, kSortThreads, 0, s>>>(a, b, plan, plan, p, p * spk::kRadixBits, sc.status.as<u64>(), nullptr,
                                             ex->epoch++, err);
        SPK_CUDA(cudaGetLastError(), "radix_pass");
    }
    ex->end(tp, s, 0.0, 0);
    ex->stats.total_launches += kPasses;
    if (hist_timing) *hist_timing = th;
    if (pass_timing) *pass_timing = tp;
    return 0;
}


size_t target_count_base(const sparkalog_executor* ex, size_t t) {
    // Layout per target: [rules + 1 join counts][newt count][distinct join rows]
    size_t base = 0;
    for (size_t i = 0; i < t; ++i) base += ex->targets[i].rules.size() + 3;
    return base;
}

constexpr int kFusedThreads = 256;
// 40 KB of shared memory per tile: five CTAs fit an SM (the kernel waits on
// its barriers and shared-memory dependencies, so resident tiles are what
// hides that latency; tiles of 1920 / 1024, four per SM, took 7.0 ms of the
// fixpoint over the 16.7M-node ER graph against 4.5 ms).
constexpr int kFusedCap = 1280;    // join output rows per fused tile (shared memory)
constexpr int kFusedRowCap = 768;  // DELTA rows per fused tile
constexpr size_t kFusedFlagBase = 8;      // fallback flags live at err + 8 + target
constexpr size_t kFusedMaxTargets = 48;
constexpr size_t kMaxTraceRounds = 1u << 20;
constexpr size_t kMemberErrOffset = kFusedFlagBase + kFusedMaxTargets + 4;  // from the error word

// The fused round applies to a target with one rule whose join output starts
// with DELTA's first column (then the join output is sorted by it) while
// DELTA is sorted.
bool fused_eligible(const sparkalog_executor* ex, sparkalog_store* st, size_t ti) {
    const TargetRT& t = ex->targets[ti];
    if (!ex->fused_enabled || t.force_generic || t.rules.size() != 1 || ti >= kFusedMaxTargets) return false;
    const sparkalog_rule_plan& p = ex->rules[t.rules[0]];
    if (p.proj_side[0] != 0 || p.proj_col[0] != 0) return false;
    const RelState* d = st->find(p.delta_input);
    return d && d->delta_sorted;
}

int launch_fused(const spk::FusedRoundArgs& a, size_t tiles, cudaStream_t s) {
    auto kernel = spk::fused_join_distinct_kernel<kFusedThreads, kFusedCap, kFusedRowCap>;
    constexpr size_t smem = spk::FusedLayout<kFusedThreads, kFusedCap, kFusedRowCap>::kBytes;
    // The shared-memory opt-in is per device.
    static std::atomic<u64> configured{0};
    int device = 0;
    SPK_CUDA(cudaGetDevice(&device), "cudaGetDevice");
    const u64 bit = 1ull << (device & 63);
    if (!(configured.load() & bit)) {
        SPK_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
                 "cudaFuncSetAttribute");
        configured.fetch_or(bit);
    }
    const unsigned grid = spk::persistent_grid(reinterpret_cast<const void*>(kernel), kFusedThreads, smem,
                                               std::max<size_t>(tiles, 1));
    kernel<<<grid, kFusedThreads, smem, s>>>(a);
    SPK_CUDA(cudaGetLastError(), "fused_join_distinct_kernel");
    return 0;
}

}  // namespace

// Scratch of store-level operations: a rule-less executor supplies the sort
// scratch, look-back epochs and launch counting; the rest are buffers.
struct StoreOps {
    sparkalog_executor ex;
    DevArray a, b;       // sort ping-pong of operation inputs
    DevArray counts;     // u64 words
    DevArray counters;   // u32 tile counters; error bits at word 32
    DevArray status;     // look-back words
    DevArray bitmap;     // dead-segment bitmap
    u64* host = nullptr; // pinned 256 bytes
};

namespace {

// The store's operation scratch, created on first use; null (with the error
// recorded) when its buffers cannot be allocated.
StoreOps* store_ops(sparkalog_store* st) {
    if (!st->ops) {
        auto* ops = new StoreOps();
        cudaStream_t s = st->stream;
        cudaError_t e = ops->counts.ensure(256, s);
        if (e == cudaSuccess) e = ops->counters.ensure(256, s);
        if (e == cudaSuccess) e = cudaMemsetAsync(ops->counters.ptr, 0, 256, s);
        if (e == cudaSuccess) e = pinned_get(reinterpret_cast<void**>(&ops->host), 256);
        if (e != cudaSuccess) {
            ops->counts.release(s);
            ops->counters.release(s);
            delete ops;
            fail(static_cast<int>(e), std::string("store scratch: ") + cudaGetErrorString(e));
            return nullptr;
        }
        st->ops = ops;
    }
    StoreOps& ops = *st->ops;
    if (ops.ex.epoch > spk::kEpochMask - 4096) {
        cudaStream_t s = st->stream;
        if (ops.status.ptr) cudaMemsetAsync(ops.status.ptr, 0, ops.status.bytes, s);
        if (ops.ex.index_sort.status.ptr) cudaMemsetAsync(ops.ex.index_sort.status.ptr, 0, ops.ex.index_sort.status.bytes, s);
        ops.ex.epoch = 1;
    }
    return &ops;
}

void release_store_ops(sparkalog_store* st) {
    if (!st->ops) return;
    cudaStream_t s = st->stream;
    StoreOps& o = *st->ops;
    for (DevArray* d : {&o.a, &o.b, &o.counts, &o.counters, &o.status, &o.bitmap, &o.ex.index_sort.plan,
                        &o.ex.index_sort.status})
        d->release(s);
    cudaStreamSynchronize(s);
    pinned_put(o.host, 256);
    delete st->ops;
    st->ops = nullptr;
}

int refresh_directories(sparkalog_store* st, RelState& r, cudaStream_t s, u64* launches);

// out = sort + unique of the n packed rows in ops.a, minus every FULL level of
// `right` (the anti-join of GeneralCpu negation, and the novelty check of an
// append). ops.b is the sort's second buffer.
int sorted_difference(sparkalog_store* st, u64 n, RelState& right, DevArray& out, u64* out_n) {
    cudaStream_t s = st->stream;
    StoreOps* ops_ptr = store_ops(st);
    if (!ops_ptr) return static_cast<int>(cudaErrorMemoryAllocation);
    StoreOps& ops = *ops_ptr;
    u32* err = ops.counters.as<u32>() + 32;
    SPK_CUDA(ops.b.ensure(n * 8, s), "cudaMallocAsync");
    SPK_CUDA(out.ensure(std::max<u64>(n, 1) * 8, s), "cudaMallocAsync");
    int rc = radix_sort(ops.a.as<u64>(), ops.b.as<u64>(), nullptr, n, ops.ex.index_sort, &ops.ex, err, s, nullptr,
                        nullptr);
    if (rc) return rc;
    rc = refresh_directories(st, right, s, nullptr);
    if (rc) return rc;
    spk::Levels lv{};
    lv.n = 0;
    for (int l = 0; l < spk::kMaxLevels; ++l) {
        if (right.level_n[l] == 0) continue;
        lv.keys[lv.n] = right.level[l].as<u64>();
        lv.count[lv.n] = right.level_n[l];
        lv.dir[lv.n] = right.dir[l].as<u32>();
        lv.shift[lv.n] = right.dir_shift[l];
        lv.buckets[lv.n] = right.dir_buckets[l];
        ++lv.n;
    }
    SPK_CUDA(ops.status.ensure_zeroed(((n + kSetTile - 1) / kSetTile + 1) * 8, s), "cudaMallocAsync");
    SPK_CUDA(cudaMemsetAsync(ops.counters.ptr, 0, 32 * 4, s), "cudaMemsetAsync");
    ops.host[0] = n;
    u64* nptr = ops.counts.as<u64>() + 1;
    SPK_CUDA(cudaMemcpyAsync(nptr, ops.host, 8, cudaMemcpyHostToDevice, s), "cudaMemcpyAsync");
    auto kernel = spk::anti_join_levels_kernel<kThreads, kSetItems, kLevelStage>;
    const size_t tiles = (n + kSetTile - 1) / kSetTile;
    kernel<<<grid_for(reinterpret_cast<const void*>(kernel), kThreads, tiles), kThreads, 0, s>>>(
        ops.a.as<u64>(), ops.b.as<u64>(), &ops.ex.index_sort.plan.as<spk::RadixPlan>()->final_sel, nptr, lv,
        out.as<u64>(), ops.counts.as<u64>(), ops.status.as<u64>(), ops.counters.as<u32>(), ops.ex.epoch++, err,
        nullptr);
    SPK_CUDA(cudaGetLastError(), "anti_join_levels_kernel");
    SPK_CUDA(cudaMemcpyAsync(ops.host, ops.counts.ptr, 8, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync");
    SPK_CUDA(cudaMemcpyAsync(ops.host + 1, err, 4, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync");
    SPK_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    const u32 bits = static_cast<u32>(ops.host[1] & 0xffffffffu);
    if (bits) return fail(SPARKALOG_E_DEVICE_FAULT, "device error bits " + std::to_string(bits));
    *out_n = ops.host[0];
    return 0;
}

// Sorts and deduplicates DELTA of r in place (it may have been inserted unsorted).
int sort_unique_delta(sparkalog_store* st, RelState& r) {
    cudaStream_t s = st->stream;
    StoreOps* ops_ptr = store_ops(st);
    if (!ops_ptr) return static_cast<int>(cudaErrorMemoryAllocation);
    StoreOps& ops = *ops_ptr;
    if (r.delta_n) {
        SPK_CUDA(ops.a.ensure(r.delta_n * 8, s), "cudaMallocAsync");
        SPK_CUDA(cudaMemcpyAsync(ops.a.ptr, r.delta.ptr, r.delta_n * 8, cudaMemcpyDeviceToDevice, s),
                 "cudaMemcpyAsync");
        RelState none;
        u64 n = 0;
        int rc = sorted_difference(st, r.delta_n, none, r.newt, &n);
        if (rc) return rc;
        swap_arrays(r.delta, r.newt);
        r.delta_n = n;
    }
    r.delta_sorted = true;
    return 0;
}

int build_index_impl(sparkalog_executor* ex, sparkalog_store* st, IndexCache& ic, u32 relation, u32 column);

// Builds a rule's right index; its kernels are counted as launches but kept
// out of the per-class timings of the round's operators.
int build_index(sparkalog_executor* ex, sparkalog_store* st, IndexCache& ic, u32 relation, u32 column) {
    const bool profiling = ex->profiling;
    ex->profiling = false;
    const int rc = build_index_impl(ex, st, ic, relation, column);
    ex->profiling = profiling;
    return rc;
}

int build_index_impl(sparkalog_executor* ex, sparkalog_store* st, IndexCache& ic, u32 relation, u32 column) {
    cudaStream_t s = st->stream;
    ic.key_class = ic.key_word = nullptr;
    RelState* r = st->find(relation);
    if (!r) return fail(SPARKALOG_E_MISSING, "relation " + std::to_string(relation) + " is not registered");
    if (r->recursive) {
        int rc = materialize(st, *r);
        if (rc) return rc;
    }
    const u64 n = r->level_n[0];
    const u64* rows = r->level[0].as<u64>();
    const u64* sorted_keys = rows;
    ic.identity = (column == 0 && r->sorted);
    if (!ic.identity) {
        // Index rows ordered by (key value, row id): sort (key << 32 | row).
        SPK_CUDA(ex->index_pairs[0].ensure(std::max<u64>(n, 1) * 8, s), "cudaMallocAsync");
        SPK_CUDA(ex->index_pairs[1].ensure(std::max<u64>(n, 1) * 8, s), "cudaMallocAsync");
        if (n) {
            spk::key_row_pairs_kernel<<<simple_grid(n), 256, 0, s>>>(rows, n, column, ex->index_pairs[0].as<u64>());
            SPK_CUDA(cudaGetLastError(), "key_row_pairs_kernel");
            u32* err = ex->err_words();
            int rc = radix_sort(ex->index_pairs[0].as<u64>(), ex->index_pairs[1].as<u64>(), nullptr, n, ex->index_sort,
                                ex, err, s, nullptr, nullptr);
            if (rc) return rc;
            // Bring the sorted pairs to buffer 0 regardless of pass parity.
            u32 sel = 0;
            SPK_CUDA(cudaMemcpyAsync(&sel, &ex->index_sort.plan.as<spk::RadixPlan>()->final_sel, 4,
                                     cudaMemcpyDeviceToHost, s),
                     "cudaMemcpyAsync");
            SPK_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
            if (sel) swap_arrays(ex->index_pairs[0], ex->index_pairs[1]);
        }
        sorted_keys = ex->index_pairs[0].as<u64>();
        SPK_CUDA(ic.rows.ensure(std::max<u64>(n, 1) * 4, s), "cudaMallocAsync");
        if (n) {
            spk::low_words_kernel<<<simple_grid(n), 256, 0, s>>>(sorted_keys, n, ic.rows.as<u32>());
            SPK_CUDA(cudaGetLastError(), "low_words_kernel");
        }
    }
    // Key domain: [0, max key]. The keys are the high words of sorted_keys.
    u64 last = 0;
    if (n) {
        SPK_CUDA(cudaMemcpyAsync(&last, sorted_keys + (n - 1), 8, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync");
        SPK_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    }
    ic.num_keys = n ? (last >> 32) + 1 : 0;
    u32* maxdeg = ex->err_words() + 1;
    SPK_CUDA(cudaMemsetAsync(maxdeg, 0, 4, s), "cudaMemsetAsync");
    ic.bucketed = n && ic.num_keys > std::max<u64>(4 * n, u64(1) << 22);
    if (ic.bucketed) {
        // ~8 keys per bucket.
        const u64 max_key = last >> 32;
        const int key_bits = 64 - __builtin_clzll(max_key | 1);
        const int target_bits = 64 - __builtin_clzll(std::max<u64>(n / 8, 1));
        ic.bucket_shift = static_cast<u32>(std::max(0, key_bits - target_bits));
        ic.buckets = (max_key >> ic.bucket_shift) + 1;
        SPK_CUDA(ic.keys32.ensure(n * 4, s), "cudaMallocAsync");
        SPK_CUDA(ic.bucket_dir.ensure((ic.buckets + 1) * 4, s), "cudaMallocAsync");
        spk::high_words_kernel<<<simple_grid(n), 256, 0, s>>>(sorted_keys, n, ic.keys32.as<u32>());
        SPK_CUDA(cudaGetLastError(), "high_words_kernel");
        spk::key_directory_kernel<<<simple_grid(ic.buckets + 1), 256, 0, s>>>(ic.keys32.as<u32>(), n, ic.bucket_shift,
                                                                             ic.buckets, ic.bucket_dir.as<u32>());
        SPK_CUDA(cudaGetLastError(), "key_directory_kernel");
        spk::max_run_kernel<<<simple_grid(n), 256, 0, s>>>(sorted_keys, n, maxdeg);
        SPK_CUDA(cudaGetLastError(), "max_run_kernel");
        ex->stats.total_launches += ic.identity ? 3 : 5;
        ic.values_ptr = nullptr;
    } else {
        // An identity index keeps the second column right after the offsets.
        const u64 off_bytes = spk::align_up((ic.num_keys + 1) * 4, 256);
        SPK_CUDA(ic.offsets.ensure(off_bytes + (ic.identity ? n * 4 : 0), s), "cudaMallocAsync");
        ic.values_ptr = ic.identity ? reinterpret_cast<u32*>(static_cast<char*>(ic.offsets.ptr) + off_bytes) : nullptr;
    }
    if (ic.bucketed) {
    } else if (n) {
        spk::dense_offsets_kernel<<<simple_grid(n), 256, 0, s>>>(sorted_keys, n, ic.num_keys, ic.offsets.as<u32>(),
                                                                 maxdeg);
        SPK_CUDA(cudaGetLastError(), "dense_offsets_kernel");
        ex->stats.total_launches += ic.identity ? 1 : 3;
        if (ic.identity) {
            spk::low_words_kernel<<<simple_grid(n), 256, 0, s>>>(rows, n, ic.values_ptr);
            SPK_CUDA(cudaGetLastError(), "low_words_kernel");
            ex->stats.total_launches += 1;
        }
        if (ic.identity && ex->tuning.compact_index) {
            const u64 class_bytes = spk::align_up((ic.num_keys + 7) / 8 * 4, 256);
            SPK_CUDA(ic.compact.ensure(class_bytes + ic.num_keys * 4, s), "cudaMallocAsync");
            ic.key_class = ic.compact.as<u32>();
            ic.key_word = reinterpret_cast<u32*>(static_cast<char*>(ic.compact.ptr) + class_bytes);
            spk::compact_index_kernel<<<simple_grid(ic.num_keys), 256, 0, s>>>(ic.offsets.as<u32>(), ic.values_ptr,
                                                                              ic.num_keys, ic.key_class, ic.key_word);
            SPK_CUDA(cudaGetLastError(), "compact_index_kernel");
            ex->stats.total_launches += 1;
        }
    } else {
        SPK_CUDA(cudaMemsetAsync(ic.offsets.ptr, 0, 4, s), "cudaMemsetAsync");
    }
    u32 md = 0;
    SPK_CUDA(cudaMemcpyAsync(&md, maxdeg, 4, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync");
    SPK_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    ic.max_degree = md;
    ic.valid = true;
    ic.relation = relation;
    ic.version = r->version;
    ic.column = column;
    return 0;
}

bool valid_cols(const u32 c[2]) { return c[0] <= 1 && c[1] <= 1; }

// Cascade after TAIL grew: a level merges down once it outgrows
// 1/level_ratio of the next (an empty next level just takes it).
int cascade_levels(sparkalog_executor* ex, sparkalog_store* st, RelState& tr) {
    cudaStream_t s = st->stream;
    const int tail = static_cast<int>(ex->tuning.levels) - 1;
    for (int l = tail; l > 0; --l) {
        if (tr.level_n[l] == 0 || tr.level_n[l] * ex->tuning.level_ratio <= tr.level_n[l - 1]) continue;
        if (tr.level_n[l - 1] == 0) {
            swap_arrays(tr.level[l - 1], tr.level[l]);
            swap_arrays(tr.dir[l - 1], tr.dir[l]);
            std::swap(tr.dir_valid[l - 1], tr.dir_valid[l]);
            std::swap(tr.dir_shift[l - 1], tr.dir_shift[l]);
            std::swap(tr.dir_buckets[l - 1], tr.dir_buckets[l]);
            tr.level_n[l - 1] = tr.level_n[l];
            tr.level_n[l] = 0;
            continue;
        }
        const u64 mn = tr.level_n[l - 1] + tr.level_n[l];
        u64 launched = 0;
        int rc = merge_buffers(st, tr, l - 1, mn, s);
        if (rc) return rc;
        const int tm = ex->begin(SPARKALOG_K_MERGE, s);
        rc = merge_into_level(st, tr, l - 1, tr.level[l - 1].as<u64>(), tr.level_n[l - 1], tr.level[l].as<u64>(),
                              tr.level_n[l], s, &launched);
        if (rc) return rc;
        ex->end(tm, s, 16.0 * static_cast<double>(mn), launched);
        ex->stats.total_launches += launched;
        tr.level_n[l] = 0;
        tr.dir_valid[l] = false;
    }
    return 0;
}

// ---------------------------------------------------------------------------
// Device-driven tail rounds (spk_loop.cuh): a CUDA graph whose WHILE node runs
// one round per iteration until the round-end kernel stops it. The graph and
// the small buffers it names (descriptor, counters, look-back words, trace)
// are cached per (device, stream, shape), so executors created one after the
// other (a fresh executor per fixpoint) reuse one instantiated graph. Streams
// of different host threads get different entries.
// ---------------------------------------------------------------------------
constexpr u64 kLoopTraceCap = 4096;     // rounds one graph launch may apply
constexpr int kLoopWordBytes = 256;     // counts[4] u64 | tile counters u32[16] | error bits u32[16]
constexpr u32 kLoopMinFusedRows = 64;

struct LoopGraph {
    int device = -1;
    cudaStream_t stream = nullptr;
    u64 bound = 0;
    u32 lanes = 0, items = 0;
    bool segments = false;
    bool bloom = false;                   // the anti-join probes FULL's Bloom filter
    std::mutex use;
    spk::LoopDesc* desc = nullptr;        // device
    spk::LoopDesc* host_desc = nullptr;   // pinned
    u64* words = nullptr;                 // device
    u64* fused_status = nullptr;
    u64* anti_status = nullptr;
    size_t fused_status_words = 0, anti_status_words = 0;
    spk::LoopTrace* trace = nullptr;      // device, kLoopTraceCap records
    spk::LoopTrace* host_trace = nullptr; // pinned
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

std::mutex g_loop_mu;
std::vector<LoopGraph*> g_loops;  // kept for the life of the process

struct LoopGrids {
    unsigned fused, anti, anti_bloom, merge, split, segment;
};

// Shared-memory opt-ins and persistent grid sizes of the loop's kernels.
template <int G, int ITEMS>
cudaError_t prepare_loop_kernels(const LoopGraph& g, LoopGrids* grids) {
    using FL = spk::FusedLayout<kFusedThreads, kFusedCap, kFusedRowCap>;
    using ML = spk::MergeBulkLayout<kThreads, ITEMS>;
    auto fused = spk::loop_fused_kernel<kFusedThreads, kFusedCap, kFusedRowCap>;
    auto anti = spk::loop_anti_join_kernel<kWideThreads, G>;
    auto merge = spk::loop_merge_kernel<kThreads, ITEMS>;
    cudaError_t e = cudaFuncSetAttribute(fused, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(FL::kBytes));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(merge, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(ML::kBytes));
    if (e != cudaSuccess) return e;
    const u64 fused_tiles = (g.bound + kLoopMinFusedRows - 1) / kLoopMinFusedRows;
    const u64 anti_tiles = (g.bound + (kWideThreads / G) - 1) / (kWideThreads / G);
    grids->fused = spk::persistent_grid(reinterpret_cast<const void*>(fused), kFusedThreads, FL::kBytes, fused_tiles);
    grids->anti = spk::persistent_grid(reinterpret_cast<const void*>(anti), kWideThreads, 0, anti_tiles);
    {
        auto bloom = spk::loop_anti_join_bloom_kernel<kSparseThreads, kSparseItems>;
        grids->anti_bloom = spk::persistent_grid(reinterpret_cast<const void*>(bloom), kSparseThreads, 0,
                                                 (g.bound + kSparseTile - 1) / kSparseTile);
    }
    grids->merge = spk::persistent_grid(reinterpret_cast<const void*>(merge), kThreads, ML::kBytes, ~0ull >> 1);
    grids->split = static_cast<unsigned>(spk::device_sm_count()) * 4;
    grids->segment = simple_grid(g.bound);
    return cudaGetLastError();
}

// Appends a node to the round body, depending on the previous one.
cudaError_t add_kernel_node(cudaGraph_t body, cudaGraphNode_t* last, const void* func, unsigned grid,
                            unsigned threads, size_t smem, void** args) {
    cudaKernelNodeParams kp{};
    kp.func = const_cast<void*>(func);
    kp.gridDim = dim3(grid);
    kp.blockDim = dim3(threads);
    kp.sharedMemBytes = static_cast<unsigned>(smem);
    kp.kernelParams = args;
    cudaGraphNode_t node;
    cudaError_t e = cudaGraphAddKernelNode(&node, body, *last ? last : nullptr, *last ? 1 : 0, &kp);
    if (e == cudaSuccess) *last = node;
    return e;
}

cudaError_t add_memset_node(cudaGraph_t body, cudaGraphNode_t* last, void* dst, size_t bytes) {
    cudaMemsetParams mp{};
    mp.dst = dst;
    mp.value = 0;
    mp.elementSize = 4;
    mp.width = bytes / 4;
    mp.height = 1;
    mp.pitch = 0;
    cudaGraphNode_t node;
    cudaError_t e = cudaGraphAddMemsetNode(&node, body, *last ? last : nullptr, *last ? 1 : 0, &mp);
    if (e == cudaSuccess) *last = node;
    return e;
}

// The graph: a WHILE node (condition 1 at every launch) whose body is one
// round, built node by node (no stream capture, so other host threads'
// device-wide calls cannot interfere with its construction).
template <int G, int ITEMS>
cudaError_t build_loop_graph_shape(LoopGraph& g) {
    using FL = spk::FusedLayout<kFusedThreads, kFusedCap, kFusedRowCap>;
    using ML = spk::MergeBulkLayout<kThreads, ITEMS>;
    LoopGrids gr{};
    cudaError_t e = prepare_loop_kernels<G, ITEMS>(g, &gr);
    if (e != cudaSuccess) return e;
    e = cudaGraphCreate(&g.graph, 0);
    if (e != cudaSuccess) return e;
    cudaGraphConditionalHandle handle;
    e = cudaGraphConditionalHandleCreate(&handle, g.graph, 1, cudaGraphCondAssignDefault);
    if (e != cudaSuccess) return e;
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = handle;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    e = cudaGraphAddNode(&node, g.graph, nullptr, 0, &cp);
    if (e != cudaSuccess) return e;
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    spk::LoopDesc* desc = g.desc;
    u32 tile = static_cast<u32>(kThreads * ITEMS);
    void* desc_args[] = {&desc};
    void* split_args[] = {&desc, &tile};
    void* end_args[] = {&desc, &handle};
    cudaGraphNode_t last = nullptr;
    if (e == cudaSuccess) e = add_memset_node(body, &last, g.words, kLoopWordBytes);
    if (e == cudaSuccess) e = add_memset_node(body, &last, g.fused_status, g.fused_status_words * 8);
    if (e == cudaSuccess) e = add_memset_node(body, &last, g.anti_status, g.anti_status_words * 8);
    if (e == cudaSuccess)
        e = add_kernel_node(body, &last,
                            reinterpret_cast<const void*>(spk::loop_fused_kernel<kFusedThreads, kFusedCap, kFusedRowCap>),
                            gr.fused, kFusedThreads, FL::kBytes, desc_args);
    if (e == cudaSuccess && g.bloom)
        e = add_kernel_node(body, &last,
                            reinterpret_cast<const void*>(spk::loop_anti_join_bloom_kernel<kSparseThreads, kSparseItems>),
                            gr.anti_bloom, kSparseThreads, 0, desc_args);
    else if (e == cudaSuccess)
        e = add_kernel_node(body, &last, reinterpret_cast<const void*>(spk::loop_anti_join_kernel<kWideThreads, G>),
                            gr.anti, kWideThreads, 0, desc_args);
    if (e == cudaSuccess)
        e = add_kernel_node(body, &last, reinterpret_cast<const void*>(spk::loop_split_kernel), gr.split, 256, 0,
                            split_args);
    if (e == cudaSuccess)
        e = add_kernel_node(body, &last, reinterpret_cast<const void*>(spk::loop_merge_kernel<kThreads, ITEMS>),
                            gr.merge, kThreads, ML::kBytes, desc_args);
    if (e == cudaSuccess)
        e = add_kernel_node(body, &last, reinterpret_cast<const void*>(spk::loop_round_end_kernel), 1, 32, 0,
                            end_args);
    if (e == cudaSuccess && g.segments)
        e = add_kernel_node(body, &last, reinterpret_cast<const void*>(spk::loop_segment_kernel), gr.segment, 256, 0,
                            desc_args);
    if (e != cudaSuccess) return e;
    return cudaGraphInstantiate(&g.exec, g.graph, 0);
}

template <int G>
cudaError_t build_loop_graph_lanes(LoopGraph& g) {
    if (g.items == 7) return build_loop_graph_shape<G, 7>(g);
    if (g.items == 15) return build_loop_graph_shape<G, 15>(g);
    return build_loop_graph_shape<G, 11>(g);
}

cudaError_t build_loop_graph(LoopGraph& g) {
    if (g.lanes == 4) return build_loop_graph_lanes<4>(g);
    if (g.lanes == 16) return build_loop_graph_lanes<16>(g);
    return build_loop_graph_lanes<8>(g);
}

// The cached graph for this shape (built on first use).
cudaError_t loop_graph(cudaStream_t s, u64 bound, u32 lanes, u32 items, bool segments, bool bloom,
                       LoopGraph** out) {
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(g_loop_mu);
    for (LoopGraph* g : g_loops) {
        if (g->device == device && g->stream == s && g->bound == bound && g->lanes == lanes && g->items == items &&
            g->segments == segments && g->bloom == bloom) {
            *out = g;
            return cudaSuccess;
        }
    }
    auto* g = new LoopGraph();
    g->device = device;
    g->stream = s;
    g->bound = bound;
    g->lanes = lanes;
    g->items = items;
    g->segments = segments;
    g->bloom = bloom;
    g->fused_status_words = (bound + kLoopMinFusedRows - 1) / kLoopMinFusedRows + 2;
    g->anti_status_words = (bound + (kWideThreads / lanes) - 1) / (kWideThreads / lanes) + 2;
    e = cudaMalloc(reinterpret_cast<void**>(&g->desc), sizeof(spk::LoopDesc));
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&g->words), kLoopWordBytes);
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&g->fused_status), g->fused_status_words * 8);
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&g->anti_status), g->anti_status_words * 8);
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&g->trace), kLoopTraceCap * sizeof(spk::LoopTrace));
    if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void**>(&g->host_desc), sizeof(spk::LoopDesc));
    if (e == cudaSuccess)
        e = cudaMallocHost(reinterpret_cast<void**>(&g->host_trace), kLoopTraceCap * sizeof(spk::LoopTrace));
    if (e == cudaSuccess) e = build_loop_graph(*g);
    // A half-built entry is dropped (not freed: freeing device memory here
    // would synchronise the device) and never reused.
    if (e != cudaSuccess) return e;
    g_loops.push_back(g);
    *out = g;
    return cudaSuccess;
}

// Runs device-driven rounds of a single-rule, fused-eligible target while
// its rounds stay small; returns the rounds applied through *applied and
// their new rows through *new_rows. On return the host state (levels,
// DELTA, trace) matches what the same rounds run by the host would leave.
int run_device_loop(sparkalog_executor* ex, sparkalog_store* st, size_t ti, u64 max_rounds, u64* applied,
                    u64* new_rows) {
    cudaStream_t s = st->stream;
    *applied = 0;
    *new_rows = 0;
    TargetRT& t = ex->targets[ti];
    const size_t k = t.rules[0];
    const sparkalog_rule_plan& p = ex->rules[k];
    RelState& tr = *st->find(t.id);
    RelState& right = *st->find(p.right_input);
    IndexCache& ic = ex->index[k];
    const int tail = static_cast<int>(ex->tuning.levels) - 1;
    const u64 bound = ex->tuning.group_candidates;
    const u64 max_degree = std::max<u64>(ic.max_degree, 1);
    const u64 ratio = ex->tuning.level_ratio;
    const u64 upper_n = tr.level_n[tail - 1];
    const u64 tail_max = upper_n / ratio + bound + 1;

    // Capacities for every round the loop may run (it stops before a round
    // that could exceed them).
    if (t.j_cap < bound) {
        const u64 cap = bound + bound / 4;
        SPK_CUDA(t.j_a.ensure(cap * 8, s), "cudaMallocAsync");
        SPK_CUDA(t.j_b.ensure(cap * 8, s), "cudaMallocAsync");
        t.j_cap = cap;
    }
    SPK_CUDA(tr.delta.ensure(bound * 8, s, tr.delta_n * 8), "cudaMallocAsync");
    SPK_CUDA(tr.newt.ensure(bound * 8, s), "cudaMallocAsync");
    SPK_CUDA(tr.level[tail].ensure(tail_max * 8, s, tr.level_n[tail] * 8), "cudaMallocAsync");
    SPK_CUDA(tr.spare.ensure(tail_max * 8, s), "cudaMallocAsync");
    SPK_CUDA(st->merge_splits.ensure((tail_max / (kThreads * 7) + 4) * 8, s), "cudaMallocAsync");
    // TAIL's directory in the loop's fixed shape (sized for its largest TAIL).
    u32 shift;
    u64 buckets;
    directory_shape(st, tail_max, &shift, &buckets);
    if (!tr.dir_valid[tail] || tr.dir_shift[tail] != shift || tr.dir_buckets[tail] != buckets) {
        SPK_CUDA(tr.dir[tail].ensure((buckets + 1) * 4, s), "cudaMallocAsync");
        if (tr.level_n[tail]) {
            spk::level_directory_kernel<<<simple_grid(buckets + 1), 256, 0, s>>>(
                tr.level[tail].as<u64>(), tr.level_n[tail], shift, buckets, tr.dir[tail].as<u32>());
            SPK_CUDA(cudaGetLastError(), "level_directory_kernel");
            ex->stats.total_launches += 1;
        }
        tr.dir_shift[tail] = shift;
        tr.dir_buckets[tail] = buckets;
        tr.dir_valid[tail] = true;
    }
    int rc = refresh_directories(st, tr, s, nullptr);
    if (rc) return rc;
    const bool use_bloom = ex->tuning.bloom_bits != 0;
    if (use_bloom) {
        // Sized for the largest FULL the loop may reach (it stops at a cascade).
        if (!tr.bloom_valid || tr.full_rows() + upper_n / ratio + bound > tr.bloom_capacity) {
            rc = bloom_build(tr, ex->tuning.bloom_bits, s, nullptr);
            if (rc) return rc;
        }
    } else {
        tr.bloom_valid = false;
    }

    LoopGraph* g = nullptr;
    SPK_CUDA(loop_graph(s, bound, ex->tuning.group_lanes, st->merge_items, ex->seg_count != 0, use_bloom, &g),
             "device loop graph");
    std::lock_guard<std::mutex> use(g->use);
    spk::LoopDesc& d = *g->host_desc;
    d = spk::LoopDesc{};
    u64* counts = g->words;
    u32* counters = reinterpret_cast<u32*>(g->words + 4);
    u32* err = reinterpret_cast<u32*>(g->words + 12);
    spk::FusedRoundArgs& a = d.fused;
    a.delta = tr.delta.as<u64>();
    a.delta_rows = 0;
    a.delta_rows_ptr = &g->desc->delta_n;
    a.rows_per_tile = std::max(t.fused_rows, kLoopMinFusedRows);
    a.left_key = p.left_key;
    if (ic.bucketed) {
        a.bucket_dir = ic.bucket_dir.as<u32>();
        a.bucket_shift = ic.bucket_shift;
        a.buckets = ic.buckets;
        a.keys32 = ic.keys32.as<u32>();
    } else {
        a.dense_offsets = ic.offsets.as<u32>();
        a.dense_keys = ic.num_keys;
    }
    a.rows = ic.identity ? nullptr : ic.rows.as<u32>();
    a.right = right.level[0].as<u64>();
    a.v1_side = p.proj_side[1];
    a.v1_col = p.proj_col[1];
    a.right_values = (ic.identity && !ic.bucketed && a.v1_side == 1 && a.v1_col == 1 && ic.num_keys)
                         ? ic.values_ptr : nullptr;
    a.key_class = (a.right_values && ex->tuning.compact_index) ? ic.key_class : nullptr;
    a.key_word = a.key_class ? ic.key_word : nullptr;
    a.v1_bits = static_cast<u32>(32 - __builtin_clz(st->max_value | 1));
    a.out = t.j_a.as<u64>();
    a.out_count = counts + 1;
    a.join_rows = reinterpret_cast<unsigned long long*>(counts);
    a.status = g->fused_status;
    a.tile_counter = counters;
    a.epoch = 1;
    a.err = err;
    a.fallback = err + 8;
    d.lv.n = tail + 1;
    u64 other = 0;
    for (int l = 0; l <= tail; ++l) {
        d.lv.keys[l] = tr.level[l].as<u64>();
        d.lv.count[l] = tr.level_n[l];
        d.lv.dir[l] = tr.dir[l].as<u32>();
        d.lv.shift[l] = tr.dir_shift[l];
        // An empty level is never searched (every key falls past its buckets).
        d.lv.buckets[l] = tr.level_n[l] ? tr.dir_buckets[l] : 0;
        if (l != tail) other += tr.level_n[l];
    }
    for (int l = tail + 1; l < spk::kMaxLevels; ++l) other += tr.level_n[l];
    d.tail_slot = static_cast<u32>(tail);
    d.counts = counts;
    d.counters = counters;
    d.anti_status = g->anti_status;
    d.err = err;
    d.delta = tr.delta.as<u64>();
    d.newt = tr.newt.as<u64>();
    d.delta_n = tr.delta_n;
    d.tail = tr.level[tail].as<u64>();
    d.spare = tr.spare.as<u64>();
    d.tail_n = tr.level_n[tail];
    d.splits = st->merge_splits.as<u64>();
    d.md = spk::MergeDirectory{tr.dir[tail].as<u32>(), shift, buckets};
    d.bound = bound;
    d.max_degree = max_degree;
    d.upper_n = upper_n;
    d.ratio = ratio;
    d.other_rows = other;
    d.limit = std::min<u64>(max_rounds, kLoopTraceCap);
    d.rounds_total = ex->rounds_total;
    d.seg_shift = ex->seg_shift;
    d.seg_count = ex->seg_count;
    d.seg_seen = ex->seg_seen.as<u32>();
    d.seg_new = ex->seg_new.as<unsigned long long>();
    d.trace = g->trace;
    d.bloom = use_bloom ? bloom_of(tr) : spk::Bloom{nullptr, 0};
    SPK_CUDA(cudaMemcpyAsync(g->desc, &d, sizeof(d), cudaMemcpyHostToDevice, s), "cudaMemcpyAsync");
    SPK_CUDA(cudaGraphLaunch(g->exec, s), "cudaGraphLaunch");
    SPK_CUDA(cudaMemcpyAsync(&d, g->desc, sizeof(d), cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync");
    SPK_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    const u64 done = d.iterations;
    if (done) {
        SPK_CUDA(cudaMemcpyAsync(g->host_trace, g->trace, done * sizeof(spk::LoopTrace), cudaMemcpyDeviceToHost, s),
                 "cudaMemcpyAsync");
        SPK_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    }
    ex->loop_launches += 1;
    ex->loop_rounds += done;
    // The host state after the applied rounds.
    if (d.tail != tr.level[tail].as<u64>()) swap_arrays(tr.level[tail], tr.spare);
    tr.level_n[tail] = d.tail_n;
    if (d.delta != tr.delta.as<u64>()) swap_arrays(tr.delta, tr.newt);
    tr.delta_n = d.delta_n;
    tr.delta_sorted = true;
    tr.version += done;
    if (done) tr.member_valid = false;
    // A refused round's merge wrote the directory of rows that were not
    // applied: rebuild it from TAIL when next needed.
    if (d.stop == spk::kLoopRedo || d.stop == spk::kLoopFault || d.stop == spk::kLoopRowLimit)
        tr.dir_valid[tail] = false;
    for (u64 r = 0; r < done; ++r) {
        const spk::LoopTrace& lt = g->host_trace[r];
        sparkalog_round_trace rec{};
        rec.round = ex->rounds_total + r + 1;
        rec.delta_rows = lt.delta_rows;
        rec.join_rows = lt.join_rows;
        rec.unique_rows = lt.unique_rows;
        rec.new_rows = lt.new_rows;
        rec.full_rows = lt.full_rows;
        if (ex->trace.size() < kMaxTraceRounds) ex->trace.push_back(rec);
    }
    ex->rounds_total += done;
    ex->stats.rounds += done;
    ex->stats.total_launches += done * (ex->seg_count ? 6 : 5);
    *applied = done;
    *new_rows = d.total_new;
    if (d.stop == spk::kLoopFault) {
        u32* bits = reinterpret_cast<u32*>(ex->host_counts + ex->counts_words) + 31;
        SPK_CUDA(cudaMemcpyAsync(bits, err, 4, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync");
        SPK_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
        return fail(SPARKALOG_E_DEVICE_FAULT, "device error bits " + std::to_string(*bits) + " (device loop)");
    }
    if (d.stop == spk::kLoopCascade) return cascade_levels(ex, st, tr);
    return 0;
}

}  // namespace

extern "C" {

const char* sparkalog_last_error(void) { return g_last_error.c_str(); }

int sparkalog_reserve_device_memory(size_t bytes, void* stream) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int dev = 0;
    cudaMemPool_t pool;
    SPK_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
    SPK_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev), "cudaDeviceGetDefaultMemPool");
    uint64_t threshold = ~0ull;
    SPK_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold), "cudaMemPoolSetAttribute");
    if (bytes == 0) return 0;
    void* p = nullptr;
    SPK_CUDA(cudaMallocAsync(&p, bytes, s), "cudaMallocAsync");
    SPK_CUDA(cudaFreeAsync(p, s), "cudaFreeAsync");
    SPK_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    return 0;
}

// ---------------------------------------------------------------------------
// Value catalog on the device (ValueCatalog, crates/sparkalog-datalog/src/
// catalog.rs:98-127): see the interning kernels in spk_ingest.cuh.
// ---------------------------------------------------------------------------
struct sparkalog_catalog {
    cudaStream_t stream = nullptr;
    sparkalog_executor ex;          // radix-sort scratch and look-back epochs (no rules)
    DevArray keys, keys_spare;      // U32 values: (value << 32 | id), sorted by value
    DevArray dict;                  // id -> U32 value, or a String/Symbol's string index
    DevArray a, b, list_a, list_b;  // sort buffers
    DevArray staging, ids;          // host input / output staging, ids of a batch
    DevArray words;                 // u64 new-value count, then the u32 error word
    DevArray splits;                // merge diagonals
    u64 size = 0;                   // values (ids 0 .. size - 1)
    u64 u32_count = 0;              // U32 values (entries of `keys`)
    u64* host = nullptr;            // pinned 64 bytes
    // String and Symbol values (spk::StringTable), present once one is interned.
    DevArray kinds;                 // u32 per id: 0 U32, 1 String, 2 Symbol
    DevArray arena;                 // raw bytes of every string
    DevArray str_offset, str_length;
    DevArray skeys, sids, sidx;     // lookup index sorted by key
    DevArray skeys_spare, sids_spare, sidx_spare;
    u64 str_count = 0;
    u64 arena_used = 0;
    // Scratch of a mixed batch.
    DevArray tokens, v_keys, v_pos, v_sorted, v_pairs, v_pairs_b, g_head, g_id, g_si, g_new, joint, joint_b,
        str_src, nk, nid, nsi;
};

namespace {

// Radix-sorts n packed keys held in x (y is the other buffer); returns the one
// holding the sorted keys.
int catalog_sort(sparkalog_catalog* c, DevArray& x, DevArray& y, u64 n, u32* err, DevArray** sorted) {
    cudaStream_t s = c->stream;
    int rc = radix_sort(x.as<u64>(), y.as<u64>(), nullptr, n, c->ex.index_sort, &c->ex, err, s, nullptr, nullptr);
    if (rc) return rc;
    u32* sel = reinterpret_cast<u32*>(c->host + 4);
    SPK_CUDA(cudaMemcpyAsync(sel, &c->ex.index_sort.plan.as<spk::RadixPlan>()->final_sel, 4, cudaMemcpyDeviceToHost,
                             s),
             "cudaMemcpyAsync");
    SPK_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    *sorted = *sel ? &y : &x;
    return 0;
}

}  // namespace

namespace {

// Interns n tokens (spk_ingest.cuh: U32 values and String/Symbol spans of
// `text`, all on the device) in order, as ValueCatalog::intern applied to
// each in turn would (catalog.rs:108-117): ids[p] receives token p's id.
int catalog_intern_tokens(sparkalog_catalog* c, const u64* tokens, u64 n, const unsigned char* text, u64 text_bytes,
                          u32* ids) {
    cudaStream_t s = c->stream;
    if (n == 0) return 0;
    if (n > (1ull << 31)) return fail(SPARKALOG_E_TOO_MANY_ROWS, "more than 2^31 values in one batch");
    u32* err = reinterpret_cast<u32*>(c->words.as<u64>() + 1);
    auto* counts = reinterpret_cast<unsigned long long*>(c->words.as<u64>() + 2);  // [0] U32, [1] strings, [2] new
    SPK_CUDA(cudaMemsetAsync(c->words.ptr, 0, 64, s), "cudaMemsetAsync");
    SPK_CUDA(c->v_keys.ensure(n * 8, s), "cudaMallocAsync");      // U32 (value << 32 | pos)
    SPK_CUDA(c->a.ensure(n * 8, s), "cudaMallocAsync");           // string keys
    SPK_CUDA(c->v_pos.ensure(n * 4, s), "cudaMallocAsync");
    spk::classify_tokens_kernel<<<simple_grid(n), 256, 0, s>>>(tokens, n, text, c->v_keys.as<u64>(), counts,
                                                               c->a.as<u64>(), c->v_pos.as<u32>(), counts + 1);
    SPK_CUDA(cudaGetLastError(), "classify_tokens_kernel");
    SPK_CUDA(cudaMemcpyAsync(c->host, counts, 16, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync");
    SPK_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    const u64 nu = c->host[0], ns = c->host[1];

    // U32 values: the batch sorted by (value, position); heads the catalog lacks.
    DevArray* usorted = nullptr;
    u64 mu = 0;
    if (nu) {
        SPK_CUDA(c->b.ensure(nu * 8, s), "cudaMallocAsync");
        int rc = catalog_sort(c, c->v_keys, c->b, nu, err, &usorted);
        if (rc) return rc;
        // Keep the sorted U32 keys in v_keys: `b` is reused below.
        if (usorted == &c->b) swap_arrays(c->v_keys, c->b);
        usorted = &c->v_keys;
        SPK_CUDA(c->list_a.ensure(nu * 8, s), "cudaMallocAsync");
        spk::new_value_heads_kernel<<<simple_grid(nu), 256, 0, s>>>(usorted->as<u64>(), nu, c->keys.as<u64>(),
                                                                    c->u32_count, c->list_a.as<u64>(), counts + 2);
        SPK_CUDA(cudaGetLastError(), "new_value_heads_kernel");
        SPK_CUDA(cudaMemcpyAsync(c->host, counts + 2, 8, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync");
        SPK_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
        mu = c->host[0];
        SPK_CUDA(cudaMemsetAsync(counts + 2, 0, 8, s), "cudaMemsetAsync");
    }

    // Strings and Symbols: keys sorted, values grouped by key in position
    // order, heads looked up in the catalog.
    DevArray* ksorted = nullptr;
    DevArray* psorted = nullptr;
    u64 ms = 0;
    if (ns) {
        SPK_CUDA(c->v_sorted.ensure(ns * 8, s), "cudaMallocAsync");
        SPK_CUDA(cudaMemcpyAsync(c->v_sorted.ptr, c->a.ptr, ns * 8, cudaMemcpyDeviceToDevice, s), "cudaMemcpyAsync");
        SPK_CUDA(c->b.ensure(ns * 8, s), "cudaMallocAsync");
        int rc = catalog_sort(c, c->v_sorted, c->b, ns, err, &ksorted);
        if (rc) return rc;
        SPK_CUDA(c->v_pairs.ensure(ns * 8, s), "cudaMallocAsync");
        SPK_CUDA(c->v_pairs_b.ensure(ns * 8, s), "cudaMallocAsync");
        spk::group_pairs_kernel<<<simple_grid(ns), 256, 0, s>>>(c->a.as<u64>(), c->v_pos.as<u32>(), ns,
                                                                ksorted->as<u64>(), c->v_pairs.as<u64>());
        SPK_CUDA(cudaGetLastError(), "group_pairs_kernel");
        // The sorted keys must survive the next sort: keep them apart.
        if (ksorted == &c->b) swap_arrays(c->v_sorted, c->b);
        rc = catalog_sort(c, c->v_pairs, c->v_pairs_b, ns, err, &psorted);
        if (rc) return rc;
        for (DevArray* d : {&c->g_head, &c->g_id, &c->g_si, &c->g_new}) SPK_CUDA(d->ensure(ns * 4, s), "cudaMallocAsync");
        SPK_CUDA(cudaMemsetAsync(c->g_new.ptr, 0, ns * 4, s), "cudaMemsetAsync");
        SPK_CUDA(c->list_b.ensure(ns * 8, s), "cudaMallocAsync");
        spk::StringTable cat{c->arena.as<unsigned char>(), c->str_offset.as<u64>(), c->str_length.as<u32>(),
                             c->skeys.as<u64>(), c->sids.as<u32>(), c->sidx.as<u32>(), c->str_count};
        spk::string_heads_kernel<<<simple_grid(ns), 256, 0, s>>>(
            psorted->as<u64>(), ns, c->v_sorted.as<u64>(), tokens, text, cat, c->g_head.as<u32>(), c->g_id.as<u32>(),
            c->g_new.as<u32>(), c->list_b.as<u64>(), counts + 2, err);
        SPK_CUDA(cudaGetLastError(), "string_heads_kernel");
        spk::verify_groups_kernel<<<simple_grid(ns), 256, 0, s>>>(psorted->as<u64>(), ns, c->g_head.as<u32>(), tokens,
                                                                  text, err);
        SPK_CUDA(cudaGetLastError(), "verify_groups_kernel");
        SPK_CUDA(cudaMemcpyAsync(c->host, counts + 2, 8, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync");
        SPK_CUDA(cudaMemcpyAsync(c->host + 1, err, 4, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync");
        SPK_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
        ms = c->host[0];
        const u32 bits = static_cast<u32>(c->host[1] & 0xffffffffu);
        if (bits & spk::kErrHashCollision)
            return fail(SPARKALOG_E_DEVICE_FAULT, "two different values share a 62-bit value key");
        if (bits) return fail(SPARKALOG_E_DEVICE_FAULT, "device error bits " + std::to_string(bits));
    }
    const u64 m = mu + ms;
    if (c->size + m > kMaxRelationRows) return fail(SPARKALOG_E_TOO_MANY_ROWS, "more than 2^32 - 1 values");

    if (m) {
        // New values of both sorts, numbered together by first position.
        SPK_CUDA(c->joint.ensure(m * 8, s), "cudaMallocAsync");
        SPK_CUDA(c->joint_b.ensure(m * 8, s), "cudaMallocAsync");
        spk::joint_entries_kernel<<<simple_grid(m), 256, 0, s>>>(c->list_a.as<u64>(), mu, c->list_b.as<u64>(), ms,
                                                                 c->joint.as<u64>());
        SPK_CUDA(cudaGetLastError(), "joint_entries_kernel");
        DevArray* jsorted = nullptr;
        int rc = catalog_sort(c, c->joint, c->joint_b, m, err, &jsorted);
        if (rc) return rc;
        if (!c->kinds.ptr || c->kinds.bytes < (c->size + m) * 4) {
            const bool fresh = !c->kinds.ptr;
            SPK_CUDA(c->kinds.ensure((c->size + m) * 4, s, c->size * 4), "cudaMallocAsync");
            if (fresh && c->size) SPK_CUDA(cudaMemsetAsync(c->kinds.ptr, 0, c->size * 4, s), "cudaMemsetAsync");
        }
        SPK_CUDA(c->dict.ensure((c->size + m) * 4, s, c->size * 4), "cudaMallocAsync");
        SPK_CUDA(c->list_a.ensure(std::max<u64>(mu, 1) * 8, s), "cudaMallocAsync");  // new U32 pairs (in place)
        SPK_CUDA(c->str_offset.ensure((c->str_count + ms + 1) * 8, s, c->str_count * 8), "cudaMallocAsync");
        SPK_CUDA(c->str_length.ensure((c->str_count + ms + 1) * 4, s, c->str_count * 4), "cudaMallocAsync");
        SPK_CUDA(c->str_src.ensure((ms + 1) * 4, s), "cudaMallocAsync");
        // New strings are distinct spans of this text, so they fit in its size.
        SPK_CUDA(c->arena.ensure(c->arena_used + text_bytes + 16, s, c->arena_used), "cudaMallocAsync");
        c->host[0] = c->arena_used;
        SPK_CUDA(cudaMemcpyAsync(counts + 3, c->host, 8, cudaMemcpyHostToDevice, s), "cudaMemcpyAsync");
        SPK_CUDA(cudaMemsetAsync(counts, 0, 16, s), "cudaMemsetAsync");
        spk::assign_joint_ids_kernel<<<simple_grid(m), 256, 0, s>>>(
            jsorted->as<u64>(), m, c->size, c->str_count, c->dict.as<u32>(), c->kinds.as<u32>(), c->list_a.as<u64>(),
            counts, c->g_id.as<u32>(), c->g_si.as<u32>(), c->g_head.as<u32>(), tokens, c->str_offset.as<u64>(),
            c->str_length.as<u32>(), counts + 3, c->str_src.as<u32>(), counts + 1);
        SPK_CUDA(cudaGetLastError(), "assign_joint_ids_kernel");
        if (ms) {
            spk::copy_strings_kernel<<<simple_grid(ms * 32), 256, 0, s>>>(c->str_src.as<u32>(), ms, c->str_count,
                                                                          tokens, text, c->str_offset.as<u64>(),
                                                                          c->arena.as<unsigned char>());
            SPK_CUDA(cudaGetLastError(), "copy_strings_kernel");
            // The new keys (group order is key order) into the catalog's index.
            for (DevArray* d : {&c->nk}) SPK_CUDA(d->ensure(ms * 8, s), "cudaMallocAsync");
            for (DevArray* d : {&c->nid, &c->nsi}) SPK_CUDA(d->ensure(ms * 4, s), "cudaMallocAsync");
            SPK_CUDA(cudaMemsetAsync(counts + 2, 0, 8, s), "cudaMemsetAsync");
            spk::new_string_keys_kernel<<<simple_grid(ns), 256, 0, s>>>(
                c->v_sorted.as<u64>(), ns, c->g_id.as<u32>(), c->g_si.as<u32>(), c->g_new.as<u32>(), c->nk.as<u64>(),
                c->nid.as<u32>(), c->nsi.as<u32>(), counts + 2);
            SPK_CUDA(cudaGetLastError(), "new_string_keys_kernel");
            // Atomic order: sort the new keys, then fetch each one's payload
            // back through its group (the keys are distinct).
            DevArray* nsorted = nullptr;
            SPK_CUDA(c->b.ensure(ms * 8, s), "cudaMallocAsync");
            rc = catalog_sort(c, c->nk, c->b, ms, err, &nsorted);
            if (rc) return rc;
            DevArray& other = nsorted == &c->nk ? c->b : c->nk;
            SPK_CUDA(other.ensure(ms * 8, s), "cudaMallocAsync");
            spk::keyed_payload_kernel<<<simple_grid(ms), 256, 0, s>>>(nsorted->as<u64>(), ms, c->v_sorted.as<u64>(),
                                                                      ns, c->g_id.as<u32>(), c->g_si.as<u32>(),
                                                                      c->nid.as<u32>(), c->nsi.as<u32>());
            SPK_CUDA(cudaGetLastError(), "keyed_payload_kernel");
            const u64 total = c->str_count + ms;
            SPK_CUDA(c->skeys_spare.ensure(total * 8, s), "cudaMallocAsync");
            SPK_CUDA(c->sids_spare.ensure(total * 4, s), "cudaMallocAsync");
            SPK_CUDA(c->sidx_spare.ensure(total * 4, s), "cudaMallocAsync");
            spk::merge_keyed_kernel<<<simple_grid(total), 256, 0, s>>>(
                c->skeys.as<u64>(), c->sids.as<u32>(), c->sidx.as<u32>(), c->str_count, nsorted->as<u64>(),
                c->nid.as<u32>(), c->nsi.as<u32>(), ms, c->skeys_spare.as<u64>(), c->sids_spare.as<u32>(),
                c->sidx_spare.as<u32>());
            SPK_CUDA(cudaGetLastError(), "merge_keyed_kernel");
            swap_arrays(c->skeys, c->skeys_spare);
            swap_arrays(c->sids, c->sids_spare);
            swap_arrays(c->sidx, c->sidx_spare);
            SPK_CUDA(cudaMemcpyAsync(c->host, counts + 3, 8, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync");
            SPK_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
            c->arena_used = c->host[0];
        }
        if (mu) {
            // The new U32 values into the U32 index.
            DevArray* pairs_sorted = nullptr;
            SPK_CUDA(c->list_b.ensure(mu * 8, s), "cudaMallocAsync");
            rc = catalog_sort(c, c->list_a, c->list_b, mu, err, &pairs_sorted);
            if (rc) return rc;
            SPK_CUDA(c->keys_spare.ensure((c->u32_count + mu) * 8, s), "cudaMallocAsync");
            SPK_CUDA(launch_merge(c->keys.as<u64>(), c->u32_count, pairs_sorted->as<u64>(), mu,
                                  c->keys_spare.as<u64>(), c->splits, s, 11, err),
                     "merge_bulk_kernel");
            swap_arrays(c->keys, c->keys_spare);
        }
        c->size += m;
        c->u32_count += mu;
        c->str_count += ms;
    }
    // Every token's id.
    if (nu) {
        spk::lookup_ids_kernel<8><<<simple_grid((nu + 7) / 8), 256, 0, s>>>(usorted->as<u64>(), nu,
                                                                           c->keys.as<u64>(), c->u32_count, ids, err);
        SPK_CUDA(cudaGetLastError(), "lookup_ids_kernel");
    }
    if (ns) {
        spk::string_ids_kernel<<<simple_grid(ns), 256, 0, s>>>(psorted->as<u64>(), ns, c->g_id.as<u32>(), ids);
        SPK_CUDA(cudaGetLastError(), "string_ids_kernel");
    }
    SPK_CUDA(cudaMemcpyAsync(c->host + 1, err, 4, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync");
    SPK_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    const u32 bits = static_cast<u32>(c->host[1] & 0xffffffffu);
    if (bits) return fail(SPARKALOG_E_DEVICE_FAULT, "device error bits " + std::to_string(bits));
    return 0;
}

}  // namespace

int sparkalog_catalog_create(void* stream, sparkalog_catalog** out) {
    if (!out) return fail(SPARKALOG_E_INVALID_ARGUMENT, "null output");
    auto* c = new sparkalog_catalog();
    c->stream = static_cast<cudaStream_t>(stream);
    cudaError_t e = c->words.ensure(256, c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->words.ptr, 0, 256, c->stream);
    if (e == cudaSuccess) e = pinned_get(reinterpret_cast<void**>(&c->host), 64);
    if (e != cudaSuccess) {
        c->words.release(c->stream);
        delete c;
        return cuda_fail(e, "sparkalog_catalog_create");
    }
    *out = c;
    return 0;
}

void sparkalog_catalog_destroy(sparkalog_catalog* c) {
    if (!c) return;
    cudaStream_t s = c->stream;
    for (DevArray* d : {&c->keys, &c->keys_spare, &c->dict, &c->a, &c->b, &c->list_a, &c->list_b, &c->staging,
                        &c->ids, &c->words, &c->splits, &c->ex.index_sort.plan, &c->ex.index_sort.status, &c->kinds,
                        &c->arena, &c->str_offset, &c->str_length, &c->skeys, &c->sids, &c->sidx, &c->skeys_spare,
                        &c->sids_spare, &c->sidx_spare, &c->tokens, &c->v_keys, &c->v_pos, &c->v_sorted, &c->v_pairs,
                        &c->v_pairs_b, &c->g_head, &c->g_id, &c->g_si, &c->g_new, &c->joint, &c->joint_b, &c->str_src,
                        &c->nk, &c->nid, &c->nsi})
        d->release(s);
    cudaStreamSynchronize(s);
    pinned_put(c->host, 64);
    delete c;
}

int sparkalog_catalog_size(sparkalog_catalog* c, size_t* size) {
    if (!c || !size) return fail(SPARKALOG_E_INVALID_ARGUMENT, "null argument");
    *size = c->size;
    return 0;
}

int sparkalog_catalog_intern_u32(sparkalog_catalog* c, const u32* values, size_t n, int location, u32* ids,
                                 size_t* size) {
    if (!c || (n && (!values || !ids))) return fail(SPARKALOG_E_INVALID_ARGUMENT, "null argument");
    if (n > kMaxRelationRows) return fail(SPARKALOG_E_TOO_MANY_ROWS, "more than 2^32 - 1 values in one batch");
    cudaStream_t s = c->stream;
    if (n) {
        u32* err = reinterpret_cast<u32*>(c->words.as<u64>() + 1);
        unsigned long long* new_count = reinterpret_cast<unsigned long long*>(c->words.as<u64>());
        SPK_CUDA(cudaMemsetAsync(c->words.ptr, 0, 16, s), "cudaMemsetAsync");
        const u32* dvalues = values;
        if (location == SPARKALOG_HOST) {
            SPK_CUDA(c->staging.ensure(n * 4, s), "cudaMallocAsync");
            SPK_CUDA(cudaMemcpyAsync(c->staging.ptr, values, n * 4, cudaMemcpyHostToDevice, s), "cudaMemcpyAsync");
            dvalues = c->staging.as<u32>();
        }
        SPK_CUDA(c->a.ensure(n * 8, s), "cudaMallocAsync");
        SPK_CUDA(c->b.ensure(n * 8, s), "cudaMallocAsync");
        spk::value_positions_kernel<<<simple_grid(n), 256, 0, s>>>(dvalues, n, c->a.as<u64>());
        SPK_CUDA(cudaGetLastError(), "value_positions_kernel");
        DevArray* sorted = nullptr;
        int rc = catalog_sort(c, c->a, c->b, n, err, &sorted);
        if (rc) return rc;
        // Values the catalog lacks, with their first positions.
        SPK_CUDA(c->list_a.ensure(n * 8, s), "cudaMallocAsync");
        SPK_CUDA(c->list_b.ensure(n * 8, s), "cudaMallocAsync");
        spk::new_value_heads_kernel<<<simple_grid(n), 256, 0, s>>>(sorted->as<u64>(), n, c->keys.as<u64>(),
                                                                   c->u32_count, c->list_a.as<u64>(), new_count);
        SPK_CUDA(cudaGetLastError(), "new_value_heads_kernel");
        SPK_CUDA(cudaMemcpyAsync(c->host, new_count, 8, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync");
        SPK_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
        const u64 m = c->host[0];
        if (c->size + m > kMaxRelationRows) return fail(SPARKALOG_E_TOO_MANY_ROWS, "more than 2^32 - 1 values");
        if (m) {
            DevArray* by_position = nullptr;
            rc = catalog_sort(c, c->list_a, c->list_b, m, err, &by_position);
            if (rc) return rc;
            DevArray& pairs = by_position == &c->list_a ? c->list_b : c->list_a;
            SPK_CUDA(c->dict.ensure((c->size + m) * 4, s, c->size * 4), "cudaMallocAsync");
            if (c->kinds.ptr) {
                SPK_CUDA(c->kinds.ensure((c->size + m) * 4, s, c->size * 4), "cudaMallocAsync");
                SPK_CUDA(cudaMemsetAsync(c->kinds.as<u32>() + c->size, 0, m * 4, s), "cudaMemsetAsync");
            }
            spk::assign_new_ids_kernel<<<simple_grid(m), 256, 0, s>>>(by_position->as<u64>(), m, c->size,
                                                                      pairs.as<u64>(), c->dict.as<u32>());
            SPK_CUDA(cudaGetLastError(), "assign_new_ids_kernel");
            DevArray& other = &pairs == &c->list_a ? c->list_b : c->list_a;
            DevArray* sorted_pairs = nullptr;
            rc = catalog_sort(c, pairs, other, m, err, &sorted_pairs);
            if (rc) return rc;
            SPK_CUDA(c->keys_spare.ensure((c->u32_count + m) * 8, s), "cudaMallocAsync");
            SPK_CUDA(launch_merge(c->keys.as<u64>(), c->u32_count, sorted_pairs->as<u64>(), m,
                                  c->keys_spare.as<u64>(), c->splits, s, 11, err),
                     "merge_bulk_kernel");
            swap_arrays(c->keys, c->keys_spare);
            c->size += m;
            c->u32_count += m;
        }
        u32* dids = ids;
        if (location == SPARKALOG_HOST) {
            SPK_CUDA(c->ids.ensure(n * 4, s), "cudaMallocAsync");
            dids = c->ids.as<u32>();
        }
        spk::lookup_ids_kernel<8><<<simple_grid((n + 7) / 8), 256, 0, s>>>(sorted->as<u64>(), n, c->keys.as<u64>(),
                                                                          c->u32_count, dids, err);
        SPK_CUDA(cudaGetLastError(), "lookup_ids_kernel");
        if (location == SPARKALOG_HOST)
            SPK_CUDA(cudaMemcpyAsync(ids, dids, n * 4, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync");
        SPK_CUDA(cudaMemcpyAsync(c->host + 1, err, 4, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync");
        SPK_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
        const u32 bits = static_cast<u32>(c->host[1] & 0xffffffffu);
        if (bits) return fail(SPARKALOG_E_DEVICE_FAULT, "device error bits " + std::to_string(bits));
    }
    if (size) *size = c->size;
    return 0;
}

int sparkalog_catalog_decode_u32(sparkalog_catalog* c, const u32* ids, size_t n, int location, u32* values) {
    if (!c || (n && (!values || !ids))) return fail(SPARKALOG_E_INVALID_ARGUMENT, "null argument");
    if (n == 0) return 0;
    cudaStream_t s = c->stream;
    u32* err = reinterpret_cast<u32*>(c->words.as<u64>() + 1);
    SPK_CUDA(cudaMemsetAsync(err, 0, 4, s), "cudaMemsetAsync");
    const u32* dids = ids;
    u32* dvalues = values;
    if (location == SPARKALOG_HOST) {
        SPK_CUDA(c->staging.ensure(n * 4, s), "cudaMallocAsync");
        SPK_CUDA(c->ids.ensure(n * 4, s), "cudaMallocAsync");
        SPK_CUDA(cudaMemcpyAsync(c->staging.ptr, ids, n * 4, cudaMemcpyHostToDevice, s), "cudaMemcpyAsync");
        dids = c->staging.as<u32>();
        dvalues = c->ids.as<u32>();
    }
    spk::decode_ids_kernel<<<simple_grid(n), 256, 0, s>>>(dids, n, c->dict.as<u32>(),
                                                          c->kinds.ptr ? c->kinds.as<u32>() : nullptr, c->size,
                                                          dvalues, err);
    SPK_CUDA(cudaGetLastError(), "decode_ids_kernel");
    if (location == SPARKALOG_HOST)
        SPK_CUDA(cudaMemcpyAsync(values, dvalues, n * 4, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync");
    SPK_CUDA(cudaMemcpyAsync(c->host + 1, err, 4, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync");
    SPK_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    if (c->host[1] & 0xffffffffu) return fail(SPARKALOG_E_INVALID_ARGUMENT, "value id outside the catalog");
    return 0;
}

int sparkalog_store_create(void* stream, sparkalog_store** out) {
    if (!out) return fail(SPARKALOG_E_INVALID_ARGUMENT, "null output pointer");
    auto* st = new sparkalog_store();
    st->stream = static_cast<cudaStream_t>(stream);
    {
        // Relations grow and shrink every round through cudaMallocAsync; keep
        // freed blocks in the device's pool instead of returning them at
        // every synchronisation.
        int dev = 0;
        cudaMemPool_t pool;
        if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
            uint64_t threshold = ~0ull;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold);
        }
    }
    cudaError_t e = st->flags.ensure(256, st->stream);
    if (e == cudaSuccess) e = st->fault.ensure(256, st->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(st->fault.ptr, 0, 256, st->stream);
    if (e == cudaSuccess) e = pinned_get(reinterpret_cast<void**>(&st->pinned), 256);
    if (e != cudaSuccess) {
        delete st;
        return cuda_fail(e, "sparkalog_store_create");
    }
    *out = st;
    return 0;
}

void sparkalog_store_destroy(sparkalog_store* st) {
    if (!st) return;
    cudaStream_t s = st->stream;
    for (auto& kv : st->relations) {
        for (auto& l : kv.second.level) l.release(s);
        for (auto& d : kv.second.dir) d.release(s);
        kv.second.bloom.release(s);
        kv.second.spare.release(s);
        kv.second.delta.release(s);
        kv.second.newt.release(s);
        kv.second.member.release(s);
        kv.second.member_flag.release(s);
    }
    st->scratch_u32[0].release(s);
    st->scratch_u32[1].release(s);
    st->flags.release(s);
    st->fault.release(s);
    st->merge_splits.release(s);
    release_store_ops(st);
    cudaStreamSynchronize(s);
    pinned_put(st->pinned, 256);
    delete st;
}

int sparkalog_store_insert_static(sparkalog_store* st, u32 id, const u32* first, const u32* second, size_t rows,
                                  int location) {
    if (!st) return fail(SPARKALOG_E_INVALID_ARGUMENT, "null store");
    if (st->find(id)) return fail(SPARKALOG_E_DUPLICATE, "relation " + std::to_string(id) + " is already registered");
    if (rows > kMaxRelationRows) return fail(SPARKALOG_E_TOO_MANY_ROWS, "too many rows for u32 row ids");
    RelState r;
    int rc = pack_columns(st, first, second, rows, location, r.level[0], &r.sorted, &r.has_dups);
    if (rc) return rc;
    r.level_n[0] = rows;
    st->relations[id] = std::move(r);
    return 0;
}

int sparkalog_store_insert_recursive(sparkalog_store* st, u32 id, const u32* full_first, const u32* full_second,
                                     size_t full_rows, const u32* delta_first, const u32* delta_second,
                                     size_t delta_rows, int location) {
    if (!st) return fail(SPARKALOG_E_INVALID_ARGUMENT, "null store");
    if (st->find(id)) return fail(SPARKALOG_E_DUPLICATE, "relation " + std::to_string(id) + " is already registered");
    if (full_rows > kMaxRelationRows || delta_rows > kMaxRelationRows)
        return fail(SPARKALOG_E_TOO_MANY_ROWS, "too many rows for u32 row ids");
    RelState r;
    r.recursive = true;
    int rc = pack_columns(st, full_first, full_second, full_rows, location, r.level[0], &r.sorted, &r.has_dups);
    if (rc) return rc;
    r.level_n[0] = full_rows;
    if (delta_first == full_first && delta_second == full_second && delta_rows == full_rows) {
        // DELTA = FULL (how execute_binary seeds every recursive relation,
        // datalog/src/subset.rs:406-408): copy on the device, upload once.
        SPK_CUDA(r.delta.ensure(std::max<size_t>(full_rows, 1) * 8, st->stream), "cudaMallocAsync");
        if (full_rows)
            SPK_CUDA(cudaMemcpyAsync(r.delta.ptr, r.level[0].ptr, full_rows * 8, cudaMemcpyDeviceToDevice,
                                     st->stream),
                     "cudaMemcpyAsync");
        r.delta_sorted = r.sorted && !r.has_dups;
    } else {
        bool dsorted, ddups;
        rc = pack_columns(st, delta_first, delta_second, delta_rows, location, r.delta, &dsorted, &ddups);
        if (rc) return rc;
        r.delta_sorted = dsorted && !ddups;
    }
    r.delta_n = delta_rows;
    SPK_CUDA(r.newt.ensure(4096, st->stream), "cudaMallocAsync");
    st->relations[id] = std::move(r);
    return 0;
}

namespace {

// Host re-parse of the one line the device reported as failing, for the
// error's details (the same rules as spk::parse_line).
void describe_load_error(const unsigned char* line, u64 line_offset, u64 len, sparkalog_load_error* e) {
    auto space = [](unsigned char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r'; };
    u64 b = 0, end = len;
    while (b < end && space(line[b])) ++b;
    while (end > b && space(line[end - 1])) --end;
    u64 fb[3] = {0, 0, 0}, fe[3] = {0, 0, 0};
    int fields = 0;
    for (u64 p = b; p < end;) {
        while (p < end && space(line[p])) ++p;
        if (p == end) break;
        const u64 q = p;
        while (p < end && !space(line[p])) ++p;
        if (fields < 3) {
            fb[fields] = q;
            fe[fields] = p;
        }
        if (++fields > 2) break;
    }
    if (fields != 2) {
        e->kind = SPARKALOG_LOAD_INVALID_FIELD_COUNT;
        return;
    }
    for (int c = 0; c < 2; ++c) {
        u64 i = fb[c];
        if (i < fe[c] && line[i] == '+') ++i;
        bool ok = i < fe[c];
        u64 v = 0;
        for (; ok && i < fe[c]; ++i) {
            ok = line[i] >= '0' && line[i] <= '9';
            v = v * 10 + (line[i] - '0');
            ok = ok && v <= 0xffffffffull;
        }
        if (!ok) {
            e->kind = SPARKALOG_LOAD_INVALID_U32;
            e->column = static_cast<u32>(c + 1);
            e->field_offset = line_offset + fb[c];
            e->field_length = fe[c] - fb[c];
            return;
        }
    }
}

// parse_record (crates/sparkalog-datalog/src/ingest.rs:43-120) on the one
// failing line of a delimited text (without the '\r' before its '\n'), for
// the details: the first syntax error with its 1-based byte column, else a
// row that does not hold two values, else its first value that is not a u32.
void describe_delimited_error(const unsigned char* t, u64 offset, u64 len, unsigned char delim,
                              sparkalog_load_error* e) {
    u64 pos = 0;
    u32 fields = 0;
    bool bad = false;
    u32 bad_column = 0;
    u64 bad_begin = 0, bad_len = 0;
    for (;;) {
        const u32 column = static_cast<u32>(pos + 1);
        if (pos < len && t[pos] == '"') {
            ++pos;
            bool closed = false;
            while (pos < len) {
                if (t[pos] == '"') {
                    if (pos + 1 < len && t[pos + 1] == '"') {
                        pos += 2;
                    } else {
                        ++pos;
                        closed = true;
                        break;
                    }
                } else {
                    ++pos;
                }
            }
            if (!closed) {
                e->kind = SPARKALOG_LOAD_UNTERMINATED_QUOTE;
                e->column = column;
                return;
            }
            if (!bad) {
                bad = true;
                bad_column = column;
                bad_begin = column - 1;
                bad_len = pos - bad_begin;
            }
            if (pos < len && t[pos] != delim) {
                e->kind = SPARKALOG_LOAD_EXPECTED_DELIMITER;
                e->column = static_cast<u32>(pos + 1);
                return;
            }
        } else {
            const u64 start = pos;
            while (pos < len && t[pos] != delim) ++pos;
            u64 fb = start, fe = pos;
            spk::unicode_trim(t, &fb, &fe);
            if (fb == fe) {
                e->kind = SPARKALOG_LOAD_EMPTY_FIELD;
                e->column = column;
                return;
            }
            u32 v = 0;
            if (!bad && !spk::parse_u32_field(t + fb, fe - fb, &v)) {
                bad = true;
                bad_column = column;
                bad_begin = fb;
                bad_len = fe - fb;
            }
        }
        ++fields;
        if (pos == len) break;
        ++pos;
        if (pos == len) {
            e->kind = SPARKALOG_LOAD_TRAILING_DELIMITER;
            e->column = static_cast<u32>(pos);
            return;
        }
    }
    if (fields != 2) {
        e->kind = SPARKALOG_LOAD_ARITY;
        e->column = fields;
        return;
    }
    if (bad) {
        e->kind = SPARKALOG_LOAD_NOT_U32;
        e->column = bad_column;
        e->field_offset = offset + bad_begin;
        e->field_length = bad_len;
    }
}

const char* delimited_message(int kind) {
    switch (kind) {
    case SPARKALOG_LOAD_UNTERMINATED_QUOTE: return "unterminated quoted field";
    case SPARKALOG_LOAD_EXPECTED_DELIMITER: return "expected delimiter after quoted field";
    case SPARKALOG_LOAD_EMPTY_FIELD: return "empty fields are not values";
    case SPARKALOG_LOAD_TRAILING_DELIMITER: return "record ends with an empty field";
    case SPARKALOG_LOAD_ARITY: return "the row does not hold two values";
    default: return "a value is not a u32 (this entry point loads u32 relations)";
    }
}

// A text format for load_text_u32: load_binary_u32's whitespace-separated
// pairs, or a delimited text (load_delimited) whose values are all u32.
struct TextFormat {
    bool delimited = false;
    unsigned char delim = ',';
    bool header = false;
};

int load_text_u32(sparkalog_store* st, u32 id, const char* text, size_t bytes, int location, int recursive,
                  size_t* rows, sparkalog_load_error* error, const TextFormat& fmt);

}  // namespace

int sparkalog_store_load_binary_u32(sparkalog_store* st, u32 id, const char* text, size_t bytes, int location,
                                    int recursive, size_t* rows, sparkalog_load_error* error) {
    return load_text_u32(st, id, text, bytes, location, recursive, rows, error, TextFormat{});
}

int sparkalog_store_load_delimited_u32(sparkalog_store* st, u32 id, const char* text, size_t bytes, int location,
                                       unsigned char delimiter, int has_header, int recursive, size_t* rows,
                                       sparkalog_load_error* error) {
    // parse_delimited_parallel refuses whitespace delimiters other than tab (ingest.rs:24-30).
    if (delimiter == ' ' || delimiter == '\n' || delimiter == '\f' || delimiter == '\r')
        return fail(SPARKALOG_E_INVALID_ARGUMENT, "delimiter must be a visible ASCII byte or tab");
    TextFormat fmt;
    fmt.delimited = true;
    fmt.delim = delimiter;
    fmt.header = has_header != 0;
    return load_text_u32(st, id, text, bytes, location, recursive, rows, error, fmt);
}

namespace {

int load_text_u32(sparkalog_store* st, u32 id, const char* text, size_t bytes, int location, int recursive,
                  size_t* rows, sparkalog_load_error* error, const TextFormat& fmt) {
    if (!st || !rows || (bytes && !text)) return fail(SPARKALOG_E_INVALID_ARGUMENT, "null argument");
    if (st->find(id)) return fail(SPARKALOG_E_DUPLICATE, "relation " + std::to_string(id) + " is already registered");
    if (error) *error = sparkalog_load_error{};
    *rows = 0;
    cudaStream_t s = st->stream;
    StoreOps* ops_ptr = store_ops(st);
    if (!ops_ptr) return static_cast<int>(cudaErrorMemoryAllocation);
    StoreOps& ops = *ops_ptr;
    u32* err = ops.counters.as<u32>() + 32;
    // The text on the device (ops.b holds it for a host text).
    const unsigned char* dtext = reinterpret_cast<const unsigned char*>(text);
    if (location == SPARKALOG_HOST && bytes) {
        SPK_CUDA(ops.b.ensure(bytes, s), "cudaMallocAsync");
        SPK_CUDA(cudaMemcpyAsync(ops.b.ptr, text, bytes, cudaMemcpyHostToDevice, s), "cudaMemcpyAsync");
        dtext = ops.b.as<unsigned char>();
    }
    // Pass 0: count '\n' to size the line ends; pass 1: their positions.
    unsigned long long* dcount = reinterpret_cast<unsigned long long*>(ops.counts.as<u64>());
    SPK_CUDA(cudaMemsetAsync(ops.counts.ptr, 0, 64, s), "cudaMemsetAsync");
    if (bytes) {
        spk::count_newlines_kernel<<<simple_grid(bytes), 256, 0, s>>>(dtext, bytes, dcount);
        SPK_CUDA(cudaGetLastError(), "count_newlines_kernel");
    }
    SPK_CUDA(cudaMemcpyAsync(ops.host, dcount, 8, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync");
    SPK_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    const u64 newlines = ops.host[0];
    unsigned char last = 0;
    if (bytes) {
        if (location == SPARKALOG_HOST) {
            last = static_cast<unsigned char>(text[bytes - 1]);
        } else {
            SPK_CUDA(cudaMemcpyAsync(&last, dtext + bytes - 1, 1, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync");
            SPK_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
        }
    }
    const u64 lines = newlines + ((bytes && last != '\n') ? 1 : 0);
    constexpr int kByteItems = 16, kLineItems = 8;
    const u64 byte_tiles = (bytes + kThreads * kByteItems - 1) / (kThreads * kByteItems);
    const u64 line_tiles = (lines + kSetTile - 1) / kSetTile;
    SPK_CUDA(ops.a.ensure(std::max<u64>(newlines, 1) * 8, s), "cudaMallocAsync");
    SPK_CUDA(ops.status.ensure_zeroed((std::max(byte_tiles, line_tiles) + 1) * 8, s), "cudaMallocAsync");
    SPK_CUDA(st->scratch_u32[0].ensure(std::max<u64>(lines, 1) * 4, s), "cudaMallocAsync");
    SPK_CUDA(st->scratch_u32[1].ensure(std::max<u64>(lines, 1) * 4, s), "cudaMallocAsync");
    SPK_CUDA(cudaMemsetAsync(ops.counters.ptr, 0, 33 * 4, s), "cudaMemsetAsync");  // tile counters + error word
    SPK_CUDA(cudaMemsetAsync(ops.counts.as<u64>() + 2, 0xff, 16, s), "cudaMemsetAsync");
    u64* ends_n = ops.counts.as<u64>() + 1;
    unsigned long long* first_error = reinterpret_cast<unsigned long long*>(ops.counts.as<u64>() + 2);
    u64* out_n = ops.counts.as<u64>() + 4;
    {
        auto kernel = spk::line_ends_kernel<kThreads, kByteItems>;
        kernel<<<grid_for(reinterpret_cast<const void*>(kernel), kThreads, std::max<u64>(byte_tiles, 1)), kThreads, 0,
                 s>>>(dtext, bytes, ops.a.as<u64>(), ends_n, ops.status.as<u64>(), ops.counters.as<u32>(),
                      ops.ex.epoch++, err);
        SPK_CUDA(cudaGetLastError(), "line_ends_kernel");
    }
    auto parse = [&](auto parser) -> int {
        auto kernel = spk::parse_lines_kernel<kThreads, kLineItems, decltype(parser)>;
        kernel<<<grid_for(reinterpret_cast<const void*>(kernel), kThreads, std::max<u64>(line_tiles, 1)), kThreads, 0,
                 s>>>(dtext, bytes, ops.a.as<u64>(), ends_n, lines, parser, st->scratch_u32[0].as<u32>(),
                      st->scratch_u32[1].as<u32>(), out_n, first_error, ops.status.as<u64>(),
                      ops.counters.as<u32>() + 1, ops.ex.epoch++, err);
        SPK_CUDA(cudaGetLastError(), "parse_lines_kernel");
        return 0;
    };
    {
        const int rc = fmt.delimited ? parse(spk::DelimitedLineParser{fmt.delim, fmt.header})
                                     : parse(spk::BinaryLineParser{});
        if (rc) return rc;
    }
    SPK_CUDA(cudaMemcpyAsync(ops.host, ops.counts.as<u64>() + 2, 24, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync");
    SPK_CUDA(cudaMemcpyAsync(ops.host + 3, err, 4, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync");
    SPK_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    const u64 field_error = ops.host[0], lfs_line = ops.host[1], parsed = ops.host[2];
    const u32 bits = static_cast<u32>(ops.host[3] & 0xffffffffu);
    if (bits) return fail(SPARKALOG_E_DEVICE_FAULT, "device error bits " + std::to_string(bits));
    // The bytes of line `index` (without its '\n'), copied to the host.
    auto line_bytes = [&](u64 index, u64* offset, std::vector<unsigned char>* out) -> int {
        u64 bounds[2] = {0, bytes};
        if (index > 0)
            SPK_CUDA(cudaMemcpyAsync(&bounds[0], ops.a.as<u64>() + index - 1, 8, cudaMemcpyDeviceToHost, s),
                     "cudaMemcpyAsync");
        if (index < newlines)
            SPK_CUDA(cudaMemcpyAsync(&bounds[1], ops.a.as<u64>() + index, 8, cudaMemcpyDeviceToHost, s),
                     "cudaMemcpyAsync");
        SPK_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
        if (index > 0) bounds[0] += 1;
        out->resize(bounds[1] - bounds[0]);
        if (!out->empty())
            SPK_CUDA(cudaMemcpy(out->data(), dtext + bounds[0], out->size(), cudaMemcpyDefault), "cudaMemcpy");
        *offset = bounds[0];
        return 0;
    };
    if (fmt.delimited && (field_error != spk::kNoLine || lfs_line != spk::kNoLine)) {
        // A syntax error anywhere comes first (parse_delimited_parallel
        // fails before any row is inserted); then the first row that is not
        // two u32 values.
        const u64 index = field_error != spk::kNoLine ? field_error : lfs_line;
        u64 offset = 0;
        std::vector<unsigned char> line;
        int rc = line_bytes(index, &offset, &line);
        if (rc) return rc;
        if (index < newlines && !line.empty() && line.back() == '\r') line.pop_back();
        sparkalog_load_error e{};
        e.line = index + 1;
        describe_delimited_error(line.data(), offset, line.size(), fmt.delim, &e);
        if (error) *error = e;
        return fail(SPARKALOG_E_LOAD, "line " + std::to_string(e.line) + ", column " + std::to_string(e.column) +
                                          ": " + delimited_message(e.kind));
    }
    if (lfs_line != spk::kNoLine || field_error != spk::kNoLine) {
        sparkalog_load_error e{};
        if (lfs_line != spk::kNoLine) {
            // count_rows (io.rs:92-105) meets the pointer header before any field is parsed.
            e.kind = SPARKALOG_LOAD_GIT_LFS_POINTER;
            e.line = lfs_line + 1;
        } else {
            // The failing line's bytes, re-read on the host for the details.
            u64 offset = 0;
            std::vector<unsigned char> line;
            int rc = line_bytes(field_error, &offset, &line);
            if (rc) return rc;
            e.line = field_error + 1;
            describe_load_error(line.data(), offset, line.size(), &e);
        }
        if (error) *error = e;
        return fail(SPARKALOG_E_LOAD, e.kind == SPARKALOG_LOAD_GIT_LFS_POINTER
                                          ? "the text is a Git LFS pointer, not materialized graph data"
                                          : "line " + std::to_string(e.line) +
                                                (e.kind == SPARKALOG_LOAD_INVALID_FIELD_COUNT
                                                     ? " does not contain exactly two fields"
                                                     : ", column " + std::to_string(e.column) + " is not a u32"));
    }
    if (parsed > kMaxRelationRows) return fail(SPARKALOG_E_TOO_MANY_ROWS, "too many rows for u32 row ids");
    *rows = parsed;
    const u32* c0 = st->scratch_u32[0].as<u32>();
    const u32* c1 = st->scratch_u32[1].as<u32>();
    return recursive ? sparkalog_store_insert_recursive(st, id, c0, c1, parsed, c0, c1, parsed, SPARKALOG_DEVICE)
                     : sparkalog_store_insert_static(st, id, c0, c1, parsed, SPARKALOG_DEVICE);
}

}  // namespace

int sparkalog_store_load_delimited_values(sparkalog_store* st, sparkalog_catalog* c, u32 id, const char* text,
                                          size_t bytes, int location, unsigned char delimiter, int has_header,
                                          int recursive, size_t* rows, sparkalog_load_error* error) {
    if (!st || !c || !rows || (bytes && !text)) return fail(SPARKALOG_E_INVALID_ARGUMENT, "null argument");
    // parse_delimited_parallel refuses whitespace delimiters other than tab (ingest.rs:24-30).
    if (delimiter == ' ' || delimiter == '\n' || delimiter == '\f' || delimiter == '\r')
        return fail(SPARKALOG_E_INVALID_ARGUMENT, "delimiter must be a visible ASCII byte or tab");
    if (st->find(id)) return fail(SPARKALOG_E_DUPLICATE, "relation " + std::to_string(id) + " is already registered");
    if (error) *error = sparkalog_load_error{};
    *rows = 0;
    cudaStream_t s = st->stream;
    StoreOps* ops_ptr = store_ops(st);
    if (!ops_ptr) return static_cast<int>(cudaErrorMemoryAllocation);
    StoreOps& ops = *ops_ptr;
    u32* err = ops.counters.as<u32>() + 32;
    const unsigned char* dtext = reinterpret_cast<const unsigned char*>(text);
    if (location == SPARKALOG_HOST && bytes) {
        SPK_CUDA(c->staging.ensure(bytes + 16, s), "cudaMallocAsync");
        SPK_CUDA(cudaMemcpyAsync(c->staging.ptr, text, bytes, cudaMemcpyHostToDevice, s), "cudaMemcpyAsync");
        dtext = c->staging.as<unsigned char>();
    }
    unsigned long long* dcount = reinterpret_cast<unsigned long long*>(ops.counts.as<u64>());
    SPK_CUDA(cudaMemsetAsync(ops.counts.ptr, 0, 64, s), "cudaMemsetAsync");
    if (bytes) {
        spk::count_newlines_kernel<<<simple_grid(bytes), 256, 0, s>>>(dtext, bytes, dcount);
        SPK_CUDA(cudaGetLastError(), "count_newlines_kernel");
    }
    SPK_CUDA(cudaMemcpyAsync(ops.host, dcount, 8, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync");
    SPK_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    const u64 newlines = ops.host[0];
    unsigned char last = 0;
    if (bytes) {
        SPK_CUDA(cudaMemcpyAsync(&last, dtext + bytes - 1, 1, cudaMemcpyDefault, s), "cudaMemcpyAsync");
        SPK_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    }
    const u64 lines = newlines + ((bytes && last != '\n') ? 1 : 0);
    constexpr int kByteItems = 16, kLineItems = 8;
    const u64 byte_tiles = (bytes + kThreads * kByteItems - 1) / (kThreads * kByteItems);
    const u64 line_tiles = (lines + kThreads * kLineItems - 1) / (kThreads * kLineItems);
    SPK_CUDA(ops.a.ensure(std::max<u64>(newlines, 1) * 8, s), "cudaMallocAsync");
    SPK_CUDA(ops.status.ensure_zeroed((std::max(byte_tiles, line_tiles) + 1) * 8, s), "cudaMallocAsync");
    SPK_CUDA(c->tokens.ensure(std::max<u64>(lines, 1) * 16, s), "cudaMallocAsync");
    SPK_CUDA(cudaMemsetAsync(ops.counters.ptr, 0, 33 * 4, s), "cudaMemsetAsync");
    SPK_CUDA(cudaMemsetAsync(ops.counts.as<u64>() + 2, 0xff, 24, s), "cudaMemsetAsync");
    u64* ends_n = ops.counts.as<u64>() + 1;
    unsigned long long* first_error = reinterpret_cast<unsigned long long*>(ops.counts.as<u64>() + 2);
    u64* out_n = ops.counts.as<u64>() + 5;
    {
        auto kernel = spk::line_ends_kernel<kThreads, kByteItems>;
        kernel<<<grid_for(reinterpret_cast<const void*>(kernel), kThreads, std::max<u64>(byte_tiles, 1)), kThreads, 0,
                 s>>>(dtext, bytes, ops.a.as<u64>(), ends_n, ops.status.as<u64>(), ops.counters.as<u32>(),
                      ops.ex.epoch++, err);
        SPK_CUDA(cudaGetLastError(), "line_ends_kernel");
        auto parse = spk::parse_value_lines_kernel<kThreads, kLineItems>;
        parse<<<grid_for(reinterpret_cast<const void*>(parse), kThreads, std::max<u64>(line_tiles, 1)), kThreads, 0,
                s>>>(dtext, bytes, ops.a.as<u64>(), ends_n, lines, delimiter, has_header != 0, c->tokens.as<u64>(),
                     out_n, first_error, ops.status.as<u64>(), ops.counters.as<u32>() + 1, ops.ex.epoch++, err);
        SPK_CUDA(cudaGetLastError(), "parse_value_lines_kernel");
    }
    SPK_CUDA(cudaMemcpyAsync(ops.host, ops.counts.as<u64>() + 2, 32, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync");
    SPK_CUDA(cudaMemcpyAsync(ops.host + 4, err, 4, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync");
    SPK_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    const u64 syntax_line = ops.host[0], arity_line = ops.host[1], long_line = ops.host[2], parsed = ops.host[3];
    const u32 bits = static_cast<u32>(ops.host[4] & 0xffffffffu);
    if (bits) return fail(SPARKALOG_E_DEVICE_FAULT, "device error bits " + std::to_string(bits));
    if (syntax_line != spk::kNoLine || arity_line != spk::kNoLine) {
        // A syntax error anywhere comes first (parse_delimited_parallel fails
        // before any row is inserted); then the first row that does not hold
        // two values (Database::insert's arity check).
        const u64 index = syntax_line != spk::kNoLine ? syntax_line : arity_line;
        u64 bounds[2] = {0, bytes};
        if (index > 0)
            SPK_CUDA(cudaMemcpyAsync(&bounds[0], ops.a.as<u64>() + index - 1, 8, cudaMemcpyDeviceToHost, s),
                     "cudaMemcpyAsync");
        if (index < newlines)
            SPK_CUDA(cudaMemcpyAsync(&bounds[1], ops.a.as<u64>() + index, 8, cudaMemcpyDeviceToHost, s),
                     "cudaMemcpyAsync");
        SPK_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
        if (index > 0) bounds[0] += 1;
        std::vector<unsigned char> line(bounds[1] - bounds[0]);
        if (!line.empty())
            SPK_CUDA(cudaMemcpy(line.data(), dtext + bounds[0], line.size(), cudaMemcpyDefault), "cudaMemcpy");
        if (index < newlines && !line.empty() && line.back() == '\r') line.pop_back();
        sparkalog_load_error e{};
        e.line = index + 1;
        describe_delimited_error(line.data(), bounds[0], line.size(), delimiter, &e);
        if (e.kind == SPARKALOG_LOAD_NOT_U32) e.kind = SPARKALOG_LOAD_ARITY;  // any value kind is taken here
        if (error) *error = e;
        return fail(SPARKALOG_E_LOAD, "line " + std::to_string(e.line) + ", column " + std::to_string(e.column) +
                                          ": " + delimited_message(e.kind));
    }
    if (long_line != spk::kNoLine)
        return fail(SPARKALOG_E_INVALID_ARGUMENT, "line " + std::to_string(long_line + 1) +
                                                      " holds a value longer than 16 MiB - 1 bytes");
    if (parsed > kMaxRelationRows) return fail(SPARKALOG_E_TOO_MANY_ROWS, "too many rows for u32 row ids");
    // The catalog works on its own stream: wait for the parse first.
    if (c->stream != s) SPK_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    SPK_CUDA(c->ids.ensure(std::max<u64>(parsed, 1) * 8, c->stream), "cudaMallocAsync");
    int rc = catalog_intern_tokens(c, c->tokens.as<u64>(), parsed * 2, dtext, bytes, c->ids.as<u32>());
    if (rc) return rc;
    SPK_CUDA(st->scratch_u32[0].ensure(std::max<u64>(parsed, 1) * 4, c->stream), "cudaMallocAsync");
    SPK_CUDA(st->scratch_u32[1].ensure(std::max<u64>(parsed, 1) * 4, c->stream), "cudaMallocAsync");
    if (parsed) {
        spk::split_rows_kernel<<<simple_grid(parsed), 256, 0, c->stream>>>(
            c->ids.as<u32>(), parsed, st->scratch_u32[0].as<u32>(), st->scratch_u32[1].as<u32>());
        SPK_CUDA(cudaGetLastError(), "split_rows_kernel");
    }
    if (c->stream != s) SPK_CUDA(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
    *rows = parsed;
    const u32* c0 = st->scratch_u32[0].as<u32>();
    const u32* c1 = st->scratch_u32[1].as<u32>();
    return recursive ? sparkalog_store_insert_recursive(st, id, c0, c1, parsed, c0, c1, parsed, SPARKALOG_DEVICE)
                     : sparkalog_store_insert_static(st, id, c0, c1, parsed, SPARKALOG_DEVICE);
}

int sparkalog_catalog_export(sparkalog_catalog* c, uint32_t* kinds, uint32_t* numbers, uint64_t* offsets,
                             unsigned char* bytes, size_t bytes_capacity, size_t* bytes_used) {
    if (!c || !bytes_used) return fail(SPARKALOG_E_INVALID_ARGUMENT, "null argument");
    cudaStream_t s = c->stream;
    const u64 n = c->size;
    std::vector<u32> dict(n), kind(n, 0);
    std::vector<u64> soff(c->str_count);
    std::vector<u32> slen(c->str_count);
    std::vector<unsigned char> arena(c->arena_used);
    if (n) SPK_CUDA(cudaMemcpyAsync(dict.data(), c->dict.ptr, n * 4, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync");
    if (n && c->kinds.ptr)
        SPK_CUDA(cudaMemcpyAsync(kind.data(), c->kinds.ptr, n * 4, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync");
    if (c->str_count) {
        SPK_CUDA(cudaMemcpyAsync(soff.data(), c->str_offset.ptr, c->str_count * 8, cudaMemcpyDeviceToHost, s),
                 "cudaMemcpyAsync");
        SPK_CUDA(cudaMemcpyAsync(slen.data(), c->str_length.ptr, c->str_count * 4, cudaMemcpyDeviceToHost, s),
                 "cudaMemcpyAsync");
    }
    if (c->arena_used)
        SPK_CUDA(cudaMemcpyAsync(arena.data(), c->arena.ptr, c->arena_used, cudaMemcpyDeviceToHost, s),
                 "cudaMemcpyAsync");
    SPK_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    // A String's raw span is its quoted text: drop the quotes and undo the
    // doubled quotes (parse_record, ingest.rs:43-120); a Symbol is its span.
    size_t used = 0;
    for (u64 i = 0; i < n; ++i) {
        if (kinds) kinds[i] = kind[i];
        if (numbers) numbers[i] = kind[i] == 0 ? dict[i] : 0;
        if (offsets) offsets[i] = used;
        if (kind[i] == 0) continue;
        const unsigned char* raw = arena.data() + soff[dict[i]];
        const u32 len = slen[dict[i]];
        u32 b = 0, e = len;
        if (kind[i] == 1 && len >= 2) {
            b = 1;
            e = len - 1;
        }
        for (u32 k = b; k < e; ++k) {
            if (kind[i] == 1 && raw[k] == '"' && k + 1 < e && raw[k + 1] == '"') ++k;
            if (bytes && used < bytes_capacity) bytes[used] = raw[k];
            ++used;
        }
    }
    if (offsets) offsets[n] = used;
    *bytes_used = used;
    if (bytes && used > bytes_capacity) return fail(SPARKALOG_E_INVALID_ARGUMENT, "byte buffer too small");
    return 0;
}

int sparkalog_store_compact(sparkalog_store* st, u32 id) {
    if (!st) return fail(SPARKALOG_E_INVALID_ARGUMENT, "null store");
    RelState* r = st->find(id);
    if (!r) return fail(SPARKALOG_E_MISSING, "relation " + std::to_string(id) + " is not registered");
    int rc = materialize(st, *r);
    if (rc) return rc;
    return check_store_fault(st);
}

int sparkalog_store_rows(sparkalog_store* st, u32 id, int version, size_t* rows) {
    if (!st || !rows) return fail(SPARKALOG_E_INVALID_ARGUMENT, "null argument");
    RelState* r = st->find(id);
    if (!r) return fail(SPARKALOG_E_MISSING, "relation " + std::to_string(id) + " is not registered");
    if (version == SPARKALOG_FULL) {
        *rows = r->full_rows();
        return 0;
    }
    if (!r->recursive) return fail(SPARKALOG_E_NOT_RECURSIVE, "relation has no DELTA/NEWT state");
    *rows = r->delta_n;
    return 0;
}

int sparkalog_store_read(sparkalog_store* st, u32 id, int version, u32* first, u32* second, int location) {
    if (!st) return fail(SPARKALOG_E_INVALID_ARGUMENT, "null store");
    RelState* r = st->find(id);
    if (!r) return fail(SPARKALOG_E_MISSING, "relation " + std::to_string(id) + " is not registered");
    cudaStream_t s = st->stream;
    const u64* src;
    u64 n;
    if (version == SPARKALOG_FULL) {
        if (r->recursive) {
            int rc = materialize(st, *r);
            if (rc) return rc;
        }
        src = r->level[0].as<u64>();
        n = r->level_n[0];
    } else {
        if (!r->recursive) return fail(SPARKALOG_E_NOT_RECURSIVE, "relation has no DELTA/NEWT state");
        src = r->delta.as<u64>();
        n = r->delta_n;
    }
    if (n == 0) return 0;
    if (!first || !second) return fail(SPARKALOG_E_INVALID_ARGUMENT, "null output column");
    u32* d0 = first;
    u32* d1 = second;
    if (location == SPARKALOG_HOST) {
        SPK_CUDA(st->scratch_u32[0].ensure(n * 4, s), "cudaMallocAsync");
        SPK_CUDA(st->scratch_u32[1].ensure(n * 4, s), "cudaMallocAsync");
        d0 = st->scratch_u32[0].as<u32>();
        d1 = st->scratch_u32[1].as<u32>();
    }
    spk::unpack_rows_kernel<<<simple_grid(n), 256, 0, s>>>(src, n, d0, d1);
    SPK_CUDA(cudaGetLastError(), "unpack_rows_kernel");
    if (location == SPARKALOG_HOST) SPK_CUDA(columns_to_host(first, second, d0, d1, n, s), "cudaMemcpyAsync");
    SPK_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    return check_store_fault(st);
}

int sparkalog_store_anti_join(sparkalog_store* st, u32 left_id, u32 right_id, u32 out_id) {
    if (!st) return fail(SPARKALOG_E_INVALID_ARGUMENT, "null store");
    RelState* left = st->find(left_id);
    RelState* right = st->find(right_id);
    if (!left) return fail(SPARKALOG_E_MISSING, "relation " + std::to_string(left_id) + " is not registered");
    if (!right) return fail(SPARKALOG_E_MISSING, "relation " + std::to_string(right_id) + " is not registered");
    if (st->find(out_id))
        return fail(SPARKALOG_E_DUPLICATE, "relation " + std::to_string(out_id) + " is already registered");
    cudaStream_t s = st->stream;
    int rc = materialize(st, *left);
    if (rc) return rc;
    if (!right->sorted && right->level_n[0] > 1)
        return fail(SPARKALOG_E_UNSORTED_FULL, "FULL of relation " + std::to_string(right_id) + " is not sorted");
    const u64 n = left->level_n[0];
    RelState out;
    u64 out_n = 0;
    if (n > 0) {
        StoreOps* ops_ptr = store_ops(st);
    if (!ops_ptr) return static_cast<int>(cudaErrorMemoryAllocation);
    StoreOps& ops = *ops_ptr;
        SPK_CUDA(ops.a.ensure(n * 8, s), "cudaMallocAsync");
        SPK_CUDA(cudaMemcpyAsync(ops.a.ptr, left->level[0].ptr, n * 8, cudaMemcpyDeviceToDevice, s), "cudaMemcpyAsync");
        rc = sorted_difference(st, n, *right, out.level[0], &out_n);
        if (rc) return rc;
    } else {
        SPK_CUDA(out.level[0].ensure(8, s), "cudaMallocAsync");
    }
    out.level_n[0] = out_n;
    out.sorted = true;
    out.has_dups = false;
    st->relations[out_id] = std::move(out);
    return 0;
}

namespace {

// Stores `n` packed rows of ops.a, sorted and deduplicated, as the new static
// relation out_id.
int store_sorted_unique(sparkalog_store* st, u64 n, u32 out_id, size_t* rows) {
    cudaStream_t s = st->stream;
    RelState out;
    u64 out_n = 0;
    if (n > 0) {
        RelState none;
        int rc = sorted_difference(st, n, none, out.level[0], &out_n);
        if (rc) return rc;
    } else {
        SPK_CUDA(out.level[0].ensure(8, s), "cudaMallocAsync");
    }
    out.level_n[0] = out_n;
    out.sorted = true;
    out.has_dups = false;
    st->relations[out_id] = std::move(out);
    if (rows) *rows = out_n;
    return 0;
}

// Reads a device count word (synchronises the stream).
int read_count(sparkalog_store* st, StoreOps& ops, const u64* word, u64* out) {
    cudaStream_t s = st->stream;
    SPK_CUDA(cudaMemcpyAsync(ops.host, word, 8, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync");
    SPK_CUDA(cudaMemcpyAsync(reinterpret_cast<u32*>(ops.host + 1), ops.counters.as<u32>() + 32, 4,
                             cudaMemcpyDeviceToHost, s),
             "cudaMemcpyAsync");
    SPK_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    const u32 bits = static_cast<u32>(ops.host[1] & 0xffffffffu);
    if (bits) return fail(SPARKALOG_E_DEVICE_FAULT, "device error bits " + std::to_string(bits));
    *out = ops.host[0];
    return 0;
}

}  // namespace

int sparkalog_store_drop(sparkalog_store* st, u32 id) {
    if (!st) return fail(SPARKALOG_E_INVALID_ARGUMENT, "null store");
    auto it = st->relations.find(id);
    if (it == st->relations.end()) return fail(SPARKALOG_E_MISSING, "relation " + std::to_string(id) + " is not registered");
    cudaStream_t s = st->stream;
    RelState& r = it->second;
    for (auto& l : r.level) l.release(s);
    for (auto& d : r.dir) d.release(s);
    for (DevArray* d : {&r.spare, &r.delta, &r.newt, &r.member, &r.member_flag, &r.bloom}) d->release(s);
    st->relations.erase(it);
    return 0;
}

int sparkalog_store_select(sparkalog_store* st, u32 in_id, const sparkalog_select* spec, u32 out_id, size_t* rows) {
    if (!st || !spec) return fail(SPARKALOG_E_INVALID_ARGUMENT, "null argument");
    if (spec->where_mask > 7 || spec->out_source[0] > 2 || spec->out_source[1] > 2)
        return fail(SPARKALOG_E_INVALID_ARGUMENT, "select names a column outside a binary relation");
    RelState* in = st->find(in_id);
    if (!in) return fail(SPARKALOG_E_MISSING, "relation " + std::to_string(in_id) + " is not registered");
    if (st->find(out_id))
        return fail(SPARKALOG_E_DUPLICATE, "relation " + std::to_string(out_id) + " is already registered");
    cudaStream_t s = st->stream;
    int rc = materialize(st, *in);
    if (rc) return rc;
    const u64 n = in->level_n[0];
    StoreOps* ops_ptr = store_ops(st);
    if (!ops_ptr) return static_cast<int>(cudaErrorMemoryAllocation);
    StoreOps& ops = *ops_ptr;
    u64 m = 0;
    if (n > 0) {
        SPK_CUDA(ops.a.ensure(n * 8, s), "cudaMallocAsync");
        SPK_CUDA(ops.status.ensure_zeroed(((n + kSetTile - 1) / kSetTile + 1) * 8, s), "cudaMallocAsync");
        SPK_CUDA(cudaMemsetAsync(ops.counters.ptr, 0, 33 * 4, s), "cudaMemsetAsync");
        spk::SelectSpec sp{spec->where_mask,
                           {spec->where_value[0], spec->where_value[1]},
                           {spec->out_source[0], spec->out_source[1]},
                           {spec->out_value[0], spec->out_value[1]}};
        auto kernel = spk::select_rows_kernel<kThreads, kSetItems>;
        const size_t tiles = (n + kSetTile - 1) / kSetTile;
        kernel<<<grid_for(reinterpret_cast<const void*>(kernel), kThreads, tiles), kThreads, 0, s>>>(
            in->level[0].as<u64>(), n, sp, ops.a.as<u64>(), ops.counts.as<u64>(), ops.status.as<u64>(),
            ops.counters.as<u32>(), ops.ex.epoch++, ops.counters.as<u32>() + 32);
        SPK_CUDA(cudaGetLastError(), "select_rows_kernel");
        rc = read_count(st, ops, ops.counts.as<u64>(), &m);
        if (rc) return rc;
    }
    if (m > 0) {
        const u32 mv = std::max(spec->out_source[0] == 2 ? spec->out_value[0] : 0u,
                                spec->out_source[1] == 2 ? spec->out_value[1] : 0u);
        st->max_value = std::max(st->max_value, mv);
    }
    return store_sorted_unique(st, m, out_id, rows);
}

int sparkalog_store_join(sparkalog_store* st, u32 left_id, u32 right_id, u32 left_key, u32 right_key,
                         const u32* proj_side, const u32* proj_col, u32 out_id, size_t* rows) {
    if (!st || !proj_side || !proj_col) return fail(SPARKALOG_E_INVALID_ARGUMENT, "null argument");
    if (left_key > 1 || right_key > 1 || proj_side[0] > 1 || proj_side[1] > 1 || proj_col[0] > 1 || proj_col[1] > 1)
        return fail(SPARKALOG_E_MISSING_COLUMN, "join names a column outside a binary relation");
    RelState* left = st->find(left_id);
    RelState* right = st->find(right_id);
    if (!left) return fail(SPARKALOG_E_MISSING, "relation " + std::to_string(left_id) + " is not registered");
    if (!right) return fail(SPARKALOG_E_MISSING, "relation " + std::to_string(right_id) + " is not registered");
    if (st->find(out_id))
        return fail(SPARKALOG_E_DUPLICATE, "relation " + std::to_string(out_id) + " is already registered");
    cudaStream_t s = st->stream;
    int rc = materialize(st, *left);
    if (rc) return rc;
    StoreOps* ops_ptr = store_ops(st);
    if (!ops_ptr) return static_cast<int>(cudaErrorMemoryAllocation);
    StoreOps& ops = *ops_ptr;
    sparkalog_executor& ex = ops.ex;
    if (!ex.counters.ptr) {
        // The index build reports through the executor's error words.
        const size_t bytes = (kCounterWords + 64) * 4;
        SPK_CUDA(ex.counters.ensure(bytes, s), "cudaMallocAsync");
        SPK_CUDA(cudaMemsetAsync(ex.counters.ptr, 0, bytes, s), "cudaMemsetAsync");
    }
    IndexCache ic;
    rc = build_index(&ex, st, ic, right_id, right_key);
    if (rc) return rc;
    const u64 n = left->level_n[0];
    const u64 bound = n * static_cast<u64>(ic.max_degree);
    u64 m = 0;
    if (bound > 0) {
        SPK_CUDA(ops.a.ensure(bound * 8, s), "cudaMallocAsync");
        SPK_CUDA(ops.status.ensure_zeroed(((n + kJoinTile - 1) / kJoinTile + 1) * 8, s), "cudaMallocAsync");
        SPK_CUDA(cudaMemsetAsync(ops.counters.ptr, 0, 33 * 4, s), "cudaMemsetAsync");
        SPK_CUDA(cudaMemsetAsync(ops.counts.ptr, 0, 32, s), "cudaMemsetAsync");
        ops.host[0] = n;
        SPK_CUDA(cudaMemcpyAsync(ops.counts.as<u64>() + 1, ops.host, 8, cudaMemcpyHostToDevice, s), "cudaMemcpyAsync");
        spk::FusedJoinArgs a{};
        a.delta = left->level[0].as<u64>();
        a.delta_count = ops.counts.as<u64>() + 1;
        a.left_key = left_key;
        if (ic.bucketed) {
            a.bucket_dir = ic.bucket_dir.as<u32>();
            a.bucket_shift = ic.bucket_shift;
            a.buckets = ic.buckets;
            a.keys = ic.keys32.as<u32>();
        } else {
            a.dense_offsets = ic.offsets.as<u32>();
            a.dense_keys = ic.num_keys;
        }
        a.rows = ic.identity ? nullptr : ic.rows.as<u32>();
        a.right = right->level[0].as<u64>();
        a.side[0] = proj_side[0];
        a.side[1] = proj_side[1];
        a.col[0] = proj_col[0];
        a.col[1] = proj_col[1];
        a.out = ops.a.as<u64>();
        a.capacity = bound;
        a.count_in = ops.counts.as<u64>() + 2;
        a.count_out = ops.counts.as<u64>() + 3;
        a.status = ops.status.as<u64>();
        a.tile_counter = ops.counters.as<u32>();
        a.epoch_ptr = nullptr;
        a.epoch_add = ex.epoch++;
        a.err = ops.counters.as<u32>() + 32;
        auto kernel = spk::join_fused_kernel<kThreads, kJoinItems>;
        const size_t tiles = (n + kJoinTile - 1) / kJoinTile;
        kernel<<<grid_for(reinterpret_cast<const void*>(kernel), kThreads, std::max<size_t>(tiles, 1)), kThreads, 0,
                 s>>>(a);
        SPK_CUDA(cudaGetLastError(), "join_fused_kernel");
        rc = read_count(st, ops, ops.counts.as<u64>() + 3, &m);
        if (rc) return rc;
    }
    for (DevArray* d : {&ic.offsets, &ic.rows, &ic.keys32, &ic.bucket_dir, &ic.compact}) d->release(s);
    return store_sorted_unique(st, m, out_id, rows);
}

int sparkalog_store_append(sparkalog_store* st, u32 id, const u32* first, const u32* second, size_t rows,
                           int location) {
    if (!st) return fail(SPARKALOG_E_INVALID_ARGUMENT, "null store");
    RelState* r = st->find(id);
    if (!r) return fail(SPARKALOG_E_MISSING, "relation " + std::to_string(id) + " is not registered");
    if (rows > kMaxRelationRows) return fail(SPARKALOG_E_TOO_MANY_ROWS, "too many rows for u32 row ids");
    if (rows == 0) return 0;
    cudaStream_t s = st->stream;
    if (!r->sorted || r->has_dups) {
        int rc = materialize(st, *r);
        if (rc) return rc;
        if (!r->sorted) return fail(SPARKALOG_E_UNSORTED_FULL, "FULL of relation " + std::to_string(id) + " is not sorted");
    }
    StoreOps* ops_ptr = store_ops(st);
    if (!ops_ptr) return static_cast<int>(cudaErrorMemoryAllocation);
    StoreOps& ops = *ops_ptr;
    bool sorted_in, dups_in;
    int rc = pack_columns(st, first, second, rows, location, ops.a, &sorted_in, &dups_in);
    if (rc) return rc;
    DevArray fresh;
    u64 fresh_n = 0;
    rc = sorted_difference(st, rows, *r, fresh, &fresh_n);
    if (rc) return rc;
    if (fresh_n > 0) {
        if (r->full_rows() + fresh_n > kMaxRelationRows)
            return fail(SPARKALOG_E_TOO_MANY_ROWS, "relation would exceed 2^32 - 1 rows (u32 row ids)");
        // FULL: new rows are disjoint from every level, so they merge into TAIL
        // (level 0 for a static relation, which keeps a single run).
        const int l = r->recursive ? static_cast<int>(st->levels) - 1 : 0;
        const u64 tn = r->level_n[l] + fresh_n;
        SPK_CUDA(r->spare.ensure(tn * 8, s), "cudaMallocAsync");
        SPK_CUDA(store_merge(st, r->level[l].as<u64>(), r->level_n[l], fresh.as<u64>(), fresh_n, r->spare.as<u64>()),
                 "merge_bulk_kernel");
        swap_arrays(r->level[l], r->spare);
        r->level_n[l] = tn;
        r->dir_valid[l] = false;
        rc = member_add(*r, fresh.as<u64>(), fresh_n, ops.counters.as<u32>() + 33, s, nullptr);
        if (rc) return rc;
        if (r->bloom_valid && fresh_n) {
            // FULL's Bloom filter takes the new rows too.
            spk::bloom_insert_kernel<<<simple_grid(fresh_n), 256, 0, s>>>(fresh.as<u64>(), fresh_n, bloom_of(*r));
            SPK_CUDA(cudaGetLastError(), "bloom_insert_kernel");
        }
        if (r->recursive) {
            // DELTA u= fresh rows (DELTA is part of FULL, so they are disjoint).
            if (!r->delta_sorted) {
                rc = sort_unique_delta(st, *r);
                if (rc) return rc;
            }
            const u64 dn = r->delta_n + fresh_n;
            SPK_CUDA(r->newt.ensure(std::max<u64>(dn, 1) * 8, s), "cudaMallocAsync");
            SPK_CUDA(store_merge(st, r->delta.as<u64>(), r->delta_n, fresh.as<u64>(), fresh_n, r->newt.as<u64>()),
                     "merge_bulk_kernel");
            swap_arrays(r->delta, r->newt);
            r->delta_n = dn;
        }
        r->version += 1;
    }
    SPK_CUDA(cudaMemcpyAsync(ops.host + 2, ops.counters.as<u32>() + 33, 4, cudaMemcpyDeviceToHost, s),
             "cudaMemcpyAsync");
    SPK_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    fresh.release(s);
    const u32 member_bits = static_cast<u32>(ops.host[2] & 0xffffffffu);
    if (member_bits)
        return fail(SPARKALOG_E_DEVICE_FAULT, "device error bits " + std::to_string(member_bits) + " (hash set of FULL)");
    return 0;
}

namespace {

int extract_segment(sparkalog_store* st, u32 id, u32 shift, u32 segment, u32* first, u32* second, int location,
                    size_t* rows, u32 mask0, u32 mask1) {
    if (!st || !rows || shift > 31) return fail(SPARKALOG_E_INVALID_ARGUMENT, "invalid argument");
    RelState* r = st->find(id);
    if (!r) return fail(SPARKALOG_E_MISSING, "relation " + std::to_string(id) + " is not registered");
    cudaStream_t s = st->stream;
    if (!r->sorted) return fail(SPARKALOG_E_UNSORTED_FULL, "FULL of relation " + std::to_string(id) + " is not sorted");
    const u64 lo_key = static_cast<u64>(segment) << (shift + 32);
    const u64 next = static_cast<u64>(segment) + 1;
    const u64 hi_key = (next << shift) > 0xffffffffull ? ~0ull : next << (shift + 32);
    spk::Levels lv{};
    int map[spk::kMaxLevels];
    for (int l = 0; l < spk::kMaxLevels; ++l) {
        if (r->level_n[l] == 0) continue;
        map[lv.n] = l;
        lv.keys[lv.n] = r->level[l].as<u64>();
        lv.count[lv.n] = r->level_n[l];
        ++lv.n;
    }
    StoreOps* ops_ptr = store_ops(st);
    if (!ops_ptr) return static_cast<int>(cudaErrorMemoryAllocation);
    StoreOps& ops = *ops_ptr;
    u64 bounds[2 * spk::kMaxLevels] = {0};
    if (lv.n) {
        spk::level_bounds_kernel<<<1, 32, 0, s>>>(lv, lo_key, hi_key, ops.counts.as<u64>());
        SPK_CUDA(cudaGetLastError(), "level_bounds_kernel");
        SPK_CUDA(cudaMemcpyAsync(ops.host, ops.counts.ptr, sizeof(bounds), cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync");
        SPK_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
        std::memcpy(bounds, ops.host, sizeof(bounds));
    }
    u64 total = 0;
    for (int k = 0; k < lv.n; ++k) total += bounds[2 * k + 1] - bounds[2 * k];
    *rows = total;
    if (!first) return 0;
    if (!second) return fail(SPARKALOG_E_INVALID_ARGUMENT, "null output column");
    if (total == 0) return 0;
    // Merge the (disjoint, sorted) slices of the levels into one sorted run.
    SPK_CUDA(ops.a.ensure(total * 8, s), "cudaMallocAsync");
    SPK_CUDA(ops.b.ensure(total * 8, s), "cudaMallocAsync");
    u64 have = 0;
    for (int k = 0; k < lv.n; ++k) {
        const u64 len = bounds[2 * k + 1] - bounds[2 * k];
        if (len == 0) continue;
        const u64* slice = r->level[map[k]].as<u64>() + bounds[2 * k];
        SPK_CUDA(store_merge(st, ops.a.as<u64>(), have, slice, len, ops.b.as<u64>()), "merge_bulk_kernel");
        swap_arrays(ops.a, ops.b);
        have += len;
    }
    u32* d0 = first;
    u32* d1 = second;
    if (location == SPARKALOG_HOST) {
        SPK_CUDA(st->scratch_u32[0].ensure(total * 4, s), "cudaMallocAsync");
        SPK_CUDA(st->scratch_u32[1].ensure(total * 4, s), "cudaMallocAsync");
        d0 = st->scratch_u32[0].as<u32>();
        d1 = st->scratch_u32[1].as<u32>();
    }
    spk::unpack_rows_kernel<<<simple_grid(total), 256, 0, s>>>(ops.a.as<u64>(), total, d0, d1, mask0, mask1);
    SPK_CUDA(cudaGetLastError(), "unpack_rows_kernel");
    if (location == SPARKALOG_HOST) SPK_CUDA(columns_to_host(first, second, d0, d1, total, s), "cudaMemcpyAsync");
    SPK_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    return 0;
}

}  // namespace

int sparkalog_store_extract_segment(sparkalog_store* st, u32 id, u32 shift, u32 segment, u32* first, u32* second,
                                    int location, size_t* rows) {
    return extract_segment(st, id, shift, segment, first, second, location, rows, ~0u, ~0u);
}

int sparkalog_store_extract_segment_untagged(sparkalog_store* st, u32 id, u32 shift, u32 segment,
                                             int clear_second, u32* first, u32* second, int location,
                                             size_t* rows) {
    if (shift > 31) return fail(SPARKALOG_E_INVALID_ARGUMENT, "invalid argument");
    const u32 low = shift == 0 ? 0u : (~0u >> (32 - shift));
    return extract_segment(st, id, shift, segment, first, second, location, rows, low, clear_second ? low : ~0u);
}

int sparkalog_store_remove_segments(sparkalog_store* st, u32 id, u32 shift, const u32* segments, size_t count) {
    if (!st || shift > 31 || (count && !segments)) return fail(SPARKALOG_E_INVALID_ARGUMENT, "invalid argument");
    RelState* r = st->find(id);
    if (!r) return fail(SPARKALOG_E_MISSING, "relation " + std::to_string(id) + " is not registered");
    if (count == 0) return 0;
    cudaStream_t s = st->stream;
    const u64 segs = 1ull << (32 - shift);
    const u64 words = (segs + 31) / 32;
    std::vector<u32> bitmap(words, 0);
    for (size_t k = 0; k < count; ++k) {
        if (segments[k] >= segs) return fail(SPARKALOG_E_INVALID_ARGUMENT, "segment out of range");
        bitmap[segments[k] >> 5] |= 1u << (segments[k] & 31);
    }
    StoreOps* ops_ptr = store_ops(st);
    if (!ops_ptr) return static_cast<int>(cudaErrorMemoryAllocation);
    StoreOps& ops = *ops_ptr;
    SPK_CUDA(ops.bitmap.ensure(words * 4, s), "cudaMallocAsync");
    SPK_CUDA(cudaMemcpyAsync(ops.bitmap.ptr, bitmap.data(), words * 4, cudaMemcpyHostToDevice, s), "cudaMemcpyAsync");
    auto filter = [&](DevArray& buf, u64& n, DevArray& spare) -> int {
        if (n == 0) return 0;
        SPK_CUDA(spare.ensure(n * 8, s), "cudaMallocAsync");
        SPK_CUDA(ops.status.ensure_zeroed(((n + kSetTile - 1) / kSetTile + 1) * 8, s), "cudaMallocAsync");
        SPK_CUDA(cudaMemsetAsync(ops.counters.ptr, 0, 64, s), "cudaMemsetAsync");
        auto kernel = spk::filter_segments_kernel<kThreads, kSetItems>;
        const size_t tiles = (n + kSetTile - 1) / kSetTile;
        kernel<<<grid_for(reinterpret_cast<const void*>(kernel), kThreads, tiles), kThreads, 0, s>>>(
            buf.as<u64>(), n, shift, ops.bitmap.as<u32>(), spare.as<u64>(), ops.counts.as<u64>(),
            ops.status.as<u64>(), ops.counters.as<u32>(), ops.ex.epoch++, ops.counters.as<u32>() + 32);
        SPK_CUDA(cudaGetLastError(), "filter_segments_kernel");
        SPK_CUDA(cudaMemcpyAsync(ops.host, ops.counts.ptr, 8, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync");
        SPK_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
        swap_arrays(buf, spare);
        std::memcpy(&n, ops.host, 8);
        return 0;
    };
    for (int l = 0; l < spk::kMaxLevels; ++l) {
        int rc = filter(r->level[l], r->level_n[l], r->spare);
        if (rc) return rc;
        r->dir_valid[l] = false;
    }
    r->member_valid = false;  // the hash set cannot drop rows: rebuilt on next use
    if (r->recursive) {
        int rc = filter(r->delta, r->delta_n, r->newt);
        if (rc) return rc;
    }
    r->version += 1;
    return 0;
}

int sparkalog_executor_compile(sparkalog_store* st, const u32* relations, size_t relation_count,
                               const sparkalog_rule_plan* rules, size_t rule_count, sparkalog_executor** out) {
    if (!st || !out || (relation_count && !relations) || (rule_count && !rules))
        return fail(SPARKALOG_E_INVALID_ARGUMENT, "null argument");
    if (relation_count == 0) return fail(SPARKALOG_E_EMPTY_SCC, "recursive SCC has no relations");
    for (size_t i = 0; i < relation_count; ++i) {
        for (size_t j = 0; j < i; ++j)
            if (relations[j] == relations[i])
                return fail(SPARKALOG_E_DUPLICATE_SCC_RELATION,
                            "relation " + std::to_string(relations[i]) + " occurs twice in its SCC");
        RelState* r = st->find(relations[i]);
        if (!r) return fail(SPARKALOG_E_MISSING, "relation " + std::to_string(relations[i]) + " is not registered");
        if (!r->recursive)
            return fail(SPARKALOG_E_NOT_RECURSIVE,
                        "relation " + std::to_string(relations[i]) + " has no DELTA/NEWT state");
    }
    auto in_scc = [&](u32 id) {
        for (size_t i = 0; i < relation_count; ++i)
            if (relations[i] == id) return true;
        return false;
    };
    for (size_t k = 0; k < rule_count; ++k) {
        const sparkalog_rule_plan& p = rules[k];
        if (!st->find(p.delta_input))
            return fail(SPARKALOG_E_MISSING, "relation " + std::to_string(p.delta_input) + " is not registered");
        if (!st->find(p.right_input))
            return fail(SPARKALOG_E_MISSING, "relation " + std::to_string(p.right_input) + " is not registered");
        if (!in_scc(p.delta_input))
            return fail(SPARKALOG_E_DELTA_OUTSIDE_SCC,
                        "DELTA relation " + std::to_string(p.delta_input) + " is outside its SCC");
        if (!in_scc(p.target))
            return fail(SPARKALOG_E_TARGET_OUTSIDE_SCC,
                        "rule target " + std::to_string(p.target) + " is outside its SCC");
    }
    auto* ex = new sparkalog_executor();
    ex->relations.assign(relations, relations + relation_count);
    ex->rules.assign(rules, rules + rule_count);
    for (size_t t = 0; t < relation_count; ++t) {
        TargetRT trt;
        trt.id = relations[t];
        for (size_t k = 0; k < rule_count; ++k)
            if (rules[k].target == relations[t]) trt.rules.push_back(k);
        if (trt.rules.empty()) {
            delete ex;
            return fail(SPARKALOG_E_MISSING_RULE_TARGET,
                        "relation " + std::to_string(relations[t]) + " has no recursive rule");
        }
        const sparkalog_rule_plan& first = rules[trt.rules[0]];
        for (size_t k : trt.rules) {
            const sparkalog_rule_plan& p = rules[k];
            if (std::memcmp(p.anti_left, first.anti_left, 8) || std::memcmp(p.anti_right, first.anti_right, 8) ||
                std::memcmp(p.union_left, first.union_left, 8) || std::memcmp(p.union_right, first.union_right, 8)) {
                delete ex;
                return fail(SPARKALOG_E_INCOMPATIBLE_TARGET_PLANS,
                            "clauses for relation " + std::to_string(relations[t]) +
                                " use incompatible set plans");
            }
        }
        ex->targets.push_back(std::move(trt));
    }
    ex->index.resize(rule_count);
    ex->stream = st->stream;
    ex->counts_words = 0;
    for (auto& t : ex->targets) ex->counts_words += t.rules.size() + 3;
    cudaStream_t s = st->stream;
    const size_t counter_bytes = (kCounterWords + 2 * ex->counts_words + 64) * 4;
    cudaError_t e = ex->counters.ensure(counter_bytes, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(ex->counters.ptr, 0, counter_bytes, s);
    if (e == cudaSuccess) e = pinned_get(reinterpret_cast<void**>(&ex->host_counts), ex->counts_words * 8 + 512);
    if (e == cudaSuccess) e = ex->rule_delta.ensure(std::max<size_t>(rule_count, 1) * 8, s);
    if (e == cudaSuccess) e = pinned_get(reinterpret_cast<void**>(&ex->host_rule_delta), std::max<size_t>(rule_count, 1) * 8);
    if (e == cudaSuccess) e = pinned_get(reinterpret_cast<void**>(&ex->host_active), relation_count * spk::kMaxPasses * 4 + 64);
    if (e != cudaSuccess) {
        delete ex;
        return cuda_fail(e, "sparkalog_executor_compile");
    }
    *out = ex;
    return 0;
}

void sparkalog_executor_destroy(sparkalog_executor* ex) {
    if (!ex) return;
    // Buffers are freed in the order of the stream that used them, and the
    // pinned count buffers go back to the pool once that stream is idle.
    cudaStream_t s = ex->stream;
    for (auto& t : ex->targets) {
        t.j_a.release(s);
        t.j_b.release(s);
        t.sort.plan.release(s);
        t.sort.status.release(s);
        t.anti_plan.release(s);
        t.anti_scratch.release(s);
        t.anti_counts.release(s);
    }
    for (auto& ic : ex->index) {
        ic.offsets.release(s);
        ic.rows.release(s);
        ic.keys32.release(s);
        ic.bucket_dir.release(s);
        ic.compact.release(s);
    }
    ex->seg_seen.release(s);
    ex->seg_new.release(s);
    ex->rule_delta.release(s);
    ex->counters.release(s);
    ex->status.release(s);
    ex->index_sort.plan.release(s);
    ex->index_sort.status.release(s);
    ex->index_pairs[0].release(s);
    ex->index_pairs[1].release(s);
    cudaStreamSynchronize(s);
    pinned_put(ex->host_counts, ex->counts_words * 8 + 512);
    pinned_put(ex->host_rule_delta, std::max<size_t>(ex->rules.size(), 1) * 8);
    pinned_put(ex->host_active, ex->relations.size() * spk::kMaxPasses * 4 + 64);
    for (auto& t : ex->timings) {
        cudaEventDestroy(t.a);
        cudaEventDestroy(t.b);
    }
    for (cudaEvent_t e : ex->free_events) cudaEventDestroy(e);
    delete ex;
}

int sparkalog_executor_track_segments(sparkalog_executor* ex, u32 shift, u32 count) {
    if (!ex || shift > 31) return fail(SPARKALOG_E_INVALID_ARGUMENT, "invalid segment tracking arguments");
    cudaStream_t s = ex->stream;
    ex->seg_shift = shift;
    ex->seg_count = count;
    if (count) {
        SPK_CUDA(ex->seg_seen.ensure(static_cast<size_t>(count) * 4, s), "cudaMallocAsync");
        SPK_CUDA(ex->seg_new.ensure(static_cast<size_t>(count) * 8, s), "cudaMallocAsync");
        SPK_CUDA(cudaMemsetAsync(ex->seg_seen.ptr, 0, static_cast<size_t>(count) * 4, s), "cudaMemsetAsync");
        SPK_CUDA(cudaMemsetAsync(ex->seg_new.ptr, 0, static_cast<size_t>(count) * 8, s), "cudaMemsetAsync");
        SPK_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    }
    return 0;
}

int sparkalog_executor_segment_stats(sparkalog_executor* ex, u32* last_active_round, u64* new_rows) {
    if (!ex || !last_active_round || !new_rows) return fail(SPARKALOG_E_INVALID_ARGUMENT, "null argument");
    if (ex->seg_count == 0) return 0;
    cudaStream_t s = ex->stream;
    SPK_CUDA(cudaMemcpyAsync(last_active_round, ex->seg_seen.ptr, static_cast<size_t>(ex->seg_count) * 4,
                             cudaMemcpyDeviceToHost, s),
             "cudaMemcpyAsync");
    SPK_CUDA(cudaMemcpyAsync(new_rows, ex->seg_new.ptr, static_cast<size_t>(ex->seg_count) * 8,
                             cudaMemcpyDeviceToHost, s),
             "cudaMemcpyAsync");
    SPK_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    return 0;
}

int sparkalog_executor_set_profiling(sparkalog_executor* ex, int enable) {
    if (!ex) return fail(SPARKALOG_E_INVALID_ARGUMENT, "null executor");
    ex->profiling = enable != 0;
    return 0;
}

int sparkalog_executor_set_fused(sparkalog_executor* ex, int enable) {
    if (!ex) return fail(SPARKALOG_E_INVALID_ARGUMENT, "null executor");
    ex->fused_enabled = enable != 0;
    return 0;
}

int sparkalog_executor_trace(sparkalog_executor* ex, sparkalog_round_trace* out, size_t capacity, size_t* count,
                             int reset) {
    if (!ex || !count || (capacity && !out)) return fail(SPARKALOG_E_INVALID_ARGUMENT, "null argument");
    *count = ex->trace.size();
    const size_t n = std::min(capacity, ex->trace.size());
    for (size_t i = 0; i < n; ++i) out[i] = ex->trace[i];
    if (reset) ex->trace.clear();
    return 0;
}

int sparkalog_executor_set_member_set(sparkalog_executor* ex, int enable) {
    if (!ex) return fail(SPARKALOG_E_INVALID_ARGUMENT, "null executor");
    ex->member_enabled = enable != 0;
    return 0;
}

int sparkalog_executor_set_device_loop(sparkalog_executor* ex, int enable) {
    if (!ex) return fail(SPARKALOG_E_INVALID_ARGUMENT, "null executor");
    ex->device_loop = enable != 0;
    return 0;
}

int sparkalog_executor_device_loop_stats(sparkalog_executor* ex, uint64_t* launches, uint64_t* rounds) {
    if (!ex || !launches || !rounds) return fail(SPARKALOG_E_INVALID_ARGUMENT, "null argument");
    *launches = ex->loop_launches;
    *rounds = ex->loop_rounds;
    return 0;
}

int sparkalog_tuning_defaults(sparkalog_tuning* out) {
    if (!out) return fail(SPARKALOG_E_INVALID_ARGUMENT, "null output");
    *out = default_tuning();
    return 0;
}

int sparkalog_executor_set_tuning(sparkalog_executor* ex, const sparkalog_tuning* tuning) {
    if (!ex || !tuning) return fail(SPARKALOG_E_INVALID_ARGUMENT, "null argument");
    if (!tuning_valid(*tuning)) return fail(SPARKALOG_E_INVALID_ARGUMENT, "tuning value out of range");
    ex->tuning = *tuning;
    for (auto& t : ex->targets) {
        t.fused_rows_cap = tuning->fused_rows_cap;
        t.fused_rows = std::min(t.fused_rows, t.fused_rows_cap);
    }
    return 0;
}

int sparkalog_executor_get_tuning(sparkalog_executor* ex, sparkalog_tuning* out) {
    if (!ex || !out) return fail(SPARKALOG_E_INVALID_ARGUMENT, "null argument");
    *out = ex->tuning;
    return 0;
}

int sparkalog_executor_stats(sparkalog_executor* ex, sparkalog_kernel_stats* out, int reset) {
    if (!ex || !out) return fail(SPARKALOG_E_INVALID_ARGUMENT, "null argument");
    *out = ex->stats;
    if (reset) ex->stats = sparkalog_kernel_stats{};
    return 0;
}

// Runs rounds while any DELTA of the SCC is non-empty, at most max_iterations
// of them. With limit_is_error the limit is RecursiveExecutor::run's
// IterationLimit error; otherwise the call just stops (a step of a serving
// loop). *converged reports whether every DELTA is empty afterwards.
static int run_rounds(sparkalog_executor* ex, sparkalog_store* st, size_t max_iterations, bool limit_is_error,
                      sparkalog_scc_summary* summary, int* converged) {
    if (!ex || !st) return fail(SPARKALOG_E_INVALID_ARGUMENT, "null argument");
    cudaStream_t s = st->stream;
    for (const auto& p : ex->rules) {
        if (p.left_key > 1 || p.right_key > 1 || !valid_cols(p.proj_col) || !valid_cols(p.distinct_cols) ||
            !valid_cols(p.anti_left) || !valid_cols(p.anti_right) || !valid_cols(p.union_left) ||
            !valid_cols(p.union_right) || p.proj_side[0] > 1 || p.proj_side[1] > 1)
            return fail(SPARKALOG_E_MISSING_COLUMN, "plan names a column outside a binary relation");
        // The device pipeline keeps rows packed in (first, second) order, which
        // is the only set-operator column order the binary lowering produces
        // (datalog/src/subset.rs:226-237).
        if (p.distinct_cols[0] != 0 || p.distinct_cols[1] != 1 || p.anti_left[0] != 0 || p.anti_left[1] != 1 ||
            p.anti_right[0] != 0 || p.anti_right[1] != 1 || p.union_left[0] != 0 || p.union_left[1] != 1 ||
            p.union_right[0] != 0 || p.union_right[1] != 1)
            return fail(SPARKALOG_E_INVALID_ARGUMENT, "set operators must use columns [0, 1]");
    }
    // The directory granularity is the store's (its levels carry their
    // directories): a different one invalidates them, and they are rebuilt
    // on first use.
    st->levels = ex->tuning.levels;
    st->merge_items = ex->tuning.merge_items;
    if (st->dir_rows_log2 != ex->tuning.dir_rows_log2) {
        st->dir_rows_log2 = ex->tuning.dir_rows_log2;
        for (auto& kv : st->relations)
            for (int l = 0; l < spk::kMaxLevels; ++l) kv.second.dir_valid[l] = false;
    }
    u32* counters = ex->tile_counters();
    u32* err = ex->err_words();
    u64* counts = ex->count_words();
    // Errors of hash-set inserts, which run after a round's check: a word the
    // per-round clearing leaves alone, read once when the run ends.
    u32* member_err = err + kMemberErrOffset;
    SPK_CUDA(cudaMemsetAsync(member_err, 0, 4, s), "cudaMemsetAsync");

    // FULL of each SCC relation must be a sorted run before the first merge;
    // duplicates inside it are removed the way the reference's first union
    // would remove them (only when a round will run).
    bool any_delta = false;
    for (u32 id : ex->relations) any_delta |= st->find(id)->delta_n != 0;
    if (any_delta) {
        for (u32 id : ex->relations) {
            RelState& r = *st->find(id);
            if (r.sorted && !r.has_dups) continue;  // levels are already sorted, disjoint runs
            int rc = materialize(st, r);
            if (rc) return rc;
            if (!r.sorted)
                return fail(SPARKALOG_E_UNSORTED_FULL,
                            "FULL of relation " + std::to_string(id) + " is not sorted by (first, second)");
            if (r.has_dups && r.level_n[0] > 0) {
                const u64 n = r.level_n[0];
                SPK_CUDA(r.spare.ensure(n * 8, s), "cudaMallocAsync");
                SPK_CUDA(ex->status.ensure_zeroed(((n + kSetTile - 1) / kSetTile + 1) * 8, s), "cudaMallocAsync");
                SPK_CUDA(cudaMemsetAsync(counters, 0, kCounterWords * 4, s), "cudaMemsetAsync");
                SPK_CUDA(cudaMemsetAsync(counts, 0, 8, s), "cudaMemsetAsync");
                // unique over the packed run: anti-join against no levels.
                spk::Levels none{};
                none.n = 0;
                u64* nptr = counts + 1;
                SPK_CUDA(cudaMemcpyAsync(nptr, &r.level_n[0], 8, cudaMemcpyHostToDevice, s), "cudaMemcpyAsync");
                auto kernel = spk::anti_join_levels_kernel<kThreads, kSetItems, kLevelStage>;
                const size_t tiles = (n + kSetTile - 1) / kSetTile;
                kernel<<<grid_for(reinterpret_cast<const void*>(kernel), kThreads, tiles), kThreads, 0, s>>>(
                    r.level[0].as<u64>(), r.level[0].as<u64>(), nullptr, nptr, none, r.spare.as<u64>(), counts,
                    ex->status.as<u64>(), counters, ex->epoch++, err, nullptr);
                SPK_CUDA(cudaGetLastError(), "anti_join_levels_kernel");
                ex->stats.total_launches += 1;
                SPK_CUDA(cudaMemcpyAsync(ex->host_counts, counts, 8, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync");
                SPK_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
                swap_arrays(r.level[0], r.spare);
                r.level_n[0] = ex->host_counts[0];
                r.has_dups = false;
                r.dir_valid[0] = false;
                r.member_valid = false;
            }
        }
    }

    // Levels past the tuning's count (rows appended into the last slot, or a
    // smaller count than the last run's) fold into the tuning's TAIL.
    for (u32 id : ex->relations) {
        RelState& r = *st->find(id);
        const int tail = static_cast<int>(ex->tuning.levels) - 1;
        for (int l = tail + 1; l < spk::kMaxLevels; ++l) {
            if (r.level_n[l] == 0) continue;
            int rc = merge_into_level(st, r, tail, r.level[tail].as<u64>(), r.level_n[tail], r.level[l].as<u64>(),
                                      r.level_n[l], s, nullptr);
            if (rc) return rc;
            r.level_n[l] = 0;
            r.dir_valid[l] = false;
        }
    }

    u64 iterations = 0, total_new = 0;
    for (;;) {
        bool has_delta = false;
        u64 remaining = 0;
        for (u32 id : ex->relations) {
            has_delta |= st->find(id)->delta_n != 0;
            remaining += st->find(id)->delta_n;
        }
        if (!has_delta) break;
        if (iterations >= max_iterations) {
            if (!limit_is_error) break;
            if (summary) {
                summary->iterations = iterations;
                summary->total_new_rows = total_new;
            }
            return fail(SPARKALOG_E_ITERATION_LIMIT, "recursive SCC did not converge within " +
                                                         std::to_string(max_iterations) + " iterations; " +
                                                         std::to_string(remaining) + " delta rows remain");
        }
        if (ex->epoch > spk::kEpochMask - 4096) {
            // Epoch wrap: clear every look-back buffer so stale words never match.
            if (ex->status.ptr) SPK_CUDA(cudaMemsetAsync(ex->status.ptr, 0, ex->status.bytes, s), "cudaMemsetAsync");
            for (auto& t : ex->targets)
                if (t.sort.status.ptr)
                    SPK_CUDA(cudaMemsetAsync(t.sort.status.ptr, 0, t.sort.status.bytes, s), "cudaMemsetAsync");
            if (ex->index_sort.status.ptr)
                SPK_CUDA(cudaMemsetAsync(ex->index_sort.status.ptr, 0, ex->index_sort.status.bytes, s),
                         "cudaMemsetAsync");
            ex->epoch = 1;
        }

        // RuleRuntime::evaluate's index cache (generic.rs:217-229).
        for (size_t k = 0; k < ex->rules.size(); ++k) {
            const sparkalog_rule_plan& p = ex->rules[k];
            RelState* right = st->find(p.right_input);
            IndexCache& ic = ex->index[k];
            if (!ic.valid || ic.relation != p.right_input || ic.version != right->version ||
                ic.column != p.right_key) {
                int rc = build_index(ex, st, ic, p.right_input, p.right_key);
                if (rc) return rc;
            }
        }

        // Small rounds of a single transitive-closure-shaped target run on the
        // device, many per host round trip (spk_loop.cuh).
        if (ex->device_loop && !ex->profiling && !ex->member_enabled && ex->targets.size() == 1 &&
            ex->tuning.levels >= 2 && fused_eligible(ex, st, 0)) {
            const TargetRT& t = ex->targets[0];
            const sparkalog_rule_plan& p = ex->rules[t.rules[0]];
            RelState& tr = *st->find(t.id);
            const u64 dn = st->find(p.delta_input)->delta_n;
            const u64 bound = dn * static_cast<u64>(std::max<u32>(ex->index[t.rules[0]].max_degree, 1));
            const int tail = static_cast<int>(ex->tuning.levels) - 1;
            if (p.delta_input == t.id && dn > 0 && bound <= ex->tuning.group_candidates &&
                tr.level_n[tail - 1] > 0 && tr.level_n[tail] * ex->tuning.level_ratio <= tr.level_n[tail - 1]) {
                u64 applied = 0, added = 0;
                int rc = run_device_loop(ex, st, 0, max_iterations - iterations, &applied, &added);
                if (rc) return rc;
                iterations += applied;
                total_new += added;
                if (applied) continue;
            }
        }

        // Size the candidate buffers: |J| <= sum over rules of |DELTA| * max degree,
        // so the capacity flag below only fires if that bound is not met.
        size_t max_status_words = 64;
        for (size_t k = 0; k < ex->rules.size(); ++k) {
            const u64 dn = st->find(ex->rules[k].delta_input)->delta_n;
            ex->host_rule_delta[k] = dn;
            max_status_words = std::max<size_t>(max_status_words, (dn + kJoinTile - 1) / kJoinTile + 1);
        }
        for (auto& t : ex->targets) {
            u64 bound = 0;
            for (size_t k : t.rules)
                bound += ex->host_rule_delta[k] * static_cast<u64>(std::max<u32>(ex->index[k].max_degree, 1));
            const u64 want = std::max<u64>(bound, 1024);
            if (t.j_cap < want) {
                const u64 cap = want + want / 4;
                SPK_CUDA(t.j_a.ensure(cap * 8, s), "cudaMallocAsync");
                SPK_CUDA(t.j_b.ensure(cap * 8, s), "cudaMallocAsync");
                t.j_cap = cap;
            }
        }
        for (;;) {
            for (auto& t : ex->targets) {
                SPK_CUDA(st->find(t.id)->newt.ensure(t.j_cap * 8, s), "cudaMallocAsync");
                // One status word per anti-join tile (the sparse kernel's
                // tiles are the smallest)...
                max_status_words =
                    std::max<size_t>(max_status_words, (t.j_cap + kSparseMinTile - 1) / kSparseMinTile + 1);
                // ...or the group-searched kernel's, over at most group_candidates.
                const u64 wide = std::min<u64>(t.j_cap, ex->tuning.group_candidates);
                const u64 wide_tile = kWideThreads / ex->tuning.group_lanes;
                max_status_words = std::max<size_t>(max_status_words, (wide + wide_tile - 1) / wide_tile + 1);
                // ...or the merge-form kernel's, over FULL and the candidates...
                if (ex->tuning.merge_anti_ratio)
                    max_status_words = std::max<size_t>(
                        max_status_words, (st->find(t.id)->full_rows() + t.j_cap + kAntiMergeTile - 1) / kAntiMergeTile + 1);
                // ...and per fused tile, which are DELTA-row tiles.
                u64 delta_rows = 0;
                for (size_t k : t.rules) delta_rows += ex->host_rule_delta[k];
                max_status_words = std::max<size_t>(max_status_words, (delta_rows + t.fused_rows - 1) / t.fused_rows + 1);
            }
            SPK_CUDA(ex->status.ensure_zeroed(max_status_words * 8, s), "cudaMallocAsync");
            SPK_CUDA(cudaMemsetAsync(counters, 0,
                                     (kCounterWords + 2 * ex->counts_words + kFusedFlagBase + kFusedMaxTargets) * 4, s),
                     "cudaMemsetAsync");
            size_t counter_slot = 0;
            // Targets whose single rule projects DELTA's first column (the
            // transitive-closure shape) run the fused round kernel; the rest
            // join, radix sort and anti-join with the general kernels.
            std::vector<char> fused(ex->targets.size(), 0);
            bool any_general = false;
            for (size_t ti = 0; ti < ex->targets.size(); ++ti) {
                fused[ti] = fused_eligible(ex, st, ti) ? 1 : 0;
                any_general |= !fused[ti];
            }
            if (any_general)  // the general join reads DELTA sizes on the device
                SPK_CUDA(cudaMemcpyAsync(ex->rule_delta.ptr, ex->host_rule_delta, ex->rules.size() * 8,
                                         cudaMemcpyHostToDevice, s),
                         "cudaMemcpyAsync");
            const int join_timing = ex->begin(SPARKALOG_K_JOIN, s);
            u64 join_launches = 0;
            // Joins: every rule appends into its target's candidate buffer.
            for (size_t ti = 0; ti < ex->targets.size(); ++ti) {
                TargetRT& t = ex->targets[ti];
                if (fused[ti]) continue;
                u64* tc = counts + target_count_base(ex, ti);
                for (size_t pos = 0; pos < t.rules.size(); ++pos) {
                    const size_t k = t.rules[pos];
                    const sparkalog_rule_plan& p = ex->rules[k];
                    RelState& d = *st->find(p.delta_input);
                    RelState& right = *st->find(p.right_input);
                    IndexCache& ic = ex->index[k];
                    spk::FusedJoinArgs a{};
                    a.delta = d.delta.as<u64>();
                    a.delta_count = ex->rule_delta.as<u64>() + k;
                    a.left_key = p.left_key;
                    if (ic.bucketed) {
                        a.dense_offsets = nullptr;
                        a.bucket_dir = ic.bucket_dir.as<u32>();
                        a.bucket_shift = ic.bucket_shift;
                        a.buckets = ic.buckets;
                        a.keys = ic.keys32.as<u32>();
                    } else {
                        a.dense_offsets = ic.offsets.as<u32>();
                        a.dense_keys = ic.num_keys;
                    }
                    a.rows = ic.identity ? nullptr : ic.rows.as<u32>();
                    a.right = right.level[0].as<u64>();
                    a.side[0] = p.proj_side[0];
                    a.side[1] = p.proj_side[1];
                    a.col[0] = p.proj_col[0];
                    a.col[1] = p.proj_col[1];
                    a.out = t.j_a.as<u64>();
                    a.capacity = t.j_cap;
                    a.count_in = tc + pos;
                    a.count_out = tc + pos + 1;
                    a.status = ex->status.as<u64>();
                    a.tile_counter = counters + counter_slot++;
                    a.epoch_ptr = nullptr;
                    a.epoch_add = ex->epoch++;
                    a.err = err;
                    auto kernel = spk::join_fused_kernel<kThreads, kJoinItems>;
                    const size_t tiles = (ex->host_rule_delta[k] + kJoinTile - 1) / kJoinTile;
                    kernel<<<grid_for(reinterpret_cast<const void*>(kernel), kThreads, std::max<size_t>(tiles, 1)),
                             kThreads, 0, s>>>(a);
                    SPK_CUDA(cudaGetLastError(), "join_fused_kernel");
                    ex->stats.total_launches += 1;
                    join_launches += 1;
                }
            }
            ex->end(join_timing, s, 0.0, join_launches);
            std::vector<int> hist_t(ex->targets.size(), -1), pass_t(ex->targets.size(), -1),
                anti_t(ex->targets.size(), -1), fused_t(ex->targets.size(), -1);
            std::vector<u64> anti_full(ex->targets.size(), 0);  // FULL rows a merge-form anti-join read
            // Distinct (radix sort) + unique/anti-join per target. The sort
            // reads the clamped candidate count from the device.
            for (size_t ti = 0; ti < ex->targets.size(); ++ti) {
                TargetRT& t = ex->targets[ti];
                u64* tc = counts + target_count_base(ex, ti);
                u64* jn = tc + t.rules.size();
                RelState& tr = *st->find(t.id);
                u64 dir_launches = 0;
                bool use_member = false;
                const bool use_bloom = ex->tuning.bloom_bits != 0 && tr.recursive && !ex->member_enabled;
                if (use_bloom) {
                    int rc = bloom_ready(tr, ex->tuning.bloom_bits, s, &dir_launches);
                    if (rc) return rc;
                } else {
                    tr.bloom_valid = false;  // this round's NEWT will not reach the filter
                }
                if (ex->member_enabled && tr.recursive) {
                    if (!tr.member_valid) {
                        int rc = member_build(tr, member_err, s, &dir_launches);
                        if (rc) return rc;
                    }
                    use_member = tr.member_valid;
                }
                if (!use_member) {
                    int rc = refresh_directories(st, tr, s, &dir_launches);
                    if (rc) return rc;
                }
                spk::Levels lv{};
                lv.n = 0;
                for (int l = 0; l < spk::kMaxLevels; ++l) {
                    if (tr.level_n[l] == 0) continue;
                    lv.keys[lv.n] = tr.level[l].as<u64>();
                    lv.count[lv.n] = tr.level_n[l];
                    lv.dir[lv.n] = tr.dir[l].as<u32>();
                    lv.shift[lv.n] = tr.dir_shift[l];
                    lv.buckets[lv.n] = tr.dir_buckets[l];
                    ++lv.n;
                }
                const u64* cand = nullptr;  // sorted candidates for the anti-join
                const u32* cand_sel = nullptr;
                if (fused[ti]) {
                    // Join + distinct in one kernel: the sorted distinct
                    // candidates land in j_a, their count in jn, the join
                    // output's size in the target's first count word.
                    const size_t k = t.rules[0];
                    const sparkalog_rule_plan& p = ex->rules[k];
                    RelState& d = *st->find(p.delta_input);
                    RelState& right = *st->find(p.right_input);
                    IndexCache& ic = ex->index[k];
                    spk::FusedRoundArgs a{};
                    a.delta = d.delta.as<u64>();
                    a.delta_rows = ex->host_rule_delta[k];
                    a.rows_per_tile = t.fused_rows;
                    a.left_key = p.left_key;
                    if (ic.bucketed) {
                        a.bucket_dir = ic.bucket_dir.as<u32>();
                        a.bucket_shift = ic.bucket_shift;
                        a.buckets = ic.buckets;
                        a.keys32 = ic.keys32.as<u32>();
                    } else {
                        a.dense_offsets = ic.offsets.as<u32>();
                        a.dense_keys = ic.num_keys;
                    }
                    a.rows = ic.identity ? nullptr : ic.rows.as<u32>();
                    a.right = right.level[0].as<u64>();
                    a.v1_side = p.proj_side[1];
                    a.v1_col = p.proj_col[1];
                    a.right_values = (ic.identity && !ic.bucketed && a.v1_side == 1 && a.v1_col == 1 && ic.num_keys)
                                         ? ic.values_ptr : nullptr;
                    a.key_class = (a.right_values && ex->tuning.compact_index) ? ic.key_class : nullptr;
                    a.key_word = a.key_class ? ic.key_word : nullptr;
                    a.v1_bits = static_cast<u32>(32 - __builtin_clz(st->max_value | 1));
                    a.out = t.j_a.as<u64>();
                    a.out_count = jn;
                    a.join_rows = reinterpret_cast<unsigned long long*>(tc);
                    a.status = ex->status.as<u64>();
                    a.tile_counter = counters + counter_slot++;
                    a.epoch = ex->epoch++;
                    a.err = err;
                    a.fallback = err + kFusedFlagBase + ti;
                    const size_t tiles = (a.delta_rows + a.rows_per_tile - 1) / a.rows_per_tile;
                    fused_t[ti] = ex->begin(SPARKALOG_K_FUSED, s);
                    int rc = launch_fused(a, tiles, s);
                    if (rc) return rc;
                    ex->end(fused_t[ti], s, 0.0, 1);
                    ex->stats.total_launches += 1;
                    cand = t.j_a.as<u64>();
                } else {
                    int rc = radix_sort(t.j_a.as<u64>(), t.j_b.as<u64>(), jn, t.j_cap, t.sort, ex, err, s,
                                        &hist_t[ti], &pass_t[ti]);
                    if (rc) return rc;
                    cand = t.j_a.as<u64>();
                    cand_sel = &t.sort.plan.as<spk::RadixPlan>()->final_sel;
                }
                anti_t[ti] = ex->begin(SPARKALOG_K_ANTI_JOIN, s);
                u64 cand_bound = 0;  // the join output bound: candidates never exceed it
                for (size_t k : t.rules)
                    cand_bound += ex->host_rule_delta[k] * static_cast<u64>(std::max<u32>(ex->index[k].max_degree, 1));
                // Distinct join rows of the target (round trace).
                unsigned long long* unique_word = reinterpret_cast<unsigned long long*>(tc + t.rules.size() + 2);
                // Merge form while FULL is within merge_anti_ratio times the
                // round's candidates (estimated from the last round's distinct
                // rows per DELTA row): reading FULL once then costs less than a
                // search per candidate.
                u64 full_rows = 0;
                int partner = 0;
                for (int l = 0; l < lv.n; ++l) {
                    full_rows += lv.count[l];
                    if (lv.count[l] > lv.count[partner]) partner = l;
                }
                u64 delta_rows = 0;
                for (size_t k : t.rules) delta_rows += ex->host_rule_delta[k];
                const double cand_estimate = t.unique_per_delta >= 0.0
                                                 ? t.unique_per_delta * static_cast<double>(delta_rows)
                                                 : static_cast<double>(cand_bound);
                const bool use_merge_form = ex->tuning.merge_anti_ratio != 0 && !use_bloom && !use_member && lv.n > 0 &&
                                            static_cast<double>(full_rows) <=
                                                static_cast<double>(ex->tuning.merge_anti_ratio) * cand_estimate;
                if (use_merge_form) {
                    const u64 tiles = (full_rows + t.j_cap + kAntiMergeTile - 1) / kAntiMergeTile;
                    SPK_CUDA(t.anti_plan.ensure(std::max<u64>(tiles, 1) * sizeof(spk::AntiTile), s), "cudaMallocAsync");
                    spk::AntiTile* plan = t.anti_plan.as<spk::AntiTile>();
                    {
                        const u64 blocks = std::min<u64>((tiles + 7) / 8, static_cast<u64>(spk::device_sm_count()) * 16);
                        spk::anti_merge_plan_kernel<kAntiMergeTile><<<static_cast<unsigned>(std::max<u64>(blocks, 1)), 256,
                                                                      0, s>>>(cand, t.j_b.as<u64>(), cand_sel, jn, lv,
                                                                              partner, plan);
                        SPK_CUDA(cudaGetLastError(), "anti_merge_plan_kernel");
                    }
                    using AL = spk::AntiMergeLayout<kAntiMergeThreads, kAntiMergeItems, kAntiMergeSide>;
                    auto kernel = spk::anti_merge_kernel<kAntiMergeThreads, kAntiMergeItems, kAntiMergeSide>;
                    static std::atomic<u64> configured{0};
                    int device = 0;
                    SPK_CUDA(cudaGetDevice(&device), "cudaGetDevice");
                    const u64 bit = 1ull << (device & 63);
                    if (!(configured.load() & bit)) {
                        SPK_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                      static_cast<int>(AL::kBytes)),
                                 "cudaFuncSetAttribute");
                        configured.fetch_or(bit);
                    }
                    const unsigned grid = spk::persistent_grid(reinterpret_cast<const void*>(kernel), kAntiMergeThreads,
                                                               AL::kBytes, std::max<u64>(tiles, 1));
                    SPK_CUDA(t.anti_scratch.ensure(t.j_cap * 8, s), "cudaMallocAsync");
                    SPK_CUDA(t.anti_counts.ensure((tiles + 1) * 4, s), "cudaMallocAsync");
                    kernel<<<grid, kAntiMergeThreads, AL::kBytes, s>>>(cand, t.j_b.as<u64>(), cand_sel, jn, lv, partner,
                                                                       plan, t.anti_scratch.as<u64>(),
                                                                       t.anti_counts.as<u32>(), err, unique_word);
                    SPK_CUDA(cudaGetLastError(), "anti_merge_kernel");
                    spk::anti_merge_scan_kernel<1024, kAntiMergeTile><<<1, 1024, 0, s>>>(
                        jn, lv, partner, t.anti_counts.as<u32>(), tc + t.rules.size() + 1);
                    SPK_CUDA(cudaGetLastError(), "anti_merge_scan_kernel");
                    {
                        const u64 blocks = std::min<u64>((tiles + 7) / 8 + 1, static_cast<u64>(spk::device_sm_count()) * 8);
                        spk::anti_merge_copy_kernel<<<static_cast<unsigned>(blocks), 256, 0, s>>>(
                            jn, lv, partner, kAntiMergeTile, plan, t.anti_scratch.as<u64>(), t.anti_counts.as<u32>(),
                            tr.newt.as<u64>());
                        SPK_CUDA(cudaGetLastError(), "anti_merge_copy_kernel");
                    }
                    anti_full[ti] = full_rows;
                    ex->stats.total_launches += 3;
                } else if (use_bloom) {
                    // The filter rules out most candidates with one sector each;
                    // the rest are searched in the levels.
                    auto kernel = spk::anti_join_bloom_kernel<kSparseThreads, kSparseItems>;
                    const size_t tiles = (cand_bound + kSparseTile - 1) / kSparseTile;
                    kernel<<<grid_for(reinterpret_cast<const void*>(kernel), kSparseThreads, std::max<size_t>(tiles, 1)),
                             kSparseThreads, 0, s>>>(cand, t.j_b.as<u64>(), cand_sel, jn, lv, bloom_of(tr),
                                                     tr.newt.as<u64>(), tc + t.rules.size() + 1, ex->status.as<u64>(),
                                                     counters + counter_slot++, ex->epoch++, err, unique_word);
                    SPK_CUDA(cudaGetLastError(), "anti_join_bloom_kernel");
                } else if (use_member) {
                    auto kernel = spk::anti_join_member_kernel<kThreads, kSetItems>;
                    const size_t tiles = (t.j_cap + kSetTile - 1) / kSetTile;
                    kernel<<<grid_for(reinterpret_cast<const void*>(kernel), kThreads, std::max<size_t>(tiles, 1)),
                             kThreads, 0, s>>>(cand, t.j_b.as<u64>(), cand_sel, jn, member_set(tr),
                                               tr.newt.as<u64>(), tc + t.rules.size() + 1, ex->status.as<u64>(),
                                               counters + counter_slot++, ex->epoch++, err, unique_word);
                    SPK_CUDA(cudaGetLastError(), "anti_join_member_kernel");
                } else if (cand_bound <= ex->tuning.group_candidates) {
                    // A few candidates: lookup latency dominates, so a group
                    // of lanes searches each one together.
                    auto kernel = spk::anti_join_levels_wide_kernel<kWideThreads, 8>;
                    if (ex->tuning.group_lanes == 4) kernel = spk::anti_join_levels_wide_kernel<kWideThreads, 4>;
                    if (ex->tuning.group_lanes == 16) kernel = spk::anti_join_levels_wide_kernel<kWideThreads, 16>;
                    const u64 wide_tile = kWideThreads / ex->tuning.group_lanes;
                    const size_t tiles = (cand_bound + wide_tile - 1) / wide_tile;
                    kernel<<<grid_for(reinterpret_cast<const void*>(kernel), kWideThreads, std::max<size_t>(tiles, 1)),
                             kWideThreads, 0, s>>>(cand, t.j_b.as<u64>(), cand_sel, jn, lv, tr.newt.as<u64>(),
                                                   tc + t.rules.size() + 1, ex->status.as<u64>(),
                                                   counters + counter_slot++, ex->epoch++, err, unique_word);
                    SPK_CUDA(cudaGetLastError(), "anti_join_levels_wide_kernel");
                } else if (cand_bound <= ex->tuning.sparse_candidates) {
                    // Few candidates, far apart in every level: look each up
                    // in all levels at once.
                    const u32 items = ex->tuning.sparse_items;
                    const bool three = lv.n <= 3;
                    auto kernel = three ? spk::anti_join_levels_sparse_kernel<kSparseThreads, 4, 3>
                                        : spk::anti_join_levels_sparse_kernel<kSparseThreads, 4, 4>;
                    if (items == 3)
                        kernel = three ? spk::anti_join_levels_sparse_kernel<kSparseThreads, 3, 3>
                                       : spk::anti_join_levels_sparse_kernel<kSparseThreads, 3, 4>;
                    if (items == 2)
                        kernel = three ? spk::anti_join_levels_sparse_kernel<kSparseThreads, 2, 3>
                                       : spk::anti_join_levels_sparse_kernel<kSparseThreads, 2, 4>;
                    const u64 tile_rows = static_cast<u64>(kSparseThreads) * items;
                    const size_t tiles = (cand_bound + tile_rows - 1) / tile_rows;
                    kernel<<<grid_for(reinterpret_cast<const void*>(kernel), kSparseThreads, std::max<size_t>(tiles, 1)),
                             kSparseThreads, 0, s>>>(cand, t.j_b.as<u64>(), cand_sel, jn, lv, tr.newt.as<u64>(),
                                                     tc + t.rules.size() + 1, ex->status.as<u64>(),
                                                     counters + counter_slot++, ex->epoch++, err, unique_word);
                    SPK_CUDA(cudaGetLastError(), "anti_join_levels_sparse_kernel");
                } else {
                    auto kernel = spk::anti_join_levels_kernel<kThreads, kSetItems, kLevelStage>;
                    const size_t tiles = (t.j_cap + kSetTile - 1) / kSetTile;
                    kernel<<<grid_for(reinterpret_cast<const void*>(kernel), kThreads, std::max<size_t>(tiles, 1)),
                             kThreads, 0, s>>>(cand, t.j_b.as<u64>(), cand_sel, jn, lv, tr.newt.as<u64>(),
                                               tc + t.rules.size() + 1, ex->status.as<u64>(), counters + counter_slot++,
                                               ex->epoch++, err, unique_word);
                    SPK_CUDA(cudaGetLastError(), "anti_join_levels_kernel");
                }
                ex->end(anti_t[ti], s, 0.0, use_merge_form ? 4 : 1);
                ex->stats.total_launches += 1 + dir_launches;
                if (!fused[ti])
                    SPK_CUDA(cudaMemcpyAsync(ex->host_active + ti * spk::kMaxPasses,
                                             t.sort.plan.as<spk::RadixPlan>()->active, spk::kMaxPasses * 4,
                                             cudaMemcpyDeviceToHost, s),
                             "cudaMemcpyAsync");
            }
            // The round's only host synchronisation: counts and error bits.
            SPK_CUDA(cudaMemcpyAsync(ex->host_counts, counts,
                                     ex->counts_words * 8 + (kFusedFlagBase + kFusedMaxTargets) * 4,
                                     cudaMemcpyDeviceToHost, s),
                     "cudaMemcpyAsync");
            SPK_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
            const u32 bits = static_cast<u32>(ex->host_counts[ex->counts_words] & 0xffffffffu);
            const u32* flags = reinterpret_cast<const u32*>(ex->host_counts + ex->counts_words) + kFusedFlagBase;
            if (ex->profiling) {
                // Algorithmic bytes (each input row read once, each output written once).
                double join_bytes = 0.0;
                for (size_t ti = 0; ti < ex->targets.size(); ++ti) {
                    const TargetRT& t = ex->targets[ti];
                    if (!fused[ti])
                        for (size_t k : t.rules) join_bytes += 16.0 * ex->host_rule_delta[k];
                    const double jn = static_cast<double>(ex->host_counts[target_count_base(ex, ti) + t.rules.size()]);
                    const double nn =
                        static_cast<double>(ex->host_counts[target_count_base(ex, ti) + t.rules.size() + 1]);
                    if (!fused[ti]) join_bytes += 12.0 * jn;
                    u64 active = 0;
                    for (int p = 0; p < spk::kMaxPasses; ++p) active += ex->host_active[ti * spk::kMaxPasses + p] ? 1 : 0;
                    if (hist_t[ti] >= 0) ex->timings[hist_t[ti]].bytes = 8.0 * jn;
                    if (pass_t[ti] >= 0) {
                        ex->timings[pass_t[ti]].bytes = 16.0 * jn * static_cast<double>(active);
                        ex->timings[pass_t[ti]].launches = active;
                    }
                    // The merge form reads FULL once as well.
                    if (anti_t[ti] >= 0)
                        ex->timings[anti_t[ti]].bytes = 8.0 * jn + 8.0 * nn + 8.0 * static_cast<double>(anti_full[ti]);
                    if (fused_t[ti] >= 0) {
                        // DELTA rows and their index entries, the joined right
                        // rows, the distinct candidates out.
                        const double delta_rows = static_cast<double>(ex->host_rule_delta[t.rules[0]]);
                        const double joined = static_cast<double>(ex->host_counts[target_count_base(ex, ti)]);
                        ex->timings[fused_t[ti]].bytes = 16.0 * delta_rows + 8.0 * joined + 8.0 * jn;
                    }
                }
                if (join_timing >= 0) ex->timings[join_timing].bytes = join_bytes;
                ex->collect();
            }
            bool redo_generic = false;
            for (size_t ti = 0; ti < ex->targets.size(); ++ti) {
                if (!fused[ti] || !flags[ti]) continue;
                // A fused tile overflowed shared memory: redo this round with the
                // general kernels and use smaller tiles from now on.
                TargetRT& t = ex->targets[ti];
                t.force_generic = true;
                if (t.fused_rows > 64) t.fused_rows /= 2;
                t.fused_rows_cap = std::min(t.fused_rows_cap, t.fused_rows);
                redo_generic = true;
            }
            if (redo_generic) {
                SPK_CUDA(cudaMemsetAsync(err, 0, 4, s), "cudaMemsetAsync");
                continue;
            }
            for (size_t ti = 0; ti < ex->targets.size(); ++ti) ex->targets[ti].fused_last = fused[ti] != 0;
            if (!(bits & spk::kErrCapacity)) break;
            // A candidate buffer overflowed: grow it and redo the round (no
            // relation state has changed yet).
            for (auto& t : ex->targets) {
                const u64 cap = t.j_cap * 2;
                SPK_CUDA(t.j_a.ensure(cap * 8, s), "cudaMallocAsync");
                SPK_CUDA(t.j_b.ensure(cap * 8, s), "cudaMallocAsync");
                t.j_cap = cap;
            }
            SPK_CUDA(cudaMemsetAsync(err, 0, 4, s), "cudaMemsetAsync");
        }

        for (auto& t : ex->targets) t.force_generic = false;
        const u32 err_bits = static_cast<u32>(ex->host_counts[ex->counts_words] & 0xffffffffu);
        if (err_bits & ~spk::kErrCapacity)
            return fail(SPARKALOG_E_DEVICE_FAULT, "device error bits " + std::to_string(err_bits));

        // Row ids (directories, join indexes) are u32: refuse the round before
        // any relation changes if a FULL would outgrow them.
        for (size_t ti = 0; ti < ex->targets.size(); ++ti) {
            const TargetRT& t = ex->targets[ti];
            const u64 newt_n = ex->host_counts[target_count_base(ex, ti) + t.rules.size() + 1];
            if (st->find(t.id)->full_rows() + newt_n > kMaxRelationRows)
                return fail(SPARKALOG_E_TOO_MANY_ROWS, "relation would exceed 2^32 - 1 rows (u32 row ids)");
        }

        // TargetRuntime::apply: FULL u= NEWT (into the levels), DELTA <- NEWT.
        for (size_t ti = 0; ti < ex->targets.size(); ++ti) {
            TargetRT& t = ex->targets[ti];
            RelState& tr = *st->find(t.id);
            const u64 newt_n = ex->host_counts[target_count_base(ex, ti) + t.rules.size() + 1];
            if (newt_n > 0) {
                // TAIL <- TAIL u NEWT
                const int tail = static_cast<int>(ex->tuning.levels) - 1;
                const u64 tn = tr.level_n[tail] + newt_n;
                {
                    u64 launched = 0;
                    int rc = merge_buffers(st, tr, tail, tn, s);
                    if (rc) return rc;
                    const int tm = ex->begin(SPARKALOG_K_MERGE, s);
                    rc = merge_into_level(st, tr, tail, tr.level[tail].as<u64>(), tr.level_n[tail],
                                          tr.newt.as<u64>(), newt_n, s, &launched);
                    if (rc) return rc;
                    ex->end(tm, s, 16.0 * static_cast<double>(tn), launched);
                    ex->stats.total_launches += launched;
                }
                int rc = cascade_levels(ex, st, tr);
                if (rc) return rc;
            }
            {
                // FULL's hash set takes the round's new rows (or is dropped
                // and rebuilt larger next round).
                u64 launched = 0;
                int rc = member_add(tr, tr.newt.as<u64>(), newt_n, member_err, s, &launched);
                if (rc) return rc;
                ex->stats.total_launches += launched;
            }
            if (ex->seg_count && newt_n > 0) {
                spk::segment_activity_kernel<<<simple_grid(newt_n), 256, 0, s>>>(
                    tr.newt.as<u64>(), newt_n, ex->seg_shift, ex->seg_count, static_cast<u32>(ex->rounds_total + 1),
                    ex->seg_seen.as<u32>(), ex->seg_new.as<unsigned long long>());
                SPK_CUDA(cudaGetLastError(), "segment_activity_kernel");
                ex->stats.total_launches += 1;
            }
            swap_arrays(tr.delta, tr.newt);
            tr.delta_n = newt_n;
            tr.delta_sorted = true;
            tr.version += 1;
            total_new += newt_n;
        }
        iterations += 1;
        ex->stats.rounds += 1;
        ex->rounds_total += 1;
        {
            sparkalog_round_trace rec{};
            rec.round = ex->rounds_total;
            for (size_t ti = 0; ti < ex->targets.size(); ++ti) {
                const TargetRT& t = ex->targets[ti];
                const u64* c = ex->host_counts + target_count_base(ex, ti);
                for (size_t k : t.rules) rec.delta_rows += ex->host_rule_delta[k];
                // A fused target counts its join rows in the first word; the
                // general join chains its per-rule counts up to word rules.
                rec.join_rows += t.fused_last ? c[0] : c[t.rules.size()];
                rec.new_rows += c[t.rules.size() + 1];
                rec.unique_rows += c[t.rules.size() + 2];
                rec.full_rows += st->find(t.id)->full_rows();
            }
            if (ex->trace.size() < kMaxTraceRounds) ex->trace.push_back(rec);
        }
        // Rows per fused tile for the next round: a tile holds kFusedCap join
        // rows, so aim at two thirds of that with this round's join rows per
        // DELTA row (dense graphs get short tiles instead of overflowing).
        for (size_t ti = 0; ti < ex->targets.size(); ++ti) {
            TargetRT& t = ex->targets[ti];
            u64 delta_rows = 0;
            for (size_t k : t.rules) delta_rows += ex->host_rule_delta[k];
            if (delta_rows == 0) continue;
            const u64* c = ex->host_counts + target_count_base(ex, ti);
            const double per_row = static_cast<double>(t.fused_last ? c[0] : c[t.rules.size()]) /
                                   static_cast<double>(delta_rows);
            const double rows = kFusedCap / (1.5 * std::max(per_row, 1e-3));
            t.fused_rows = static_cast<u32>(std::max(64.0, std::min<double>(t.fused_rows_cap, rows)));
            t.unique_per_delta = static_cast<double>(c[t.rules.size() + 2]) / static_cast<double>(delta_rows);
        }
    }
    u32* member_err_host = reinterpret_cast<u32*>(ex->host_counts + ex->counts_words + 30);
    SPK_CUDA(cudaMemcpyAsync(member_err_host, member_err, 4, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync");
    SPK_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    ex->collect();
    if (*member_err_host)
        return fail(SPARKALOG_E_DEVICE_FAULT, "device error bits " + std::to_string(*member_err_host) +
                                                  " (hash set of FULL)");
    {
        const int rc = check_store_fault(st);
        if (rc) return rc;
    }
    if (summary) {
        summary->iterations = iterations;
        summary->total_new_rows = total_new;
        if (summary->relation_ids && summary->relation_rows) {
            const size_t n = std::min<size_t>(summary->relation_count, ex->relations.size());
            for (size_t i = 0; i < n; ++i) {
                summary->relation_ids[i] = ex->relations[i];
                summary->relation_rows[i] = st->find(ex->relations[i])->full_rows();
            }
        }
        summary->relation_count = ex->relations.size();
    }
    if (converged) {
        bool any = false;
        for (u32 id : ex->relations) any |= st->find(id)->delta_n != 0;
        *converged = any ? 0 : 1;
    }
    return 0;
}

int sparkalog_executor_run(sparkalog_executor* ex, sparkalog_store* st, size_t max_iterations,
                           sparkalog_scc_summary* summary) {
    return run_rounds(ex, st, max_iterations, true, summary, nullptr);
}

int sparkalog_executor_step(sparkalog_executor* ex, sparkalog_store* st, size_t rounds,
                            sparkalog_scc_summary* summary, int* converged) {
    return run_rounds(ex, st, rounds, false, summary, converged);
}

}  // extern "C"
