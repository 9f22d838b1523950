// Reference-compatible C ABI of the binary recursive operator pipeline.
//
// Each entry point keeps the signature, argument meaning, null-pointer checks
// and empty-input behaviour of the reference's launcher of the same name in
// crates/sparkalog-execution/native/column_ops.cu (declared on the Rust side at
// crates/sparkalog-execution/src/lib.rs:28-169), so the Rust wrappers
// join_cuda / distinct_cuda / anti_join_cuda / union_cuda link against this
// library unchanged. The kernels behind them are this project's own (no CUB or
// Thrust). `temporary` holds look-back status words, tile counters and the
// radix plan; `*_temporary_bytes` reports its size for the given row counts.
//
// Outputs are written asynchronously on `stream`; counts land in device (or
// managed) memory, exactly as in the reference, and the caller synchronizes
// before reading them.

#include "sparkalog_b200.h"
#include "spk_common.cuh"
#include "spk_host.h"
#include "spk_join.cuh"
#include "spk_radix.cuh"
#include "spk_setops.cuh"

#include <algorithm>
#include <mutex>
#include <vector>

using spk::u32;
using spk::u64;

namespace spk {

int device_sm_count() {
    static std::mutex mu;
    static std::vector<int> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    if (static_cast<int>(cache.size()) <= dev) cache.resize(dev + 1, 0);
    if (cache[dev] == 0) {
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cache[dev] = sms > 0 ? sms : 1;
    }
    return cache[dev];
}

unsigned int persistent_grid(const void* kernel, int threads, size_t dynamic_smem, size_t tiles) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, dynamic_smem) != cudaSuccess ||
        per_sm <= 0) {
        cudaGetLastError();
        per_sm = 1;
    }
    size_t grid = static_cast<size_t>(per_sm) * device_sm_count();
    if (tiles < grid) grid = tiles;
    if (grid == 0) grid = 1;
    return static_cast<unsigned int>(grid);
}

}  // namespace spk

namespace {

constexpr int kThreads = 256;
constexpr int kSetItems = 8;                       // rows per thread in set/compaction kernels
constexpr int kSetTile = kThreads * kSetItems;
constexpr int kJoinItems = 8;
constexpr int kJoinTile = kThreads * kJoinItems;
constexpr int kSortThreads = spk::RadixSortConfig::kThreads;
constexpr int kSortItems = spk::RadixSortConfig::kItems;

// Packs (first, second) SoA rows into u64 keys and builds the histograms of
// all radix passes in the same read (pack_binary_u32 + the sort's upsweep).
template <int THREADS>
__global__ void __launch_bounds__(THREADS) pack_histogram_kernel(const u32* first, const u32* second, u64 n,
                                                                 u64* packed, spk::RadixPlan* plan, int passes) {
    __shared__ u32 sh[spk::kMaxPasses][spk::kRadix];
    for (int i = threadIdx.x; i < spk::kMaxPasses * spk::kRadix; i += THREADS) (&sh[0][0])[i] = 0;
    __syncthreads();
    const u64 stride = static_cast<u64>(gridDim.x) * THREADS;
    const u64 rounds = (n + stride - 1) / stride;
    for (u64 r = 0; r < rounds; ++r) {
        const u64 i = static_cast<u64>(blockIdx.x) * THREADS + threadIdx.x + r * stride;
        const bool valid = i < n;
        u64 k = 0;
        if (valid) {
            k = spk::pack2(first[i], second[i]);
            packed[i] = k;
        }
        for (int p = 0; p < passes; ++p) {
            const u32 d = valid ? static_cast<u32>((k >> (p * spk::kRadixBits)) & (spk::kRadix - 1)) : spk::kRadix;
            spk::warp_histogram_add(sh[p], d);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * spk::kRadix; i += THREADS) {
        const u32 c = (&sh[0][0])[i];
        if (c) atomicAdd(&plan->hist[0][0] + i, c);
    }
}

// Scratch layouts. Every region that look-back or a tile counter uses is
// cleared with one cudaMemsetAsync at the start of a call; the kernels of one
// call use distinct epochs, so regions can be shared across kernels.
struct JoinTemp {
    u64* status;
    u32* counter;
    size_t bytes;
    size_t clear_bytes;
};
JoinTemp join_temp(void* base, size_t left_rows) {
    spk::Carver c(base);
    JoinTemp t{};
    t.counter = c.take<u32>(64);
    t.status = c.take<u64>((left_rows + kJoinTile - 1) / kJoinTile + 1);
    t.bytes = spk::align_up(c.used, 256);
    t.clear_bytes = t.bytes;
    return t;
}

struct DistinctTemp {
    spk::RadixPlan* plan;
    u64* radix_status;
    u64* unique_status;
    u32* counter;
    size_t bytes;
    size_t clear_bytes;
};
DistinctTemp distinct_temp(void* base, size_t rows) {
    spk::Carver c(base);
    DistinctTemp t{};
    t.plan = c.take<spk::RadixPlan>(1);
    t.counter = c.take<u32>(64);
    t.unique_status = c.take<u64>((rows + kSetTile - 1) / kSetTile + 1);
    t.radix_status = c.take<u64>(spk::radix_status_words(rows));
    t.bytes = spk::align_up(c.used, 256);
    t.clear_bytes = t.bytes;
    return t;
}

struct SetTemp {
    u64* status;
    u32* counter;
    size_t bytes;
};
SetTemp set_temp(void* base, size_t rows) {
    spk::Carver c(base);
    SetTemp t{};
    t.counter = c.take<u32>(64);
    t.status = c.take<u64>((rows + kSetTile - 1) / kSetTile + 1);
    t.bytes = spk::align_up(c.used, 256);
    return t;
}

u32* device_error_word() {
    // One error word per device for asynchronous kernel faults that the
    // reference ABI has no output for (look-back timeouts); read it with
    // sparkalog_b200_device_error.
    static std::mutex mu;
    static std::vector<u32*> words;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    if (static_cast<int>(words.size()) <= dev) words.resize(dev + 1, nullptr);
    if (!words[dev]) {
        void* p = nullptr;
        if (cudaMalloc(&p, 256) != cudaSuccess) return nullptr;
        cudaMemset(p, 0, 256);
        words[dev] = static_cast<u32*>(p);
    }
    return words[dev];
}

}  // namespace

extern "C" {

int sparkalog_stream_synchronize(void* stream) {
    return cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
}

// Reads (and with reset != 0 clears) this device's asynchronous error bits.
int sparkalog_b200_device_error(u32* bits, int reset) {
    if (bits == nullptr) return cudaErrorInvalidValue;
    u32* word = device_error_word();
    if (!word) return cudaErrorMemoryAllocation;
    cudaError_t st = cudaMemcpy(bits, word, sizeof(u32), cudaMemcpyDeviceToHost);
    if (st == cudaSuccess && reset) st = cudaMemset(word, 0, sizeof(u32));
    return st;
}

// ---------------------------------------------------------------------------
// Join. column_ops.cu:339-444.
// ---------------------------------------------------------------------------

int sparkalog_join_u32_temporary_bytes(const u64* counts, u64* offsets, size_t left_rows,
                                               size_t* temporary_bytes, void* stream) {
    (void)stream;
    if (temporary_bytes == nullptr || (left_rows != 0 && (counts == nullptr || offsets == nullptr))) {
        return cudaErrorInvalidValue;
    }
    *temporary_bytes = join_temp(nullptr, left_rows).bytes;
    return cudaSuccess;
}

int sparkalog_join_u32_count(const u32* left_keys, size_t left_rows, const u32* index_keys,
                                     const u32* index_starts, size_t unique_keys, u64* counts, u64* offsets,
                                     u64* total, void* temporary, size_t temporary_bytes, void* stream) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (total == nullptr) return cudaErrorInvalidValue;
    if (left_rows == 0) return cudaMemsetAsync(total, 0, sizeof(*total), s);
    if (left_keys == nullptr || index_keys == nullptr || index_starts == nullptr || counts == nullptr ||
        offsets == nullptr || temporary == nullptr) {
        return cudaErrorInvalidValue;
    }
    JoinTemp t = join_temp(temporary, left_rows);
    if (temporary_bytes < t.bytes) return cudaErrorInvalidValue;
    u32* err = device_error_word();
    if (!err) return cudaErrorMemoryAllocation;
    cudaError_t st = cudaMemsetAsync(temporary, 0, t.clear_bytes, s);
    if (st != cudaSuccess) return st;
    const size_t tiles = (left_rows + kJoinTile - 1) / kJoinTile;
    auto kernel = spk::join_count_scan_kernel<kThreads, kJoinItems>;
    const unsigned grid = spk::persistent_grid(reinterpret_cast<const void*>(kernel), kThreads, 0, tiles);
    kernel<<<grid, kThreads, 0, s>>>(left_keys, left_rows, index_keys, index_starts, unique_keys, counts, offsets,
                                     total, t.status, t.counter, 1u, err);
    return cudaGetLastError();
}

int sparkalog_join_u32_emit(const u32* left_keys, size_t left_rows, const u32* index_keys,
                                    const u32* index_starts, const u32* index_rows, size_t unique_keys,
                                    const u32* projection0, u32 projection0_side, const u32* projection1,
                                    u32 projection1_side, const u64* offsets, u32* output0, u32* output1,
                                    void* stream) {
    if (left_rows == 0) return cudaSuccess;
    if (left_keys == nullptr || index_keys == nullptr || index_starts == nullptr || index_rows == nullptr ||
        projection0 == nullptr || projection1 == nullptr || offsets == nullptr || output0 == nullptr ||
        output1 == nullptr) {
        return cudaErrorInvalidValue;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t tiles = (left_rows + kJoinTile - 1) / kJoinTile;
    auto kernel = spk::join_emit_kernel<kThreads, kJoinItems>;
    const unsigned grid = spk::persistent_grid(reinterpret_cast<const void*>(kernel), kThreads, 0, tiles);
    kernel<<<grid, kThreads, 0, s>>>(left_keys, left_rows, index_keys, index_starts, index_rows, unique_keys,
                                     projection0, projection0_side, projection1, projection1_side, offsets, output0,
                                     output1);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Distinct. column_ops.cu:446-549. `packed` and `scratch` are the radix sort's
// ping-pong buffers, as in the reference.
// ---------------------------------------------------------------------------

int sparkalog_distinct_u32_temporary_bytes(u64* packed, u64* scratch, u64* unique_rows, size_t rows,
                                                   size_t* temporary_bytes, void* stream) {
    (void)stream;
    if (temporary_bytes == nullptr || unique_rows == nullptr) return cudaErrorInvalidValue;
    if (rows != 0 && (packed == nullptr || scratch == nullptr)) return cudaErrorInvalidValue;
    *temporary_bytes = distinct_temp(nullptr, rows).bytes;
    return cudaSuccess;
}

int sparkalog_distinct_u32(const u32* first, const u32* second, size_t rows, u64* packed, u64* scratch,
                                   u64* unique_rows, u32* output_first, u32* output_second, void* temporary,
                                   size_t temporary_bytes, void* stream) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (unique_rows == nullptr) return cudaErrorInvalidValue;
    if (rows == 0) return cudaMemsetAsync(unique_rows, 0, sizeof(*unique_rows), s);
    if (first == nullptr || second == nullptr || packed == nullptr || scratch == nullptr ||
        output_first == nullptr || output_second == nullptr || temporary == nullptr) {
        return cudaErrorInvalidValue;
    }
    if (rows > 0xffffffffull) return cudaErrorInvalidValue;
    DistinctTemp t = distinct_temp(temporary, rows);
    if (temporary_bytes < t.bytes) return cudaErrorInvalidValue;
    u32* err = device_error_word();
    if (!err) return cudaErrorMemoryAllocation;
    cudaError_t st = cudaMemsetAsync(temporary, 0, t.clear_bytes, s);
    if (st != cudaSuccess) return st;

    constexpr int kPasses = 8;
    {
        auto kernel = pack_histogram_kernel<kThreads>;
        const size_t blocks = (rows + kThreads - 1) / kThreads;
        const unsigned grid = spk::persistent_grid(reinterpret_cast<const void*>(kernel), kThreads, 0, blocks);
        kernel<<<grid, kThreads, 0, s>>>(first, second, rows, packed, t.plan, kPasses);
    }
    spk::radix_plan<<<1, spk::kRadix, 0, s>>>(t.plan, nullptr, rows, kPasses);
    {
        auto kernel = spk::radix_pass<kSortThreads, kSortItems>;
        const size_t tiles = (rows + spk::RadixSortConfig::kTile - 1) / spk::RadixSortConfig::kTile;
        const unsigned grid = spk::persistent_grid(reinterpret_cast<const void*>(kernel), kSortThreads, 0, tiles);
        for (int p = 0; p < kPasses; ++p) {
            kernel<<<grid, kSortThreads, 0, s>>>(packed, scratch, t.plan, t.plan, p, p * spk::kRadixBits,
                                                 t.radix_status, nullptr, 1u + p, err);
        }
    }
    {
        auto kernel = spk::unique_unpack_kernel<kThreads, kSetItems>;
        const size_t tiles = (rows + kSetTile - 1) / kSetTile;
        const unsigned grid = spk::persistent_grid(reinterpret_cast<const void*>(kernel), kThreads, 0, tiles);
        kernel<<<grid, kThreads, 0, s>>>(packed, scratch, &t.plan->final_sel, rows, output_first, output_second,
                                         unique_rows, t.unique_status, t.counter, 1u + kPasses, err);
    }
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Anti-join. column_ops.cu:551-641. flags/selected/selected_rows keep the
// reference's meaning (1 = kept, kept row ids, their u32 count).
// ---------------------------------------------------------------------------

int sparkalog_anti_join_u32_temporary_bytes(const u32* flags, u32* selected, u32* selected_rows,
                                                    size_t left_rows, size_t* temporary_bytes, void* stream) {
    (void)stream;
    if (temporary_bytes == nullptr || selected_rows == nullptr) return cudaErrorInvalidValue;
    if (left_rows != 0 && (flags == nullptr || selected == nullptr)) return cudaErrorInvalidValue;
    *temporary_bytes = set_temp(nullptr, left_rows).bytes;
    return cudaSuccess;
}

int sparkalog_anti_join_u32(const u32* left_first, const u32* left_second, size_t left_rows,
                                    const u32* right_first, const u32* right_second, size_t right_rows, u32* flags,
                                    u32* selected, u32* selected_rows, u32* output_first, u32* output_second,
                                    void* temporary, size_t temporary_bytes, void* stream) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (selected_rows == nullptr) return cudaErrorInvalidValue;
    if (left_rows == 0) return cudaMemsetAsync(selected_rows, 0, sizeof(*selected_rows), s);
    if (left_first == nullptr || left_second == nullptr || flags == nullptr || selected == nullptr ||
        output_first == nullptr || output_second == nullptr || temporary == nullptr ||
        (right_rows != 0 && (right_first == nullptr || right_second == nullptr))) {
        return cudaErrorInvalidValue;
    }
    SetTemp t = set_temp(temporary, left_rows);
    if (temporary_bytes < t.bytes) return cudaErrorInvalidValue;
    u32* err = device_error_word();
    if (!err) return cudaErrorMemoryAllocation;
    cudaError_t st = cudaMemsetAsync(temporary, 0, t.bytes, s);
    if (st != cudaSuccess) return st;
    auto kernel = spk::anti_join_soa_kernel<kThreads, kSetItems>;
    const size_t tiles = (left_rows + kSetTile - 1) / kSetTile;
    const unsigned grid = spk::persistent_grid(reinterpret_cast<const void*>(kernel), kThreads, 0, tiles);
    kernel<<<grid, kThreads, 0, s>>>(left_first, left_second, left_rows, right_first, right_second, right_rows, flags,
                                     selected, selected_rows, output_first, output_second, t.status, t.counter, 1u,
                                     err);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Filter, fill and add-one. column_ops.cu:231-246, 252-336.
// ---------------------------------------------------------------------------

int sparkalog_filter_u32_temporary_bytes(const u32* flags, u32* output, u32* count, size_t len,
                                         size_t* temporary_bytes, void* stream) {
    (void)stream;
    if (temporary_bytes == nullptr || count == nullptr) return cudaErrorInvalidValue;
    if (len != 0 && (flags == nullptr || output == nullptr)) return cudaErrorInvalidValue;
    *temporary_bytes = set_temp(nullptr, len).bytes;
    return cudaSuccess;
}

int sparkalog_filter_u32(const u32* input, size_t len, u32 operation, u32 operand, u32* flags, u32* output,
                         u32* count, void* temporary, size_t temporary_bytes, void* stream) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (count == nullptr) return cudaErrorInvalidValue;
    if (len == 0) return cudaMemsetAsync(count, 0, sizeof(*count), s);
    if (input == nullptr || flags == nullptr || output == nullptr || temporary == nullptr)
        return cudaErrorInvalidValue;
    SetTemp t = set_temp(temporary, len);
    if (temporary_bytes < t.bytes) return cudaErrorInvalidValue;
    u32* err = device_error_word();
    if (!err) return cudaErrorMemoryAllocation;
    cudaError_t st = cudaMemsetAsync(temporary, 0, t.bytes, s);
    if (st != cudaSuccess) return st;
    auto kernel = spk::filter_select_kernel<kThreads, kSetItems>;
    const size_t tiles = (len + kSetTile - 1) / kSetTile;
    const unsigned grid = spk::persistent_grid(reinterpret_cast<const void*>(kernel), kThreads, 0, tiles);
    kernel<<<grid, kThreads, 0, s>>>(input, len, operation, operand, flags, output, count, t.status, t.counter, 1u,
                                     err);
    return cudaGetLastError();
}

int sparkalog_fill_mod_u32(u32* output, size_t len, u32 modulus, void* stream) {
    if (modulus == 0 || (output == nullptr && len != 0)) return cudaErrorInvalidValue;
    if (len == 0) return cudaSuccess;
    const size_t blocks = std::min<size_t>((len + 255) / 256, static_cast<size_t>(spk::device_sm_count()) * 8);
    spk::fill_mod_kernel<<<static_cast<unsigned>(blocks), 256, 0, static_cast<cudaStream_t>(stream)>>>(output, len,
                                                                                                        modulus);
    return cudaGetLastError();
}

int sparkalog_add_one_i32(int32_t* data, size_t len, void* stream) {
    if (data == nullptr && len != 0) return cudaErrorInvalidValue;
    if (len == 0) return cudaSuccess;
    const size_t blocks = std::min<size_t>((len + 255) / 256, static_cast<size_t>(spk::device_sm_count()) * 8);
    spk::add_one_kernel<<<static_cast<unsigned>(blocks), 256, 0, static_cast<cudaStream_t>(stream)>>>(data, len);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Union. column_ops.cu:643-775. `left`, `right`, `merged` and `unique` are the
// reference's packed scratch buffers; this implementation merges straight
// from the SoA columns and does not need them, but validates them the same
// way so error behaviour is unchanged.
// ---------------------------------------------------------------------------

int sparkalog_union_u32_temporary_bytes(const u64* left, size_t left_rows, const u64* right,
                                                size_t right_rows, u64* merged, u64* unique, u64* unique_rows,
                                                size_t* temporary_bytes, void* stream) {
    (void)stream;
    const size_t total = left_rows + right_rows;
    if (temporary_bytes == nullptr || unique_rows == nullptr) return cudaErrorInvalidValue;
    if ((left_rows != 0 && left == nullptr) || (right_rows != 0 && right == nullptr) ||
        (total != 0 && (merged == nullptr || unique == nullptr))) {
        return cudaErrorInvalidValue;
    }
    *temporary_bytes = set_temp(nullptr, total).bytes;
    return cudaSuccess;
}

int sparkalog_union_u32(const u32* left_first, const u32* left_second, size_t left_rows,
                                const u32* right_first, const u32* right_second, size_t right_rows, u64* left,
                                u64* right, u64* merged, u64* unique, u64* unique_rows, u32* output_first,
                                u32* output_second, void* temporary, size_t temporary_bytes, void* stream) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t total = left_rows + right_rows;
    if (unique_rows == nullptr) return cudaErrorInvalidValue;
    if (total == 0) return cudaMemsetAsync(unique_rows, 0, sizeof(*unique_rows), s);
    if ((left_rows != 0 && (left_first == nullptr || left_second == nullptr || left == nullptr)) ||
        (right_rows != 0 && (right_first == nullptr || right_second == nullptr || right == nullptr)) ||
        merged == nullptr || unique == nullptr || output_first == nullptr || output_second == nullptr ||
        temporary == nullptr) {
        return cudaErrorInvalidValue;
    }
    SetTemp t = set_temp(temporary, total);
    if (temporary_bytes < t.bytes) return cudaErrorInvalidValue;
    u32* err = device_error_word();
    if (!err) return cudaErrorMemoryAllocation;
    cudaError_t st = cudaMemsetAsync(temporary, 0, t.bytes, s);
    if (st != cudaSuccess) return st;
    auto kernel = spk::union_soa_kernel<kThreads, kSetItems>;
    const size_t tiles = (total + kSetTile - 1) / kSetTile;
    const unsigned grid = spk::persistent_grid(reinterpret_cast<const void*>(kernel), kThreads, 0, tiles);
    kernel<<<grid, kThreads, 0, s>>>(left_first, left_second, left_rows, right_first, right_second, right_rows,
                                     output_first, output_second, unique_rows, t.status, t.counter, 1u, err);
    return cudaGetLastError();
}

}  // extern "C"
