// sparkalog_anti_join_u32_no_alloc: the sorted anti-join for callers that
// cannot allocate device memory.
//
// sparkalog_anti_join_u32 needs a caller-allocated `temporary` buffer for the
// kernel's scratch (decoupled look-back status words and a tile counter).
// Some callers cannot provide one: a host runtime that has handed its whole
// HBM budget to relation buffers up front and must not allocate on its
// per-round hot path, an FFI binding whose language has no device allocator
// of its own, or a caller that must not pay cudaMalloc's implicit device-wide
// synchronisation in the middle of a pipeline of asynchronous launches. This
// entry point takes the same inputs and outputs minus `temporary`, and keeps
// the scratch in a fixed array in the library's own device memory instead.
//
// Limits and sharing:
//   * left_rows may be at most SPARKALOG_ANTI_JOIN_NO_ALLOC_MAX_LEFT_ROWS
//     (2^27); larger inputs are rejected with cudaErrorInvalidValue before
//     any device work. The array costs about 513 KiB on every GPU that loads
//     the library, for the life of the process.
//   * Every call on a device uses the same array and leaves its last
//     contents behind; each call clears the part it needs (the tile counter
//     and its status words) on `stream` before launching. Calls whose work
//     overlaps on the GPU (different streams, no ordering between them) race
//     on the array and produce wrong results: order them on one stream.
//   * The first call on each device, with that device current, looks up the
//     array's device address (cudaGetSymbolAddress); make that first call
//     before any stream capture on the device. The address is cached with the
//     id of the CUDA context it was found in, so a call after a
//     cudaDeviceReset (a new context) looks it up again.
//   * A look-back wait that hits its spin cap cannot return an error code
//     from an asynchronous kernel; it sets a bit in a second static device
//     word, g_anti_join_no_alloc_error, which no call clears. Read (and
//     clear) it with sparkalog_anti_join_u32_no_alloc_error after the
//     stream has finished; a non-zero value means a result since the last
//     clear may be wrong.
//   * Nothing here calls cudaMalloc, cudaFree or any allocating routine.

#include "sparkalog_b200.h"
#include "spk_common.cuh"
#include "spk_setops.cuh"

#include <cuda.h>

#include <mutex>

namespace {

using spk::u32;
using spk::u64;

constexpr int kThreads = 256;
constexpr int kItems = 8;
constexpr int kTile = kThreads * kItems;
constexpr u64 kMaxLeftRows = SPARKALOG_ANTI_JOIN_NO_ALLOC_MAX_LEFT_ROWS;
constexpr u64 kStatusWords = kMaxLeftRows / kTile + 1;
constexpr int kMaxDevices = 64;

// Layout of the scratch array: a 256-byte header (the tile counter) followed
// by one look-back status word per tile of the left input.
constexpr size_t kHeaderBytes = 256;
constexpr size_t kScratchBytes = kHeaderBytes + kStatusWords * sizeof(u64);

static __device__ __align__(256) unsigned char g_anti_join_scratch[kScratchBytes];

// Error bits of every call on this device since the last read with reset
// (spk::kErrLookbackTimeout). Kept apart from the scratch array so that the
// per-call clearing of the array never erases a fault of an earlier call.
static __device__ __align__(256) u32 g_anti_join_no_alloc_error;

struct DeviceSetup {
    bool ready = false;
    unsigned long long context_id = 0;  // context the addresses belong to
    unsigned char* scratch = nullptr;   // device address of g_anti_join_scratch
    u32* error = nullptr;               // device address of g_anti_join_no_alloc_error
    int sms = 0;
    int ctas_per_sm = 0;
};

std::mutex g_setup_mutex;
DeviceSetup g_setup[kMaxDevices];

// The id of the current CUDA context (0 when none is current yet, or when the
// driver cannot tell). The two driver calls are resolved through the runtime
// (cudaGetDriverEntryPointByVersion) so that the library does not link
// libcuda itself.
unsigned long long current_context_id() {
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<GetCurrent>(f);
        f = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<GetId>(f);
    });
    if (!get_current || !get_id) return 0;
    CUcontext ctx = nullptr;
    if (get_current(&ctx) != CUDA_SUCCESS || ctx == nullptr) return 0;
    unsigned long long id = 0;
    if (get_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Once per device (and again in a new context after a cudaDeviceReset), with
// that device current: the static words' device addresses and the
// persistent grid shape of the kernel.
cudaError_t setup_for_current_device(DeviceSetup** out) {
    int dev = 0;
    cudaError_t st = cudaGetDevice(&dev);
    if (st != cudaSuccess) return st;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    // No context current on this thread yet (id 0) also redoes the set-up:
    // its runtime calls bind the device's primary context.
    const unsigned long long ctx = current_context_id();
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    DeviceSetup& d = g_setup[dev];
    if (!d.ready || ctx == 0 || d.context_id != ctx) {
        d.ready = false;
        void* ptr = nullptr;
        st = cudaGetSymbolAddress(&ptr, g_anti_join_scratch);
        if (st != cudaSuccess) return st;
        void* err_ptr = nullptr;
        st = cudaGetSymbolAddress(&err_ptr, g_anti_join_no_alloc_error);
        if (st != cudaSuccess) return st;
        int sms = 0;
        st = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (st != cudaSuccess) return st;
        int per_sm = 0;
        st = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, spk::anti_join_soa_kernel<kThreads, kItems>,
                                                           kThreads, 0);
        if (st != cudaSuccess) return st;
        d.scratch = static_cast<unsigned char*>(ptr);
        d.error = static_cast<u32*>(err_ptr);
        d.context_id = current_context_id();
        d.sms = sms > 0 ? sms : 1;
        d.ctas_per_sm = per_sm > 0 ? per_sm : 1;
        d.ready = true;
    }
    *out = &d;
    return cudaSuccess;
}

}  // namespace

extern "C" int sparkalog_anti_join_u32_no_alloc(const u32* left_first, const u32* left_second, size_t left_rows,
                                                const u32* right_first, const u32* right_second, size_t right_rows,
                                                u32* flags, u32* selected, u32* selected_rows, u32* output_first,
                                                u32* output_second, void* stream) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (selected_rows == nullptr) return cudaErrorInvalidValue;
    if (left_rows > kMaxLeftRows) return cudaErrorInvalidValue;
    if (left_rows == 0) return cudaMemsetAsync(selected_rows, 0, sizeof(*selected_rows), s);
    if (left_first == nullptr || left_second == nullptr || flags == nullptr || selected == nullptr ||
        output_first == nullptr || output_second == nullptr ||
        (right_rows != 0 && (right_first == nullptr || right_second == nullptr))) {
        return cudaErrorInvalidValue;
    }
    DeviceSetup* d = nullptr;
    cudaError_t st = setup_for_current_device(&d);
    if (st != cudaSuccess) return st;
    u32* tile_counter = reinterpret_cast<u32*>(d->scratch);
    u64* status = reinterpret_cast<u64*>(d->scratch + kHeaderBytes);
    const u64 tiles = (left_rows + kTile - 1) / kTile;
    // Clear what this call reads before it is written: the tile counter and
    // the status words of its tiles (epoch 1 then marks this call's words).
    st = cudaMemsetAsync(d->scratch, 0, kHeaderBytes + (tiles + 1) * sizeof(u64), s);
    if (st != cudaSuccess) return st;
    u64 grid = static_cast<u64>(d->sms) * static_cast<u64>(d->ctas_per_sm);
    if (tiles < grid) grid = tiles;
    spk::anti_join_soa_kernel<kThreads, kItems><<<static_cast<unsigned>(grid), kThreads, 0, s>>>(
        left_first, left_second, left_rows, right_first, right_second, right_rows, flags, selected, selected_rows,
        output_first, output_second, status, tile_counter, 1u, d->error);
    return cudaGetLastError();
}

extern "C" int sparkalog_anti_join_u32_no_alloc_error(u32* bits, int reset) {
    if (bits == nullptr) return cudaErrorInvalidValue;
    DeviceSetup* d = nullptr;
    cudaError_t st = setup_for_current_device(&d);
    if (st != cudaSuccess) return st;
    // Symbol copies are synchronous with the device's legacy default stream
    // and allocate nothing.
    st = cudaMemcpyFromSymbol(bits, g_anti_join_no_alloc_error, sizeof(u32));
    if (st == cudaSuccess && reset) {
        const u32 zero = 0;
        st = cudaMemcpyToSymbol(g_anti_join_no_alloc_error, &zero, sizeof(u32));
    }
    return st;
}
