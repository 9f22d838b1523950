// Host-side helpers shared by the C-ABI translation units.
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

namespace spk {

// Streaming multiprocessor count of the current device (cached per device).
int device_sm_count();

// Persistent grid size: resident CTAs of `kernel` per SM times the SM count,
// never more than `tiles` (and at least 1).
unsigned int persistent_grid(const void* kernel, int threads, size_t dynamic_smem, size_t tiles);

inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Carves consecutive 256-byte aligned regions out of a caller-provided buffer.
struct Carver {
    char* base;
    size_t used = 0;
    explicit Carver(void* p) : base(static_cast<char*>(p)) {}
    template <class T>
    T* take(size_t count) {
        used = align_up(used, 256);
        T* p = base ? reinterpret_cast<T*>(base + used) : nullptr;
        used += count * sizeof(T);
        return p;
    }
};

}  // namespace spk
