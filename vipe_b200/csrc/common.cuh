// Shared helpers of the vipe_b200 CUDA library (sm_100a only).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#include "../../include/vipe_b200.h"

#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ < 1000)
#error "vipe_b200 is built for sm_100a (B200) only"
#endif

namespace vipe {

// Records the last CUDA error string for vipe_last_error().
void set_last_error(const char* msg);

// Launch profiler (vipe_profile_enable / vipe_profile_collect).
bool prof_enabled();
int prof_begin(const char* name, cudaStream_t st);
void prof_end(int id, cudaStream_t st);

// RAII bracket of one launch: VIPE_PROF("kernel", stream) before the launch.
struct ProfScope {
    int id;
    cudaStream_t st;
    ProfScope(const char* n, cudaStream_t s) : id(prof_enabled() ? prof_begin(n, s) : -1), st(s) {}
    ~ProfScope() {
        if (id >= 0) prof_end(id, st);
    }
};
#define VIPE_PROF(name, st) ::vipe::ProfScope _vipe_prof_scope_##__LINE__(name, st)

#define VIPE_CUDA_TRY(expr)                                  \
    do {                                                     \
        cudaError_t _e = (expr);                             \
        if (_e != cudaSuccess) {                             \
            ::vipe::set_last_error(cudaGetErrorString(_e));  \
            return (int)VIPE_ERR_CUDA;                       \
        }                                                    \
    } while (0)

// Checks the launch that was just enqueued.
#define VIPE_LAUNCH_CHECK() VIPE_CUDA_TRY(cudaGetLastError())

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

inline unsigned ceil_div(size_t a, size_t b) { return (unsigned)((a + b - 1) / b); }

// Bump allocator over a caller-provided device workspace.  Every carve is
// 256-byte aligned; `ok` turns false when the workspace is too small.
struct Carver {
    char* base;
    size_t cap;
    size_t used = 0;
    bool ok = true;
    Carver(void* b, size_t c) : base(static_cast<char*>(b)), cap(c) {}
    template <typename T>
    T* take(size_t count) {
        size_t off = (used + 255) & ~size_t(255);
        size_t bytes = count * sizeof(T);
        if (off + bytes > cap || (base == nullptr && bytes > 0)) {
            ok = false;
            used = off + bytes;
            return nullptr;
        }
        used = off + bytes;
        return reinterpret_cast<T*>(base + off);
    }
};

// Size-only counterpart of Carver (same alignment rules).
struct Sizer {
    size_t used = 0;
    template <typename T>
    T* take(size_t count) {
        size_t off = (used + 255) & ~size_t(255);
        used = off + count * sizeof(T);
        return nullptr;
    }
};

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace vipe
