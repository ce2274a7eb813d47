// Status strings and the per-thread last CUDA error of the C ABI.
#include "common.cuh"

#include <cstring>
#include <string>
#include <vector>

namespace vipe {

namespace {
thread_local char g_last_error[256] = {0};
}

void set_last_error(const char* msg) {
    std::strncpy(g_last_error, msg ? msg : "", sizeof(g_last_error) - 1);
    g_last_error[sizeof(g_last_error) - 1] = 0;
}

// ---------------------------------------------------------------- launch profiler
// While enabled, library drivers bracket each kernel launch with CUDA events on
// the launching stream (prof_begin/prof_end); vipe_profile_collect() then
// synchronises and sums the elapsed times per kernel name.
namespace {
struct ProfSlot {
    const char* name;
    cudaEvent_t a, b;
};
bool g_prof_on = false;
std::vector<ProfSlot> g_prof;
std::vector<cudaEvent_t> g_pool;

cudaEvent_t take_event() {
    if (!g_pool.empty()) {
        cudaEvent_t e = g_pool.back();
        g_pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}
}  // namespace

bool prof_enabled() { return g_prof_on; }

int prof_begin(const char* name, cudaStream_t st) {
    if (!g_prof_on) return -1;
    ProfSlot sl{name, take_event(), take_event()};
    cudaEventRecord(sl.a, st);
    g_prof.push_back(sl);
    return (int)g_prof.size() - 1;
}

void prof_end(int id, cudaStream_t st) {
    if (id < 0 || id >= (int)g_prof.size()) return;
    cudaEventRecord(g_prof[id].b, st);
}

}  // namespace vipe

extern "C" __attribute__((visibility("default"))) void vipe_profile_enable(int on) {
    vipe::g_prof_on = on != 0;
}

extern "C" __attribute__((visibility("default"))) int vipe_profile_collect(char* names, int name_stride, float* total_ms,
                                                                          int* launches, int max_kernels) {
    using namespace vipe;
    int nk = 0;
    std::vector<std::string> keys;
    for (auto& sl : g_prof) {
        cudaEventSynchronize(sl.b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, sl.a, sl.b);
        int k = 0;
        for (; k < nk; k++)
            if (keys[k] == sl.name) break;
        if (k == nk) {
            if (nk >= max_kernels) continue;
            keys.push_back(sl.name);
            total_ms[nk] = 0.f;
            launches[nk] = 0;
            std::strncpy(names + (size_t)nk * name_stride, sl.name, name_stride - 1);
            names[(size_t)nk * name_stride + name_stride - 1] = 0;
            nk++;
        }
        total_ms[k] += ms;
        launches[k] += 1;
        g_pool.push_back(sl.a);
        g_pool.push_back(sl.b);
    }
    g_prof.clear();
    return nk;
}

extern "C" __attribute__((visibility("default"))) const char* vipe_last_error(void) { return vipe::g_last_error; }

extern "C" __attribute__((visibility("default"))) const char* vipe_status_string(int status) {
    switch (status) {
        case VIPE_OK: return "ok";
        case VIPE_ERR_ARG: return "invalid argument (shape, size or null pointer)";
        case VIPE_ERR_INDEX: return "edge index outside [0, num_frames)";
        case VIPE_ERR_RANGE: return "invalid optimisation window: need 0 <= t0 < t1 <= num_frames";
        case VIPE_ERR_KX_MISMATCH: return "eta rows do not match |unique(cat(arange(t0, t1), ii))|";
        case VIPE_ERR_WORKSPACE: return "workspace too small";
        case VIPE_ERR_CAPACITY: return "graph exceeds a kernel limit (more than 127 window poses, or more than 32 window poses coupled to one depth frame)";
        case VIPE_ERR_CUDA: return "CUDA runtime error";
        case VIPE_ERR_DTYPE: return "unsupported dtype";
        case VIPE_ERR_GROUP: return "unsupported Lie group id";
        case VIPE_ERR_DEVICE_WAIT: return "a kernel's bounded wait on tensor-core work expired";
        case VIPE_WARN_SOLVER: return "reduced camera system not positive definite: dx = 0";
        default: return "unknown status";
    }
}

// ---------------------------------------------------------------- write-bandwidth probe
namespace vipe {
namespace {
__global__ void write_probe_kernel(uint4* __restrict__ p, size_t n) {
    // four 16-byte stores per thread, consecutive threads on consecutive addresses
    const size_t base = blockIdx.x * (size_t)blockDim.x * 4 + threadIdx.x;
    const uint4 v = make_uint4(0x3c003c00u, 0x3c003c00u, 0x3c003c00u, 0x3c003c00u);
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const size_t i = base + (size_t)k * blockDim.x;
        if (i < n) p[i] = v;
    }
}
}  // namespace
}  // namespace vipe

extern "C" __attribute__((visibility("default"))) int vipe_hbm_write_probe(void* dst, size_t bytes, void* stream) {
    if (!dst || bytes % 16 != 0 || (uintptr_t)dst % 16 != 0) return VIPE_ERR_ARG;
    const size_t n = bytes / 16;
    if (n == 0) return VIPE_OK;
    const size_t blocks = (n + 1023) / 1024;
    if (blocks > 0x7fffffffull) return VIPE_ERR_CAPACITY;
    vipe::write_probe_kernel<<<(unsigned)blocks, 256, 0, vipe::as_stream(stream)>>>(static_cast<uint4*>(dst), n);
    VIPE_LAUNCH_CHECK();
    return VIPE_OK;
}
