// Status strings and the per-thread last CUDA error of the C ABI.
#include "common.cuh"

#include <cstring>

namespace vipe {

namespace {
thread_local char g_last_error[256] = {0};
}

void set_last_error(const char* msg) {
    std::strncpy(g_last_error, msg ? msg : "", sizeof(g_last_error) - 1);
    g_last_error[sizeof(g_last_error) - 1] = 0;
}

}  // namespace vipe

extern "C" __attribute__((visibility("default"))) const char* vipe_last_error(void) { return vipe::g_last_error; }

extern "C" __attribute__((visibility("default"))) const char* vipe_status_string(int status) {
    switch (status) {
        case VIPE_OK: return "ok";
        case VIPE_ERR_ARG: return "invalid argument (shape, size or null pointer)";
        case VIPE_ERR_INDEX: return "edge index outside [0, num_frames)";
        case VIPE_ERR_RANGE: return "invalid optimisation window: need 0 <= t0 < t1 <= num_frames";
        case VIPE_ERR_KX_MISMATCH: return "eta rows do not match |unique(cat(arange(t0, t1), ii))|";
        case VIPE_ERR_WORKSPACE: return "workspace too small";
        case VIPE_ERR_CAPACITY: return "graph exceeds a kernel limit (window poses > 1024 or > 32 window poses coupled to one depth frame)";
        case VIPE_ERR_CUDA: return "CUDA runtime error";
        case VIPE_ERR_DTYPE: return "unsupported dtype";
        case VIPE_ERR_GROUP: return "unsupported Lie group id";
        case VIPE_WARN_SOLVER: return "reduced camera system not positive definite: dx = 0";
        default: return "unknown status";
    }
}
