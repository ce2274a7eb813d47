// Bundle adjustment without any device allocation by the caller or the library.
//
// vipe_slam_ba_extended needs a device workspace, which its callers allocate
// (the Python layer takes it from torch's caching allocator).  Some hosts
// cannot do that: a process that must not allocate after start-up (a real-time
// or certified pipeline), or a binding whose runtime has no CUDA allocator of
// its own (a cgo / JNI / plain C host that only receives tensors).  For them,
// vipe_slam_ba_extended_noalloc runs the same solve with its scratch in a
// file-scope device array of VIPE_BA_NOALLOC_SCRATCH_BYTES, which every GPU
// that loads this library holds until the process exits.
#include "ba_internal.cuh"
#include "common.cuh"

#include <cstdio>
#include <mutex>

namespace vipe {
namespace {

// The shared scratch.  Host code must not use this name as a device address:
// its device address comes from cudaGetSymbolAddress (scratch_on_current_device).
static __device__ __align__(256) unsigned char g_ba_scratch[VIPE_BA_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
void* g_scratch_ptr[kMaxDevices] = {nullptr};

// Device address of g_ba_scratch on the current device, looked up once per
// device (the first call on a device therefore loads this module there).  The
// cached address belongs to that device's primary context: a device reset
// (cudaDeviceReset) between calls would invalidate it, so callers of this entry
// point must not reset the device while the library is loaded.
int scratch_on_current_device(void** out) {
    int dev = 0;
    VIPE_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        set_last_error("vipe_slam_ba_extended_noalloc: device ordinal beyond 63");
        return VIPE_ERR_CAPACITY;
    }
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        VIPE_CUDA_TRY(cudaGetSymbolAddress(&p, g_ba_scratch));
        g_scratch_ptr[dev] = p;
    }
    *out = g_scratch_ptr[dev];
    return VIPE_OK;
}

}  // namespace
}  // namespace vipe

using namespace vipe;

extern "C" int vipe_slam_ba_extended_noalloc(float* poses_io, float* disps_io, float* intrinsics_io,
                                             const float* disps_sens, const float* targets, const float* weights,
                                             const float* eta, const int64_t* ii, const int64_t* jj,
                                             const float* depth_active, int num_frames, int ht, int wd,
                                             int num_edges, int num_kx, int t0, int t1, int iterations, float lm,
                                             float ep, int motion_only, float alpha, int optimize_intrinsics,
                                             float intrinsics_lm, float intrinsics_ep, float intrinsics_scale,
                                             int compute_energy, float* dx_out, float* dz_out, float* energy_out,
                                             int32_t* dev_status, void* stream) {
    // the same size checks, with the same status codes, as vipe_slam_ba_extended
    const int dims_rc = ba::check_dims(num_frames, ht, wd, num_edges, num_kx, t0, t1);
    if (dims_rc != VIPE_OK) return dims_rc;
    const size_t need = vipe_slam_ba_workspace_size(num_frames, ht, wd, num_edges, num_kx, t0, t1);
    if (need == 0) return VIPE_ERR_ARG;
    if (need > (size_t)VIPE_BA_NOALLOC_SCRATCH_BYTES) {
        char msg[160];
        snprintf(msg, sizeof(msg),
                 "vipe_slam_ba_extended_noalloc: graph needs %zu bytes of scratch, the static scratch holds %zu",
                 need, (size_t)VIPE_BA_NOALLOC_SCRATCH_BYTES);
        set_last_error(msg);
        return VIPE_ERR_CAPACITY;
    }
    void* scratch = nullptr;
    const int rc = scratch_on_current_device(&scratch);
    if (rc != VIPE_OK) return rc;
    // The solve initialises every scratch word it reads, so the previous call's
    // contents need no clearing; passing the true capacity keeps the workspace
    // carver's own bound check in force as well.
    return vipe_slam_ba_extended(poses_io, disps_io, intrinsics_io, disps_sens, targets, weights, eta, ii, jj,
                                 depth_active, num_frames, ht, wd, num_edges, num_kx, t0, t1, iterations, lm, ep,
                                 motion_only, alpha, optimize_intrinsics, intrinsics_lm, intrinsics_ep,
                                 intrinsics_scale, compute_energy, dx_out, dz_out, energy_out, scratch,
                                 (size_t)VIPE_BA_NOALLOC_SCRATCH_BYTES, dev_status, stream);
}
