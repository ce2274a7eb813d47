// Geometry helpers of slam_ext: frame_distance, projmap, depth_filter, iproj.
//
// Reference: vipe csrc/slam_ext/geom_kernels.cu:526-953 (kernels) and
// :1849-1950 (hosts).  Same pinhole model, MIN_DEPTH = 0.25 validity rule,
// beta blend of full and translation-only motion with the 1000 sentinel below
// 75 % valid pixels (frame_distance), the projection fallback to (u, v) for
// z <= 0.01 (projmap), six temporal neighbours and the double-precision depth
// comparison (depth_filter).  Reductions are fixed-order block reductions, so
// frame_distance is deterministic.

#include "common.cuh"
#include "se3_device.cuh"

namespace vipe {
namespace geom {

constexpr float kMinDepth = 0.25f;

__global__ void __launch_bounds__(256)
    frame_distance_kernel(const float* __restrict__ poses, const float* __restrict__ disps,
                          const float* __restrict__ intr, const int64_t* __restrict__ pi, const int64_t* __restrict__ pj,
                          const int64_t* __restrict__ qi, const int64_t* __restrict__ qj,
                          const int64_t* __restrict__ di, int num_poses, int num_disps, int num_views, int ht, int wd,
                          float beta, float* __restrict__ dist) {
    __shared__ float red[3][8];
    const int b = blockIdx.x;
    const int64_t ix64 = pi[b], jx64 = pj[b], dix64 = di[b], rix64 = qi[b], rjx64 = qj[b];
    // indices outside the tensors give NaN instead of an out-of-bounds read
    if (ix64 < 0 || ix64 >= num_poses || jx64 < 0 || jx64 >= num_poses || dix64 < 0 || dix64 >= num_disps ||
        rix64 < 0 || rix64 >= num_views || rjx64 < 0 || rjx64 >= num_views) {
        if (threadIdx.x == 0) dist[b] = __int_as_float(0x7fc00000);
        return;
    }
    const int ix = (int)ix64, jx = (int)jx64, dix = (int)dix64, rix = (int)rix64, rjx = (int)rjx64;
    const float fxi = intr[4 * rix], fyi = intr[4 * rix + 1], cxi = intr[4 * rix + 2], cyi = intr[4 * rix + 3];
    const float fxj = intr[4 * rjx], fyj = intr[4 * rjx + 1], cxj = intr[4 * rjx + 2], cyj = intr[4 * rjx + 3];
    float Ti[7], Tj[7], tij[3], qij[4];
    for (int n = 0; n < 7; n++) {
        Ti[n] = poses[7 * ix + n];
        Tj[n] = poses[7 * jx + n];
    }
    rel_pose(Ti, Tj, tij, qij);
    float acc = 0.f, valid = 0.f, total = 0.f;
    const int HW = ht * wd;
    for (int k = threadIdx.x; k < HW; k += blockDim.x) {
        const float u = (float)(k % wd), v = (float)(k / wd);
        const float d = disps[(size_t)dix * HW + k];
        float Xi[4] = {(u - cxi) / fxi, (v - cyi) / fyi, 1.f, d};
        float Xj[4];
        act_h(tij, qij, Xi, Xj);
        float du = fxj * (Xj[0] / Xj[2]) + cxj - u;
        float dv = fyj * (Xj[1] / Xj[2]) + cyj - v;
        float dd = sqrtf(du * du + dv * dv);
        total += beta;
        if (Xj[2] > kMinDepth) {
            acc += beta * dd;
            valid += beta;
        }
        // translation-only motion
        Xj[0] = Xi[0] + Xi[3] * tij[0];
        Xj[1] = Xi[1] + Xi[3] * tij[1];
        Xj[2] = Xi[2] + Xi[3] * tij[2];
        du = fxj * (Xj[0] / Xj[2]) + cxj - u;
        dv = fyj * (Xj[1] / Xj[2]) + cyj - v;
        dd = sqrtf(du * du + dv * dv);
        total += 1.f - beta;
        if (Xj[2] > kMinDepth) {
            acc += (1.f - beta) * dd;
            valid += 1.f - beta;
        }
    }
    acc = warp_sum(acc);
    valid = warp_sum(valid);
    total = warp_sum(total);
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        red[0][w] = acc;
        red[1][w] = valid;
        red[2][w] = total;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        float a = 0.f, vv = 0.f, t = 0.f;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) {
            a += red[0][q];
            vv += red[1][q];
            t += red[2][q];
        }
        dist[b] = (vv / (t + 1e-8f) < 0.75f) ? 1000.f : a / vv;
    }
}

__global__ void projmap_kernel(const float* __restrict__ poses, const float* __restrict__ disps,
                               const float* __restrict__ intr, const int64_t* __restrict__ ii,
                               const int64_t* __restrict__ jj, int num_frames, int ht, int wd,
                               float* __restrict__ coords, float* __restrict__ valid) {
    const int b = blockIdx.y;
    const int HW = ht * wd;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= HW) return;
    if (ii[b] < 0 || ii[b] >= num_frames || jj[b] < 0 || jj[b] >= num_frames) {
        const float nan = __int_as_float(0x7fc00000);
        float* c = coords + ((size_t)b * HW + k) * 3;
        c[0] = nan;
        c[1] = nan;
        c[2] = nan;
        valid[(size_t)b * HW + k] = nan;
        return;
    }
    const int ix = (int)ii[b], jx = (int)jj[b];
    float Ti[7], Tj[7], tij[3], qij[4];
    for (int n = 0; n < 7; n++) {
        Ti[n] = poses[7 * ix + n];
        Tj[n] = poses[7 * jx + n];
    }
    rel_pose(Ti, Tj, tij, qij);
    const float fx = intr[0], fy = intr[1], cx = intr[2], cy = intr[3];
    const float u = (float)(k % wd), v = (float)(k / wd);
    float Xi[4] = {(u - cx) / fx, (v - cy) / fy, 1.f, disps[(size_t)ix * HW + k]};
    float Xj[4];
    act_h(tij, qij, Xi, Xj);
    float* c = coords + ((size_t)b * HW + k) * 3;
    c[0] = u;
    c[1] = v;
    if (Xj[2] > 0.01f) {
        c[0] = fx * (Xj[0] / Xj[2]) + cx;
        c[1] = fy * (Xj[1] / Xj[2]) + cy;
    }
    c[2] = 0.f;
    valid[(size_t)b * HW + k] = (Xj[2] > kMinDepth) ? 1.f : 0.f;
}

// grid (num, 6 neighbours, pixel blocks); counter must be zero on entry.  Each
// (frame, pixel) receives at most one increment per neighbour; the counts are
// small integers, so the atomic sum is exact and order-independent.
__global__ void depth_filter_kernel(const float* __restrict__ poses, const float* __restrict__ disps,
                                    const float* __restrict__ intr, const int64_t* __restrict__ inds,
                                    const float* __restrict__ thresh, int num_frames, int ht, int wd,
                                    float* __restrict__ counter) {
    const int b = blockIdx.x, nb = blockIdx.y;
    const int HW = ht * wd;
    const int k = blockIdx.z * blockDim.x + threadIdx.x;
    if (inds[b] < 0 || inds[b] >= num_frames) return;  // out-of-range frame: count stays 0
    const int ix = (int)inds[b];
    const int jx = (nb < 3) ? ix - nb - 1 : ix + nb - 2;
    if (jx < 0 || jx >= num_frames || k >= HW) return;
    const float t = thresh[b];
    float Ti[7], Tj[7], tij[3], qij[4];
    for (int n = 0; n < 7; n++) {
        Ti[n] = poses[7 * ix + n];
        Tj[n] = poses[7 * jx + n];
    }
    rel_pose(Ti, Tj, tij, qij);
    const float fx = intr[0], fy = intr[1], cx = intr[2], cy = intr[3];
    const float ui = (float)(k % wd), vi = (float)(k / wd);
    float Xi[4] = {(ui - cx) / fx, (vi - cy) / fy, 1.f, disps[(size_t)ix * HW + k]};
    float Xj[4];
    act_h(tij, qij, Xi, Xj);
    const float uj = fx * (Xj[0] / Xj[2]) + cx;
    const float vj = fy * (Xj[1] / Xj[2]) + cy;
    const float dj = Xj[3] / Xj[2];
    // clamp before the conversion: a projection at infinity or NaN (Xj[2] = 0) must not
    // reach an out-of-range float -> int conversion, whose result the bounds test could not trust
    const int u0 = (int)fminf(fmaxf(floorf(uj), -1.f), (float)wd);
    const int v0 = (int)fminf(fmaxf(floorf(vj), -1.f), (float)ht);
    if (u0 >= 0 && v0 >= 0 && u0 < wd - 1 && v0 < ht - 1) {
        const float* dpj = disps + (size_t)jx * HW;
        const double idj = 1.0 / (double)dj;
        const double tt = (double)t;
        const float d00 = dpj[v0 * wd + u0], d01 = dpj[v0 * wd + u0 + 1];
        const float d10 = dpj[(v0 + 1) * wd + u0], d11 = dpj[(v0 + 1) * wd + u0 + 1];
        if (fabs(idj - 1.0 / (double)d00) < tt || fabs(idj - 1.0 / (double)d01) < tt ||
            fabs(idj - 1.0 / (double)d10) < tt || fabs(idj - 1.0 / (double)d11) < tt)
            atomicAdd(counter + (size_t)b * HW + k, 1.0f);
    }
}

__global__ void iproj_kernel(const float* __restrict__ poses, const float* __restrict__ disps,
                             const float* __restrict__ intr, int ht, int wd, float* __restrict__ points) {
    const int b = blockIdx.y;
    const int HW = ht * wd;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= HW) return;
    const float* T = poses + 7 * b;
    const float fx = intr[0], fy = intr[1], cx = intr[2], cy = intr[3];
    const float ui = (float)(k % wd), vi = (float)(k / wd);
    float Xi[4] = {(ui - cx) / fx, (vi - cy) / fy, 1.f, disps[(size_t)b * HW + k]};
    float Xj[4];
    act_h(T, T + 3, Xi, Xj);
    float* o = points + ((size_t)b * HW + k) * 3;
    o[0] = Xj[0] / Xj[3];
    o[1] = Xj[1] / Xj[3];
    o[2] = Xj[2] / Xj[3];
}

}  // namespace geom
}  // namespace vipe

using namespace vipe;
using namespace vipe::geom;

extern "C" int vipe_slam_frame_distance(const float* poses, const float* disps, const float* intrinsics,
                                        const int64_t* pi, const int64_t* pj, const int64_t* qi, const int64_t* qj,
                                        const int64_t* di, int num, int num_poses, int num_disps, int num_views,
                                        int ht, int wd, float beta, float* dist_out, void* stream) {
    if (num < 0 || ht <= 0 || wd <= 0 || num_poses <= 0 || num_disps <= 0 || num_views <= 0) return VIPE_ERR_ARG;
    if (num == 0) return VIPE_OK;
    cudaStream_t st = as_stream(stream);
    VIPE_PROF("frame_distance", st);
    frame_distance_kernel<<<num, 256, 0, st>>>(poses, disps, intrinsics, pi, pj, qi, qj, di, num_poses, num_disps,
                                               num_views, ht, wd, beta, dist_out);
    VIPE_LAUNCH_CHECK();
    return VIPE_OK;
}

extern "C" int vipe_slam_projmap(const float* poses, const float* disps, const float* intrinsics, const int64_t* ii,
                                 const int64_t* jj, int num, int num_frames, int ht, int wd, float* coords_out,
                                 float* valid_out, void* stream) {
    if (num < 0 || ht <= 0 || wd <= 0 || num > 65535 || num_frames <= 0) return VIPE_ERR_ARG;
    if (num == 0) return VIPE_OK;
    cudaStream_t st = as_stream(stream);
    dim3 grid(ceil_div((size_t)ht * wd, 256), num);
    VIPE_PROF("projmap", st);
    projmap_kernel<<<grid, 256, 0, st>>>(poses, disps, intrinsics, ii, jj, num_frames, ht, wd, coords_out, valid_out);
    VIPE_LAUNCH_CHECK();
    return VIPE_OK;
}

extern "C" int vipe_slam_depth_filter(const float* poses, const float* disps, const float* intrinsics,
                                      const int64_t* ix, const float* thresh, int num_frames, int num, int ht, int wd,
                                      float* counter_out, void* stream) {
    if (num < 0 || ht <= 0 || wd <= 0 || num_frames <= 0 || num > 65535) return VIPE_ERR_ARG;
    cudaStream_t st = as_stream(stream);
    VIPE_CUDA_TRY(cudaMemsetAsync(counter_out, 0, (size_t)num * ht * wd * sizeof(float), st));
    if (num == 0) return VIPE_OK;
    dim3 grid(num, 6, ceil_div((size_t)ht * wd, 256));
    VIPE_PROF("depth_filter", st);
    depth_filter_kernel<<<grid, 256, 0, st>>>(poses, disps, intrinsics, ix, thresh, num_frames, ht, wd, counter_out);
    VIPE_LAUNCH_CHECK();
    return VIPE_OK;
}

extern "C" int vipe_slam_iproj(const float* poses, const float* disps, const float* intrinsics, int num_frames,
                               int ht, int wd, float* points_out, void* stream) {
    if (num_frames < 0 || ht <= 0 || wd <= 0 || num_frames > 65535) return VIPE_ERR_ARG;
    if (num_frames == 0) return VIPE_OK;
    cudaStream_t st = as_stream(stream);
    dim3 grid(ceil_div((size_t)ht * wd, 256), num_frames);
    VIPE_PROF("iproj", st);
    iproj_kernel<<<grid, 256, 0, st>>>(poses, disps, intrinsics, ht, wd, points_out);
    VIPE_LAUNCH_CHECK();
    return VIPE_OK;
}
