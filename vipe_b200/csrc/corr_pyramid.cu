// Channels-last feature pyramid of AltCorrBlock, forward and adjoint.
//
// The reference builds it in eager torch (vipe/slam/networks/droid_net.py:130-142):
//     f = fmaps.view(B*N, C, H, W) / 4.0
//     level l = f.permute(0, 2, 3, 1).contiguous()      (B*N, H>>l, W>>l, C)
//     f = avg_pool2d(f, 2, stride=2)                     (floor sizes)
// i.e. one division, three pooling passes and four transposes through HBM.  Here one
// kernel reads each (num, C) plane tile once and writes every level:
//   * a CTA owns an 8 x 16 tile of level-0 pixels (1 x 2 pixels of level 3) and all
//     channels, staged in shared memory;
//   * each level is rounded to the element type before the next one pools it, with the
//     pooling sum taken in FP32 in avg_pool2d's order ((0,0), (0,1), (1,0), (1,1), then
//     / 4), so every level equals the reference's bit for bit;
//   * stores are channels-last 16-byte vectors, consecutive threads on consecutive
//     channel chunks of one pixel.
// The adjoint spreads each level's gradient back over the level-0 pixels it averages
// (weight 4^-l), times the 1/4, in FP32, and writes the (num, C, H, W) gradient.
#include "common.cuh"

#include <cuda_bf16.h>
#include <cuda_fp16.h>

namespace vipe {
namespace {

constexpr int kTileH = 8, kTileW = 16, kTilePx = kTileH * kTileW;
constexpr int kPyrThreads = 256;
constexpr int kPyrMaxLevels = 4;  // the tile holds one level-3 row of 2 pixels
constexpr int kPyrMaxC = 256;

template <typename T>
__device__ __forceinline__ float to_f(T v);
template <>
__device__ __forceinline__ float to_f<float>(float v) { return v; }
template <>
__device__ __forceinline__ float to_f<__half>(__half v) { return __half2float(v); }
template <>
__device__ __forceinline__ float to_f<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }

template <typename T>
__device__ __forceinline__ T from_f(float v);
template <>
__device__ __forceinline__ float from_f<float>(float v) { return v; }
template <>
__device__ __forceinline__ __half from_f<__half>(float v) { return __float2half_rn(v); }
template <>
__device__ __forceinline__ __nv_bfloat16 from_f<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }

// value as the element type would hold it
template <typename T>
__device__ __forceinline__ float round_to(float v) { return to_f<T>(from_f<T>(v)); }

// shared-memory plane of level l: C rows of (kTilePx >> 2l) pixels, padded by one
__host__ __device__ constexpr int lvl_ld(int l) { return (kTilePx >> (2 * l)) + 1; }
__host__ __device__ constexpr int lvl_off(int l) {
    return l == 0 ? 0 : lvl_off(l - 1) + lvl_ld(l - 1);  // in units of C floats
}

// writes level l's staged tile (rows y0..y0+th, cols x0..x0+tw of the level) channels-last
template <typename T>
__device__ __forceinline__ void store_level(const float* s, int ld, int C, int th, int tw, int y0, int x0, int Hl,
                                            int Wl, T* out) {
    constexpr int V = 16 / (int)sizeof(T);  // elements per 16-byte store
    const int cv = C / V;
    for (int idx = threadIdx.x; idx < th * tw * cv; idx += kPyrThreads) {
        const int q = idx / cv, c0 = (idx % cv) * V;
        const int y = y0 + q / tw, x = x0 + q % tw;
        if (y >= Hl || x >= Wl) continue;
        alignas(16) T v[V];
#pragma unroll
        for (int i = 0; i < V; i++) v[i] = from_f<T>(s[(c0 + i) * ld + q]);
        *reinterpret_cast<uint4*>(out + ((size_t)y * Wl + x) * C + c0) = *reinterpret_cast<const uint4*>(v);
    }
}

struct PyrArgs {
    const void* in;
    void* out[kPyrMaxLevels];
    int num, C, H, W, L, tiles_x, tiles_y;
};

template <typename T>
__global__ void __launch_bounds__(kPyrThreads) pyramid_fwd_kernel(PyrArgs a) {
    extern __shared__ float sp[];
    const int C = a.C;
    const int tile = blockIdx.x % (a.tiles_x * a.tiles_y), n = blockIdx.x / (a.tiles_x * a.tiles_y);
    const int ty = tile / a.tiles_x, tx = tile % a.tiles_x;
    const int y0 = ty * kTileH, x0 = tx * kTileW;
    const T* in = static_cast<const T*>(a.in) + (size_t)n * C * a.H * a.W;
    // level 0: fmaps / 4, rounded as the reference's division rounds it
    float* s0 = sp;
    for (int idx = threadIdx.x; idx < C * kTilePx; idx += kPyrThreads) {
        const int c = idx / kTilePx, p = idx % kTilePx;
        const int y = y0 + p / kTileW, x = x0 + p % kTileW;
        const float v = (y < a.H && x < a.W) ? to_f<T>(in[((size_t)c * a.H + y) * a.W + x]) : 0.f;
        s0[c * lvl_ld(0) + p] = round_to<T>(v / 4.0f);
    }
    __syncthreads();
    store_level<T>(s0, lvl_ld(0), C, kTileH, kTileW, y0, x0, a.H, a.W,
                   static_cast<T*>(a.out[0]) + (size_t)n * a.H * a.W * C);
    for (int l = 1; l < a.L; l++) {
        const float* sp_prev = sp + (size_t)C * lvl_off(l - 1);
        float* sl = sp + (size_t)C * lvl_off(l);
        const int ldp = lvl_ld(l - 1), ld = lvl_ld(l);
        const int twp = kTileW >> (l - 1), th = kTileH >> l, tw = kTileW >> l;
        for (int idx = threadIdx.x; idx < C * th * tw; idx += kPyrThreads) {
            const int c = idx / (th * tw), q = idx % (th * tw);
            const int qy = q / tw, qx = q % tw;
            const float* src = sp_prev + c * ldp + (2 * qy) * twp + 2 * qx;
            // avg_pool2d's FP32 sum over the window, row by row, then the division
            const float sum = ((src[0] + src[1]) + src[twp]) + src[twp + 1];
            sl[c * ld + q] = round_to<T>(sum / 4.0f);
        }
        __syncthreads();
        const int Hl = a.H >> l, Wl = a.W >> l;
        store_level<T>(sl, ld, C, th, tw, y0 >> l, x0 >> l, Hl, Wl,
                       static_cast<T*>(a.out[l]) + (size_t)n * Hl * Wl * C);
    }
}

struct PyrBwdArgs {
    const float* grad[kPyrMaxLevels];  // level gradients, channels-last FP32
    void* out;                         // (num, C, H, W)
    int num, C, H, W, L, tiles_x, tiles_y;
};

template <typename T>
__global__ void __launch_bounds__(kPyrThreads) pyramid_bwd_kernel(PyrBwdArgs a) {
    extern __shared__ float sg[];  // [C][kTilePx + 1]
    const int C = a.C;
    const int tile = blockIdx.x % (a.tiles_x * a.tiles_y), n = blockIdx.x / (a.tiles_x * a.tiles_y);
    const int ty = tile / a.tiles_x, tx = tile % a.tiles_x;
    const int y0 = ty * kTileH, x0 = tx * kTileW;
    const int ld = kTilePx + 1;
    for (int idx = threadIdx.x; idx < C * kTilePx; idx += kPyrThreads) sg[(idx / kTilePx) * ld + idx % kTilePx] = 0.f;
    __syncthreads();
    for (int l = 0; l < a.L; l++) {
        const int Hl = a.H >> l, Wl = a.W >> l;
        const int th = kTileH >> l, tw = kTileW >> l;
        const float wgt = 0.25f / (float)(1 << (2 * l));  // the 1/4 of fmaps / 4, times 4^-l of the pooling
        const float* g = a.grad[l] + (size_t)n * Hl * Wl * C;
        // channel-fastest reads (coalesced), each level-l pixel spread over its 4^l sources
        for (int idx = threadIdx.x; idx < C * th * tw; idx += kPyrThreads) {
            const int q = idx / C, c = idx % C;
            const int Y = (y0 >> l) + q / tw, X = (x0 >> l) + q % tw;
            if (Y >= Hl || X >= Wl) continue;
            const float v = g[((size_t)Y * Wl + X) * C + c] * wgt;
            const int span = 1 << l;
            const int py = (q / tw) * span, px = (q % tw) * span;
            for (int dy = 0; dy < span; dy++)
                for (int dx = 0; dx < span; dx++) sg[c * ld + (py + dy) * kTileW + px + dx] += v;
        }
        __syncthreads();
    }
    T* out = static_cast<T*>(a.out) + (size_t)n * C * a.H * a.W;
    for (int idx = threadIdx.x; idx < C * kTilePx; idx += kPyrThreads) {
        const int c = idx / kTilePx, p = idx % kTilePx;
        const int y = y0 + p / kTileW, x = x0 + p % kTileW;
        if (y < a.H && x < a.W) out[((size_t)c * a.H + y) * a.W + x] = from_f<T>(sg[c * ld + p]);
    }
}

int check_pyramid(int dtype, int num, int C, int H, int W, int L) {
    if (num <= 0 || C <= 0 || H <= 0 || W <= 0 || L <= 0) return VIPE_ERR_ARG;
    if (L > kPyrMaxLevels || (H >> (L - 1)) == 0 || (W >> (L - 1)) == 0) {
        set_last_error("feature pyramid: 1 to 4 levels, each at least one pixel");
        return VIPE_ERR_ARG;
    }
    if (dtype != VIPE_F32 && dtype != VIPE_F16 && dtype != VIPE_BF16) return VIPE_ERR_DTYPE;
    const int V = dtype == VIPE_F32 ? 4 : 8;
    if (C % V != 0 || C > kPyrMaxC) {
        set_last_error("feature pyramid: C must be a multiple of 16 bytes of elements and at most 256");
        return VIPE_ERR_ARG;
    }
    return VIPE_OK;
}

size_t fwd_smem(int C, int L) { return (size_t)C * lvl_off(L) * sizeof(float); }

}  // namespace
}  // namespace vipe

using namespace vipe;

extern "C" int vipe_corr_pyramid_nhwc(int dtype, const void* fmaps, int num, int C, int H, int W, int num_levels,
                                      void* const* level_out, void* stream) {
    int rc = check_pyramid(dtype, num, C, H, W, num_levels);
    if (rc != VIPE_OK) return rc;
    if (!fmaps || !level_out) return VIPE_ERR_ARG;
    PyrArgs a{};
    a.in = fmaps;
    for (int l = 0; l < num_levels; l++) {
        if (!level_out[l] || ((uintptr_t)level_out[l] & 15u)) return VIPE_ERR_ARG;  // 16-byte stores
        a.out[l] = level_out[l];
    }
    a.num = num; a.C = C; a.H = H; a.W = W; a.L = num_levels;
    a.tiles_x = (W + kTileW - 1) / kTileW;
    a.tiles_y = (H + kTileH - 1) / kTileH;
    const long blocks = (long)num * a.tiles_x * a.tiles_y;
    if (blocks > 0x7fffffffL) return VIPE_ERR_CAPACITY;
    const size_t smem = fwd_smem(C, num_levels);
    cudaStream_t st = as_stream(stream);
    VIPE_PROF("corr_pyramid", st);
    if (dtype == VIPE_F32) {
        VIPE_CUDA_TRY(cudaFuncSetAttribute(pyramid_fwd_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem));
        pyramid_fwd_kernel<float><<<(unsigned)blocks, kPyrThreads, smem, st>>>(a);
    } else if (dtype == VIPE_F16) {
        VIPE_CUDA_TRY(cudaFuncSetAttribute(pyramid_fwd_kernel<__half>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem));
        pyramid_fwd_kernel<__half><<<(unsigned)blocks, kPyrThreads, smem, st>>>(a);
    } else {
        VIPE_CUDA_TRY(cudaFuncSetAttribute(pyramid_fwd_kernel<__nv_bfloat16>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        pyramid_fwd_kernel<__nv_bfloat16><<<(unsigned)blocks, kPyrThreads, smem, st>>>(a);
    }
    VIPE_LAUNCH_CHECK();
    return VIPE_OK;
}

extern "C" int vipe_corr_pyramid_nhwc_backward(int dtype, const float* const* level_grads, int num, int C, int H,
                                               int W, int num_levels, void* fmaps_grad_out, void* stream) {
    int rc = check_pyramid(dtype, num, C, H, W, num_levels);
    if (rc != VIPE_OK) return rc;
    if (!level_grads || !fmaps_grad_out) return VIPE_ERR_ARG;
    PyrBwdArgs a{};
    for (int l = 0; l < num_levels; l++) {
        if (!level_grads[l]) return VIPE_ERR_ARG;
        a.grad[l] = level_grads[l];
    }
    a.out = fmaps_grad_out;
    a.num = num; a.C = C; a.H = H; a.W = W; a.L = num_levels;
    a.tiles_x = (W + kTileW - 1) / kTileW;
    a.tiles_y = (H + kTileH - 1) / kTileH;
    const long blocks = (long)num * a.tiles_x * a.tiles_y;
    if (blocks > 0x7fffffffL) return VIPE_ERR_CAPACITY;
    const size_t smem = (size_t)C * (kTilePx + 1) * sizeof(float);
    cudaStream_t st = as_stream(stream);
    VIPE_PROF("corr_pyramid_bwd", st);
    if (dtype == VIPE_F32) {
        VIPE_CUDA_TRY(cudaFuncSetAttribute(pyramid_bwd_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem));
        pyramid_bwd_kernel<float><<<(unsigned)blocks, kPyrThreads, smem, st>>>(a);
    } else if (dtype == VIPE_F16) {
        VIPE_CUDA_TRY(cudaFuncSetAttribute(pyramid_bwd_kernel<__half>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem));
        pyramid_bwd_kernel<__half><<<(unsigned)blocks, kPyrThreads, smem, st>>>(a);
    } else {
        VIPE_CUDA_TRY(cudaFuncSetAttribute(pyramid_bwd_kernel<__nv_bfloat16>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        pyramid_bwd_kernel<__nv_bfloat16><<<(unsigned)blocks, kPyrThreads, smem, st>>>(a);
    }
    VIPE_LAUNCH_CHECK();
    return VIPE_OK;
}
