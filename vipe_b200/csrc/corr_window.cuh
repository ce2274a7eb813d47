// Element conversions and the radius-3 window loads shared by the correlation
// lookup kernels (corr.cu) and the lookup fused with the update operator's first
// layer (corr_encoder.cu).
#pragma once

#include "common.cuh"

#include <cuda_bf16.h>
#include <cuda_fp16.h>

namespace vipe {
namespace corr {

template <typename T>
__device__ __forceinline__ float to_f(T v) {
    return static_cast<float>(v);
}
template <>
__device__ __forceinline__ float to_f<__half>(__half v) {
    return __half2float(v);
}
template <>
__device__ __forceinline__ float to_f<__nv_bfloat16>(__nv_bfloat16 v) {
    return __bfloat162float(v);
}

template <typename T>
__device__ __forceinline__ T from_f(float v) {
    return static_cast<T>(v);
}
template <>
__device__ __forceinline__ __half from_f<__half>(float v) {
    return __float2half_rn(v);
}
template <>
__device__ __forceinline__ __nv_bfloat16 from_f<__nv_bfloat16>(float v) {
    return __float2bfloat16_rn(v);
}

__device__ __forceinline__ bool inb(int h, int w, int H, int W) { return h >= 0 && h < H && w >= 0 && w < W; }

// Integer window origin floor(c) - r.  The floored coordinate is clamped to
// +-2^24 first: any coordinate beyond that is outside every map anyway, and the
// clamp keeps the window arithmetic (origin + tap offset) clear of int overflow
// for huge or non-finite coordinates, whose taps then all fail the bounds test.
__device__ __forceinline__ int window_origin(float floored, int r) {
    return (int)fminf(fmaxf(floored, -16777216.f), 16777216.f) - r;
}

// Radius-3 lookup with vector loads.  Each pixel reads its own plane, so the
// lanes of a warp never share a row: instead of 196 scattered element loads,
// each of the 8 window rows is read as the aligned 16-byte chunks covering
// [bx, bx + 8) (two for 16-bit types, three for f32) and shifted into place in
// registers.  Needs rows that are a whole number of 16-byte chunks (w2 * size
// a multiple of 16) and a 16-byte aligned volume; a chunk is then either inside
// the row or entirely outside it, and outside chunks read as zeros.
template <typename T>
__device__ __forceinline__ void window_row8(const T* __restrict__ plane, int h2, int w2, int y, int x0, float* t) {
    const bool rowok = y >= 0 && y < h2;
    const T* rp = plane + (int64_t)(rowok ? y : 0) * w2;
    if constexpr (sizeof(T) == 2) {
        const int o = x0 & 7, a = x0 - o;  // floor to a multiple of 8 elements (also for x0 < 0)
        uint4 c0 = make_uint4(0, 0, 0, 0), c1 = c0;
        if (rowok && a >= 0 && a < w2) c0 = __ldg(reinterpret_cast<const uint4*>(rp + a));
        if (rowok && a + 8 >= 0 && a + 8 < w2) c1 = __ldg(reinterpret_cast<const uint4*>(rp + a + 8));
        const uint32_t w[8] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
        uint32_t wa[6], wb[5];
#pragma unroll
        for (int k = 0; k < 6; k++) wa[k] = (o & 4) ? w[k + 2] : w[k];  // shift by 2 words
#pragma unroll
        for (int k = 0; k < 5; k++) wb[k] = (o & 2) ? wa[k + 1] : wa[k];  // by 1 word
#pragma unroll
        for (int k = 0; k < 4; k++) {
            // word k holds elements o + 2k (low half) and o + 2k + 1 (high half)
            const uint32_t v = (o & 1) ? __funnelshift_r(wb[k], wb[k + 1], 16) : wb[k];
            const T* e = reinterpret_cast<const T*>(&v);
            t[2 * k] = to_f(e[0]);
            t[2 * k + 1] = to_f(e[1]);
        }
    } else {
        const int o = x0 & 3, a = x0 - o;
        float4 c[3];
#pragma unroll
        for (int q = 0; q < 3; q++) {
            c[q] = make_float4(0.f, 0.f, 0.f, 0.f);
            const int s = a + 4 * q;
            if (rowok && s >= 0 && s < w2) c[q] = __ldg(reinterpret_cast<const float4*>(rp + s));
        }
        const float f[12] = {c[0].x, c[0].y, c[0].z, c[0].w, c[1].x, c[1].y,
                             c[1].z, c[1].w, c[2].x, c[2].y, c[2].z, c[2].w};
        float fa[10];
#pragma unroll
        for (int k = 0; k < 10; k++) fa[k] = (o & 2) ? f[k + 2] : f[k];
#pragma unroll
        for (int k = 0; k < 8; k++) t[k] = (o & 1) ? fa[k + 1] : fa[k];
    }
}

}  // namespace corr
}  // namespace vipe
