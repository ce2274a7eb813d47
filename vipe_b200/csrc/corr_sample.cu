// Spatial correlation sampler (the reference's corr_ext, used by the AOT tracker's
// attention layers: vipe/priors/track_anything/aot/networks/layers/attention.py:174,305,769).
//
//   out[n][ph][pw][oh][ow] = sum_c sum_{i<kH, j<kW} in1[n][c][y1][x1] * in2[n][c][y1 + s][x1 + t]
//     y1 = oh * dH - padH + i * dilationH,   x1 = ow * dW - padW + j * dilationW,
//     s  = ph * dilation_patchH - dilation_patchH * (patchH - 1) / 2   (t likewise),
// a term counting only when both rows lie in [0, H) and both columns in [0, W)
// (csrc/corr_ext/correlation_cuda_kernel.cu:26-79: the GPU forward's patch radius).
//
// Forward: one thread per (n, ph, oh, ow) keeps a row of up to 16 pw accumulators in
// registers (FP32; FP64 for double maps), so each in1 value it reads serves the whole row;
// consecutive threads take consecutive ow: in1, in2 and the output are read and written
// along rows.  The reference instead gives each output pixel one 32-thread block that loops
// over every patch offset with a shared-memory reduction per offset.
// Backward: gathers, no atomics — one thread per (n, c, y, x) of each input sums, over the
// patch offsets and the kernel taps that reach (y, x), the output gradient times the other
// map, in FP32.  It is the exact adjoint of the forward above (the reference's CUDA backward,
// :82-199, matches it for odd patch sizes).
#include "common.cuh"

#include <cuda_bf16.h>
#include <cuda_fp16.h>

namespace vipe {
namespace {

struct SampleDims {
    int num, C, H, W, kH, kW, pH, pW, padH, padW, dilH, dilW, dpH, dpW, dH, dW, oH, oW;
};

template <typename T>
struct Acc {
    using type = float;
};
template <>
struct Acc<double> {
    using type = double;
};

template <typename T>
__device__ __forceinline__ typename Acc<T>::type ld_acc(const T* p) {
    return (typename Acc<T>::type)(*p);
}
template <>
__device__ __forceinline__ float ld_acc<__half>(const __half* p) { return __half2float(*p); }
template <>
__device__ __forceinline__ float ld_acc<__nv_bfloat16>(const __nv_bfloat16* p) { return __bfloat162float(*p); }

template <typename T>
__device__ __forceinline__ T st_cast(typename Acc<T>::type v) {
    return (T)v;
}
template <>
__device__ __forceinline__ __half st_cast<__half>(float v) { return __float2half_rn(v); }
template <>
__device__ __forceinline__ __nv_bfloat16 st_cast<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }

constexpr int kRowAcc = 16;  // pw accumulators a forward thread keeps in registers

__device__ __forceinline__ int patch_shift(int p, int dp, int P) { return p * dp - dp * (P - 1) / 2; }

template <typename T>
__global__ void __launch_bounds__(256) corr_sample_fwd_kernel(const T* __restrict__ in1, const T* __restrict__ in2,
                                                              T* __restrict__ out, SampleDims d) {
    using A = typename Acc<T>::type;
    const long total = (long)d.num * d.pH * d.oH * d.oW;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    const int ow = (int)(t % d.oW);
    const int oh = (int)((t / d.oW) % d.oH);
    const int ph = (int)((t / ((long)d.oW * d.oH)) % d.pH);
    const int n = (int)(t / ((long)d.oW * d.oH * d.pH));
    const int s = patch_shift(ph, d.dpH, d.pH);
    const size_t plane = (size_t)d.H * d.W;
    const T* a1 = in1 + (size_t)n * d.C * plane;
    const T* a2 = in2 + (size_t)n * d.C * plane;
    for (int pw0 = 0; pw0 < d.pW; pw0 += kRowAcc) {
        A acc[kRowAcc];
#pragma unroll
        for (int q = 0; q < kRowAcc; q++) acc[q] = A(0);
        for (int i = 0; i < d.kH; i++) {
            const int y1 = oh * d.dH - d.padH + i * d.dilH, y2 = y1 + s;
            if (y1 < 0 || y1 >= d.H || y2 < 0 || y2 >= d.H) continue;
            for (int j = 0; j < d.kW; j++) {
                const int x1 = ow * d.dW - d.padW + j * d.dilW;
                if (x1 < 0 || x1 >= d.W) continue;
                for (int c = 0; c < d.C; c++) {
                    const A v1 = ld_acc<T>(a1 + c * plane + (size_t)y1 * d.W + x1);
                    const T* r2 = a2 + c * plane + (size_t)y2 * d.W;
#pragma unroll
                    for (int q = 0; q < kRowAcc; q++) {
                        const int pw = pw0 + q;
                        const int x2 = x1 + patch_shift(pw, d.dpW, d.pW);
                        if (pw < d.pW && x2 >= 0 && x2 < d.W) acc[q] += v1 * ld_acc<T>(r2 + x2);
                    }
                }
            }
        }
#pragma unroll
        for (int q = 0; q < kRowAcc; q++) {
            const int pw = pw0 + q;
            if (pw < d.pW)
                out[((((size_t)n * d.pH + ph) * d.pW + pw) * d.oH + oh) * d.oW + ow] = st_cast<T>(acc[q]);
        }
    }
}

// which == 1: gradient of in1 (partner: in2 at +shift); which == 2: of in2 (partner: in1 at -shift)
template <typename T, int which>
__global__ void __launch_bounds__(256) corr_sample_bwd_kernel(const T* __restrict__ partner,
                                                              const T* __restrict__ gout, T* __restrict__ grad,
                                                              SampleDims d) {
    using A = typename Acc<T>::type;
    const long total = (long)d.num * d.C * d.H * d.W;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    const int x = (int)(t % d.W);
    const int y = (int)((t / d.W) % d.H);
    const int c = (int)((t / ((long)d.W * d.H)) % d.C);
    const int n = (int)(t / ((long)d.W * d.H * d.C));
    const size_t plane = (size_t)d.H * d.W;
    const T* pm = partner + ((size_t)n * d.C + c) * plane;
    const T* g = gout + (size_t)n * d.pH * d.pW * d.oH * d.oW;
    A acc = A(0);
    for (int ph = 0; ph < d.pH; ph++) {
        const int s = patch_shift(ph, d.dpH, d.pH);
        // (y1, y2) of the forward term: this element is y1 (which == 1) or y2 (which == 2)
        const int y1 = which == 1 ? y : y - s, y2 = y1 + s;
        if (y1 < 0 || y1 >= d.H || y2 < 0 || y2 >= d.H) continue;
        for (int pw = 0; pw < d.pW; pw++) {
            const int tsh = patch_shift(pw, d.dpW, d.pW);
            const int x1 = which == 1 ? x : x - tsh, x2 = x1 + tsh;
            if (x1 < 0 || x1 >= d.W || x2 < 0 || x2 >= d.W) continue;
            const A v = ld_acc<T>(pm + (which == 1 ? (size_t)y2 * d.W + x2 : (size_t)y1 * d.W + x1));
            const T* gp = g + ((size_t)ph * d.pW + pw) * d.oH * d.oW;
            // output pixels whose kernel taps reach row y1 / column x1
            for (int i = 0; i < d.kH; i++) {
                const int ny = y1 + d.padH - i * d.dilH;
                if (ny < 0 || ny % d.dH) continue;
                const int oh = ny / d.dH;
                if (oh >= d.oH) continue;
                for (int j = 0; j < d.kW; j++) {
                    const int nx = x1 + d.padW - j * d.dilW;
                    if (nx < 0 || nx % d.dW) continue;
                    const int ow = nx / d.dW;
                    if (ow >= d.oW) continue;
                    acc += ld_acc<T>(gp + (size_t)oh * d.oW + ow) * v;
                }
            }
        }
    }
    grad[t] = st_cast<T>(acc);
}

int make_sample_dims(int num, int C, int H, int W, int kH, int kW, int pH, int pW, int padH, int padW, int dilH,
                     int dilW, int dpH, int dpW, int dH, int dW, SampleDims* d) {
    if (num <= 0 || C <= 0 || H <= 0 || W <= 0 || kH <= 0 || kW <= 0 || pH <= 0 || pW <= 0 || padH < 0 ||
        padW < 0 || dilH <= 0 || dilW <= 0 || dpH <= 0 || dpW <= 0 || dH <= 0 || dW <= 0)
        return VIPE_ERR_ARG;
    const int oH = (H + 2 * padH - ((kH - 1) * dilH + 1)) / dH + 1;
    const int oW = (W + 2 * padW - ((kW - 1) * dilW + 1)) / dW + 1;
    if (oH <= 0 || oW <= 0) return VIPE_ERR_ARG;
    *d = SampleDims{num, C, H, W, kH, kW, pH, pW, padH, padW, dilH, dilW, dpH, dpW, dH, dW, oH, oW};
    return VIPE_OK;
}

}  // namespace
}  // namespace vipe

using namespace vipe;

extern "C" int vipe_corr_sample_forward(int dtype, const void* input1, const void* input2, int num, int C, int H,
                                        int W, int kH, int kW, int patchH, int patchW, int padH, int padW,
                                        int dilationH, int dilationW, int dilation_patchH, int dilation_patchW,
                                        int dH, int dW, void* out, void* stream) {
    SampleDims d;
    int rc = make_sample_dims(num, C, H, W, kH, kW, patchH, patchW, padH, padW, dilationH, dilationW,
                              dilation_patchH, dilation_patchW, dH, dW, &d);
    if (rc != VIPE_OK) return rc;
    if (!input1 || !input2 || !out) return VIPE_ERR_ARG;
    const long total = (long)num * patchH * d.oH * d.oW;
    const unsigned blocks = ceil_div((size_t)total, 256);
    cudaStream_t st = as_stream(stream);
    VIPE_PROF("corr_sample_fwd", st);
    switch (dtype) {
        case VIPE_F32:
            corr_sample_fwd_kernel<float><<<blocks, 256, 0, st>>>((const float*)input1, (const float*)input2,
                                                                  (float*)out, d);
            break;
        case VIPE_F64:
            corr_sample_fwd_kernel<double><<<blocks, 256, 0, st>>>((const double*)input1, (const double*)input2,
                                                                   (double*)out, d);
            break;
        case VIPE_F16:
            corr_sample_fwd_kernel<__half><<<blocks, 256, 0, st>>>((const __half*)input1, (const __half*)input2,
                                                                   (__half*)out, d);
            break;
        case VIPE_BF16:
            corr_sample_fwd_kernel<__nv_bfloat16><<<blocks, 256, 0, st>>>(
                (const __nv_bfloat16*)input1, (const __nv_bfloat16*)input2, (__nv_bfloat16*)out, d);
            break;
        default:
            return VIPE_ERR_DTYPE;
    }
    VIPE_LAUNCH_CHECK();
    return VIPE_OK;
}

template <typename T>
static void launch_sample_bwd(const void* in1, const void* in2, const void* gout, void* g1, void* g2,
                              const SampleDims& d, unsigned blocks, cudaStream_t st) {
    corr_sample_bwd_kernel<T, 1><<<blocks, 256, 0, st>>>((const T*)in2, (const T*)gout, (T*)g1, d);
    corr_sample_bwd_kernel<T, 2><<<blocks, 256, 0, st>>>((const T*)in1, (const T*)gout, (T*)g2, d);
}

extern "C" int vipe_corr_sample_backward(int dtype, const void* input1, const void* input2, const void* grad_output,
                                         int num, int C, int H, int W, int kH, int kW, int patchH, int patchW,
                                         int padH, int padW, int dilationH, int dilationW, int dilation_patchH,
                                         int dilation_patchW, int dH, int dW, void* grad_input1_out,
                                         void* grad_input2_out, void* stream) {
    SampleDims d;
    int rc = make_sample_dims(num, C, H, W, kH, kW, patchH, patchW, padH, padW, dilationH, dilationW,
                              dilation_patchH, dilation_patchW, dH, dW, &d);
    if (rc != VIPE_OK) return rc;
    if (!input1 || !input2 || !grad_output || !grad_input1_out || !grad_input2_out) return VIPE_ERR_ARG;
    const long total = (long)num * C * H * W;
    const unsigned blocks = ceil_div((size_t)total, 256);
    cudaStream_t st = as_stream(stream);
    VIPE_PROF("corr_sample_bwd", st);
    switch (dtype) {
        case VIPE_F32: launch_sample_bwd<float>(input1, input2, grad_output, grad_input1_out, grad_input2_out, d,
                                                blocks, st); break;
        case VIPE_F64: launch_sample_bwd<double>(input1, input2, grad_output, grad_input1_out, grad_input2_out, d,
                                                 blocks, st); break;
        case VIPE_F16: launch_sample_bwd<__half>(input1, input2, grad_output, grad_input1_out, grad_input2_out, d,
                                                 blocks, st); break;
        case VIPE_BF16: launch_sample_bwd<__nv_bfloat16>(input1, input2, grad_output, grad_input1_out,
                                                         grad_input2_out, d, blocks, st); break;
        default: return VIPE_ERR_DTYPE;
    }
    VIPE_LAUNCH_CHECK();
    return VIPE_OK;
}
