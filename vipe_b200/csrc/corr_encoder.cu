// The correlation lookup fused with the first layer of the DROID update operator.
//
// Reference: UpdateModule.forward (vipe/slam/networks/droid_net.py:452-519) receives the
// CorrBlock lookup (droid_net.py:94-102: per level l, corr_index_forward of the volume at
// coords / 2^l, radius 3, 49 channels each, concatenated: 196 channels, channel
// l*49 + i*7 + j with i the x offset) and runs corr_encoder = Conv2d(196, 128, 1) + ReLU +
// Conv2d(128, 128, 3) + ReLU.  The 196-channel lookup is written to HBM and read back by the
// 1x1 convolution (a GEMM over channels).  Here one kernel does both:
//
//   out[b][o][p] = ReLU(bias[o] + sum_k Wt[o][k] corr[b][k][p])        (o < 128, k < 196)
//
//   * persistent CTAs (one per SM) walk (pair, 128-pixel block) work items;
//   * all eight warps produce the A operand — one thread per (pixel, level) reads its 8 x 8
//     window of the level volume (16-byte row loads where the row allows) and writes the 49
//     bilinear values, rounded to the volume type, into the pixel's row of a 128 x 196
//     K-major, 128-byte-swizzled shared-memory tile (K padded with zeros to 208);
//   * the 1x1 convolution's weights are the B operand, staged once per CTA (128 x 208);
//   * one thread issues the 13 tcgen05.mma.kind::f16 (M = N = 128, K = 16) of a work item
//     into one of two tensor-memory accumulators, so the MMAs of item t overlap the
//     epilogue of item t-1 and the lookup of item t+1;
//   * the epilogue (tcgen05.ld, one pixel per thread) adds the bias, applies the ReLU and
//     writes the 128 output channels with consecutive lanes on consecutive pixels.
// The 196-channel lookup never leaves the chip.  Every mbarrier wait is bounded (2 s): on
// expiry the CTA sets the error word, stops, waits once more for its committed MMAs and frees
// its tensor memory.
#include "corr_window.cuh"
#include "tcgen05.cuh"

#include <algorithm>
#include <type_traits>

namespace vipe {
namespace cenc {

using namespace ::vipe::tc;
using ::vipe::corr::from_f;
using ::vipe::corr::inb;
using ::vipe::corr::to_f;
using ::vipe::corr::window_origin;
using ::vipe::corr::window_row8;

constexpr int kThreads = 256;
constexpr int kTile = 128;             // pixels (M) and output channels (N)
constexpr int kLevelsMax = 4;
constexpr int kK = 4 * 49;             // lookup channels
constexpr int kKSteps = 13;            // K = 208 in MMA steps of 16
constexpr int kBlk = kTile * 128;      // one 64-element K block of a 128-row operand (bytes)
constexpr int kOpBytes = 4 * kBlk;     // 128 rows x 256 K elements (blocks 0..3)
constexpr uint64_t kWaitNs = 2000000000ull;

struct Params {
    const void* vol[kLevelsMax];  // level l: (B, H, W, H >> l, W >> l)
    const float* coords;          // (B, 2, H, W) at level 0
    const void* weight;           // (128, 196)
    const float* bias;            // (128,)
    void* out;                    // (B, 128, H, W)
    int* err;
    int B, H, W, HW, L, blocks;   // blocks: 128-pixel blocks per pair
    long items;
};

__device__ __forceinline__ uint32_t sw_off(int r, int k) {
    const int byte = (k & 63) * 2;
    return (uint32_t)(k >> 6) * kBlk + (uint32_t)r * 128u + ((uint32_t)(((byte >> 4) ^ r) & 7) << 4) +
           (uint32_t)(byte & 15);
}

// the 8 x 8 window of one level around (x, y), rows that do not fill whole 16-byte chunks
// (narrow coarse levels) read element by element
template <typename T>
__device__ __forceinline__ void window8(const T* plane, int h2, int w2, int by, int bx, float (*t)[8]) {
    if (((size_t)w2 * sizeof(T)) % 16 == 0) {
#pragma unroll
        for (int j = 0; j < 8; j++) window_row8<T>(plane, h2, w2, by + j, bx, t[j]);
    } else {
#pragma unroll
        for (int j = 0; j < 8; j++)
#pragma unroll
            for (int i = 0; i < 8; i++)
                t[j][i] = inb(by + j, bx + i, h2, w2) ? to_f(plane[(int64_t)(by + j) * w2 + bx + i]) : 0.f;
    }
}

template <typename T>
__device__ void produce(const Params& a, long item, uint8_t* sA) {
    const int n = (int)(item / a.blocks), p0 = (int)(item % a.blocks) * kTile;
    for (int task = threadIdx.x; task < kTile * a.L; task += kThreads) {
        const int r = task % kTile, l = task / kTile;
        const int p = p0 + r;
        if (p >= a.HW) {
            for (int q = 0; q < 49; q++) *reinterpret_cast<T*>(sA + sw_off(r, l * 49 + q)) = from_f<T>(0.f);
            continue;
        }
        const float s = 1.f / (float)(1 << l);
        const float x0 = a.coords[((int64_t)n * 2 + 0) * a.HW + p] * s;
        const float y0 = a.coords[((int64_t)n * 2 + 1) * a.HW + p] * s;
        const float fx0 = floorf(x0), fy0 = floorf(y0);
        const bool near = fabsf(x0) < 1e6f && fabsf(y0) < 1e6f;
        const float dx = near ? x0 - fx0 : 0.f, dy = near ? y0 - fy0 : 0.f;
        const int bx = near ? window_origin(fx0, 3) : -64, by = near ? window_origin(fy0, 3) : -64;
        const int h2 = a.H >> l, w2 = a.W >> l;
        const T* plane = static_cast<const T*>(a.vol[l]) + ((int64_t)n * a.HW + p) * ((int64_t)h2 * w2);
        float t[8][8];
        window8<T>(plane, h2, w2, by, bx, t);
#pragma unroll
        for (int i = 0; i < 7; i++)
#pragma unroll
            for (int j = 0; j < 7; j++) {
                float v = (1 - dx) * (1 - dy) * t[j][i];
                v += dx * (1 - dy) * t[j][i + 1];
                v += (1 - dx) * dy * t[j + 1][i];
                v += dx * dy * t[j + 1][i + 1];
                *reinterpret_cast<T*>(sA + sw_off(r, l * 49 + i * 7 + j)) = from_f<T>(v);
            }
    }
}

template <typename T>
__device__ __forceinline__ void epilogue(const Params& a, long item, uint32_t acc, const float* bsh) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int n = (int)(item / a.blocks), p = (int)(item % a.blocks) * kTile + 32 * (warp & 3) + lane;
    const int cbase = (warp >> 2) * 64;  // warps 4-7 read the same lanes' upper 64 columns
    T* out = static_cast<T*>(a.out) + (int64_t)n * kTile * a.HW;
    for (int c0 = cbase; c0 < cbase + 64; c0 += 16) {
        float v[16];
        tmem_ld16(acc + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)c0, v);
        tmem_wait_ld();
        if (p < a.HW) {
#pragma unroll
            for (int j = 0; j < 16; j++) out[(int64_t)(c0 + j) * a.HW + p] = from_f<T>(fmaxf(v[j] + bsh[c0 + j], 0.f));
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(kThreads, 1) corr_encoder_kernel(Params a) {
    constexpr int FMT = std::is_same<T, __half>::value ? kFmtF16 : kFmtBF16;
    extern __shared__ uint8_t sm_raw[];
    __shared__ uint64_t bar[2];
    __shared__ uint32_t tmem_base;
    __shared__ int fail;
    __shared__ float bsh[kTile];
    uint8_t* sm = sm_raw + ((1024u - (smem_u32(sm_raw) & 1023u)) & 1023u);
    uint8_t* sB = sm;
    uint8_t* sA[2] = {sm + kOpBytes, sm + 2 * kOpBytes};
    const int tid = threadIdx.x, warp = tid >> 5;
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fail = 0;
        fence_barrier_init();
    }
    if (warp == 0) tmem_alloc(&tmem_base, 2 * kTile);
    // the 1x1 convolution's weights (K padded with zeros), the zero K pads of both A buffers, the bias
    const T* wt = static_cast<const T*>(a.weight);
    for (int idx = tid; idx < kTile * 256; idx += kThreads) {
        const int o = idx >> 8, k = idx & 255;
        *reinterpret_cast<T*>(sB + sw_off(o, k)) = k < kK ? wt[o * kK + k] : from_f<T>(0.f);
    }
    for (int idx = tid; idx < 2 * kTile * (256 - kK); idx += kThreads) {
        const int b = idx / (kTile * (256 - kK)), rem = idx % (kTile * (256 - kK));
        *reinterpret_cast<T*>(sA[b] + sw_off(rem / (256 - kK), kK + rem % (256 - kK))) = from_f<T>(0.f);
    }
    for (int o = tid; o < kTile; o += kThreads) bsh[o] = a.bias ? a.bias[o] : 0.f;
    fence_proxy_async();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base;
    const uint32_t idesc = instr_desc(FMT, kTile, kTile);
    long prev = -1;
    int it = 0, committed = 0;
    for (long item = blockIdx.x;; item += gridDim.x, it++) {
        const bool have = item < a.items;
        const int s = it & 1;
        if (have) {
            // buffer s was last read by the MMAs of item it-2, complete before its epilogue
            produce<T>(a, item, sA[s]);
            fence_proxy_async();
        }
        __syncthreads();
        if (have && tid == 0) {
            tc_fence_after();
            const uint64_t da = smem_desc_sw128(sA[s]), db = smem_desc_sw128(sB);
#pragma unroll
            for (int ks = 0; ks < kKSteps; ks++) {
                const uint64_t off = (uint64_t)(((ks >> 2) * kBlk) >> 4) + (uint64_t)((ks & 3) * 2);
                mma_f16(tmem + (uint32_t)(s * kTile), da + off, db + off, idesc, ks > 0 ? 1u : 0u);
            }
            mma_commit(&bar[s]);
        }
        if (have) committed++;
        if (prev >= 0) {
            const int pit = it - 1, ps = pit & 1;
            if (tid == 0 && !mbar_wait_bounded(&bar[ps], (uint32_t)(pit >> 1) & 1u, kWaitNs)) fail = 1;
            __syncthreads();
            if (fail) break;
            tc_fence_after();
            epilogue<T>(a, prev, tmem + (uint32_t)(ps * kTile), bsh);
            tc_fence_before();
        }
        if (!have) break;
        prev = item;
        __syncthreads();  // the accumulator just read is the next item's MMA target
    }
    if (fail && tid == 0) {
        atomicOr(a.err, 1);
        // the last committed MMAs get one more bounded chance before their tensor memory is freed
        if (committed > 0)
            mbar_wait_bounded(&bar[(committed - 1) & 1], (uint32_t)((committed - 1) >> 1) & 1u, kWaitNs);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, 2 * kTile);
    }
}

int g_sms = 0;

}  // namespace cenc
}  // namespace vipe

using namespace vipe;
using namespace vipe::cenc;

extern "C" int vipe_corr_encoder_lookup(int dtype, const void* const* levels, int num_levels, const float* coords,
                                        int B, int H, int W, const void* weight, const float* bias, void* out,
                                        int32_t* dev_status, void* stream) {
    if (dtype != VIPE_F16 && dtype != VIPE_BF16) return VIPE_ERR_DTYPE;
    if (B <= 0 || H <= 0 || W <= 0 || num_levels != kLevelsMax || (H >> 3) == 0 || (W >> 3) == 0) {
        set_last_error("corr encoder lookup: 4 pyramid levels of radius 3 (196 channels), H and W >= 8");
        return VIPE_ERR_ARG;
    }
    if (!levels || !coords || !weight || !out || !dev_status) return VIPE_ERR_ARG;
    Params p{};
    for (int l = 0; l < num_levels; l++) {
        if (!levels[l]) return VIPE_ERR_ARG;
        p.vol[l] = levels[l];
    }
    p.coords = coords;
    p.weight = weight;
    p.bias = bias;
    p.out = out;
    p.err = dev_status;
    p.B = B; p.H = H; p.W = W; p.HW = H * W; p.L = num_levels;
    p.blocks = (p.HW + kTile - 1) / kTile;
    p.items = (long)B * p.blocks;
    if (g_sms == 0) {
        int dev = 0;
        VIPE_CUDA_TRY(cudaGetDevice(&dev));
        VIPE_CUDA_TRY(cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev));
    }
    const unsigned grid = (unsigned)std::min<long>(p.items, g_sms);
    const size_t smem = 3 * (size_t)kOpBytes + 1024;
    cudaStream_t st = as_stream(stream);
    VIPE_PROF("corr_encoder_lookup", st);
    if (dtype == VIPE_F16) {
        VIPE_CUDA_TRY(cudaFuncSetAttribute(corr_encoder_kernel<__half>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem));
        corr_encoder_kernel<__half><<<grid, kThreads, smem, st>>>(p);
    } else {
        VIPE_CUDA_TRY(cudaFuncSetAttribute(corr_encoder_kernel<__nv_bfloat16>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        corr_encoder_kernel<__nv_bfloat16><<<grid, kThreads, smem, st>>>(p);
    }
    VIPE_LAUNCH_CHECK();
    return VIPE_OK;
}
