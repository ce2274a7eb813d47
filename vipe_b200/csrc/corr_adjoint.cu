// Adjoint of the correlation-volume pyramid build on tcgen05 tensor cores.
//
// The reference differentiates CorrBlock's volume (vipe/slam/networks/droid_net.py:56-69,
// 94-102: V = (F1/4)^T (F2/4) over channels, level l = avg_pool2d^l(V) over the target
// axes) with torch autograd: per level a matmul backward (two cuBLAS GEMMs) and the
// avg_pool2d backward.  Pooling is linear, so with G_l the level gradients the whole
// pyramid backward is two GEMMs with one unpooled gradient
//     Gt[p][q] = sum_l G_l[p][Q_l(q)] / 4^l          (Q_l(q): q's pixel at level l)
//     dF1 = (1/16) F2 Gt^T        dF2 = (1/16) F1 Gt        (C x HW each, K = HW)
// and Gt never needs to exist in memory: the CTA's producer warps form each K-block of
// it from the level gradients (one 16-byte row chunk of G_0 and 8 >> l values of G_l per
// 8 target pixels) straight into the 128-byte-swizzled K-major operand layout.
//
// One CTA per (pair, 128-pixel output block, pass); M = 128 channels (rows >= C are
// zero), N = 128 output pixels, K walked in 128-byte blocks through two shared-memory
// stages: all 8 warps stage block k+1 while the tensor cores multiply block k.
//   pass 0 (dF1): A = F2 [c][q] (K = q), B = Gt [p][q] rows of the output block;
//   pass 1 (dF2): A = F1 [c][p] (K = p), B = Gt^T [q][p]: the producers read Gt row
//                 chunks along q and scatter them into the B rows of their q.
// Operand kinds: 16-bit maps with 16-bit level gradients run kind::f16 (Gt rounded to the
// map type once); FP32 level gradients run kind::tf32 with Gt split into TF32 hi + lo
// (two MMAs; the maps are exact in TF32), so FP32 volumes keep FP32-level accuracy.
// The FP32 accumulator (128 x 128 in tensor memory) is read by tcgen05.ld, scaled by
// 1/16 and written once.  Every mbarrier wait is bounded (2 s): on expiry the CTA sets
// the error word, waits once more for its committed MMAs and frees its tensor memory.
#include "common.cuh"
#include "corr_window.cuh"
#include "tcgen05.cuh"
#include "tma.cuh"

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <type_traits>

namespace vipe {
namespace cadj {

using namespace ::vipe::tc;
using ::vipe::corr::to_f;

constexpr int kThreads = 256;
constexpr int kTile = 128;                   // M (channels) and N (output pixels)
constexpr int kOpBytes = kTile * 128;        // one K-major operand block: 128 rows x 128 B
constexpr uint64_t kWaitNs = 2000000000ull;  // bound on every mbarrier wait
constexpr int kMaxLevels = 4;

struct Params {
    const void* fa;               // pass 0: fmap2, pass 1: fmap1 (num, C, HW), operand storage type
    const void* g[kMaxLevels];    // level gradients (num, HW, HW >> 2l)
    float* out;                   // (num, C, HW) FP32
    int* err;
    int num, C, H, W, HW, L, pass, gdt;  // gdt: level-gradient dtype (vipe_dtype)
    int blocks;                   // output pixel blocks per pair (HW / 128)
};

__device__ __forceinline__ float ld_any(const void* p, size_t i, int dt) {
    if (dt == VIPE_F32) return static_cast<const float*>(p)[i];
    if (dt == VIPE_F16) return __half2float(static_cast<const __half*>(p)[i]);
    return __bfloat162float(static_cast<const __nv_bfloat16*>(p)[i]);
}

// Pooled part of Gt for one pair of target pixels (x, x+1 with x even): levels 1 .. L-1, each
// / 4^l, summed in this order.  Both kernels form Gt = G_0 + level_sum, so they round alike.
__device__ __forceinline__ float level_sum(float l1, float l2, float l3, int L) {
    float s = 0.25f * l1;
    if (L > 2) s = fmaf(0.0625f, l2, s);
    if (L > 3) s = fmaf(0.015625f, l3, s);
    return s;
}

// Gt[p][q .. q+7] (8 consecutive target pixels in one image row, q % 8 == 0): level 0 as one
// row chunk plus level_sum of the pooled values that cover each pixel pair
__device__ __forceinline__ void unpooled8(const Params& a, int n, int p, int q, float* o) {
    const int W = a.W, y = q / W, x = q % W;
    const size_t HW = (size_t)a.HW;
    const size_t row0 = ((size_t)n * HW + p) * HW + (size_t)y * W + x;
    if (a.gdt == VIPE_F32) {
        const float4* src = reinterpret_cast<const float4*>(static_cast<const float*>(a.g[0]) + row0);
        const float4 u = src[0], v = src[1];
        o[0] = u.x; o[1] = u.y; o[2] = u.z; o[3] = u.w;
        o[4] = v.x; o[5] = v.y; o[6] = v.z; o[7] = v.w;
    } else {
        const uint4 raw = *reinterpret_cast<const uint4*>(static_cast<const uint16_t*>(a.g[0]) + row0);
        const uint16_t* h = reinterpret_cast<const uint16_t*>(&raw);
#pragma unroll
        for (int i = 0; i < 8; i++)
            o[i] = a.gdt == VIPE_F16 ? __half2float(__ushort_as_half(h[i])) : __bfloat162float(__ushort_as_bfloat16(h[i]));
    }
    if (a.L < 2) return;
    float lv[4][4];  // [level][pixel pair]: the pooled value covering pair k (levels 1..3)
    for (int l = 1; l < 4; l++) {
        if (l >= a.L) {
#pragma unroll
            for (int k = 0; k < 4; k++) lv[l][k] = 0.f;
            continue;
        }
        const int Wl = W >> l, HWl = (int)(HW >> (2 * l));
        const size_t row = ((size_t)n * HW + p) * HWl + (size_t)(y >> l) * Wl + (x >> l);
#pragma unroll
        for (int k = 0; k < 4; k++) lv[l][k] = ld_any(a.g[l], row + ((2 * k) >> l), a.gdt);
    }
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const float sk = level_sum(lv[1][k], lv[2][k], lv[3][k], a.L);
        o[2 * k] += sk;
        o[2 * k + 1] += sk;
    }
}

// byte offset of element k (of `ebytes` bytes) in row r of a K-major 128-byte-swizzled block
__device__ __forceinline__ uint32_t sw_off(int r, int k, int ebytes) {
    const int byte = k * ebytes;
    return (uint32_t)r * 128u + ((uint32_t)(((byte >> 4) ^ r) & 7) << 4) + (uint32_t)(byte & 15);
}

template <typename T>
__device__ __forceinline__ T to_op(float v);
template <>
__device__ __forceinline__ __half to_op<__half>(float v) { return __float2half_rn(v); }
template <>
__device__ __forceinline__ __nv_bfloat16 to_op<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }
template <>
__device__ __forceinline__ float to_op<float>(float v) { return v; }

// fmap chunk (VE operand elements from row c, elements k .. k+VE-1) as 16 bytes of the operand
template <typename OpT, typename FT>
__device__ __forceinline__ uint4 fmap_chunk(const FT* row, int k, bool live) {
    uint4 out = make_uint4(0, 0, 0, 0);
    if (!live) return out;
    if constexpr (sizeof(OpT) == 2) {
        out = *reinterpret_cast<const uint4*>(row + k);  // same 16-bit type: a plain copy
    } else {
        float* f = reinterpret_cast<float*>(&out);
        const uint2 raw = *reinterpret_cast<const uint2*>(row + k);
        const uint16_t* h = reinterpret_cast<const uint16_t*>(&raw);
#pragma unroll
        for (int i = 0; i < 4; i++) {
            if constexpr (std::is_same<FT, __half>::value)
                f[i] = __half2float(__ushort_as_half(h[i]));
            else
                f[i] = __bfloat162float(__ushort_as_bfloat16(h[i]));
        }
    }
    return out;
}

template <typename OpT, typename FT, bool kSplit>
__global__ void __launch_bounds__(kThreads, 1) corr_vol_bwd_kernel(Params a) {
    constexpr int EB = (int)sizeof(OpT);  // bytes per operand element
    constexpr int KB = 128 / EB;          // K elements per 128-byte block
    constexpr int VE = 16 / EB;           // elements per 16-byte chunk
    constexpr int NOP = kSplit ? 3 : 2;   // operand blocks per stage: A, B (, B lo)
    constexpr int FMT = kSplit ? kFmtTF32 : (std::is_same<OpT, __half>::value ? kFmtF16 : kFmtBF16);
    extern __shared__ uint8_t sm_raw[];
    __shared__ uint64_t bar[2];
    __shared__ uint32_t tmem_base;
    __shared__ int fail;
    uint8_t* sm = sm_raw + ((1024u - (smem_u32(sm_raw) & 1023u)) & 1023u);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int n = blockIdx.x / a.blocks, o0 = (blockIdx.x % a.blocks) * kTile;
    const int C = a.C, HW = a.HW;
    const FT* fa = static_cast<const FT*>(a.fa) + (size_t)n * C * HW;
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fail = 0;
        fence_barrier_init();
    }
    if (warp == 0) tmem_alloc(&tmem_base, kTile);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base;
    const uint32_t idesc = instr_desc(FMT, kTile, kTile);
    const int nk = HW / KB;
    int committed = 0;
    for (int kb = 0; kb < nk; kb++) {
        const int s = kb & 1;
        if (kb >= 2) {
            // the MMAs that read this stage two blocks ago must be done
            if (tid == 0 && !mbar_wait_bounded(&bar[s], (uint32_t)((kb >> 1) - 1) & 1u, kWaitNs)) fail = 1;
            __syncthreads();
            if (fail) break;
        }
        uint8_t* sA = sm + (size_t)s * NOP * kOpBytes;
        uint8_t* sB = sA + kOpBytes;
        uint8_t* sBl = sB + kOpBytes;
        const int k0 = kb * KB;
        // A: the other map's rows (channels), K = this block's pixels
        for (int q = tid; q < kTile * 8; q += kThreads) {
            const int r = q >> 3, cc = q & 7;
            const uint4 v = fmap_chunk<OpT, FT>(fa + (size_t)min(r, C - 1) * HW, k0 + cc * VE, r < C);
            *reinterpret_cast<uint4*>(sA + sw_off(r, cc * VE, EB)) = v;
        }
        // B: the unpooled gradient, 8 target pixels at a time
        constexpr int G8 = KB / 8;  // 8-pixel groups along K
        for (int q = tid; q < kTile * G8; q += kThreads) {
            int row_b, kk, p, qq;
            if (a.pass == 0) {  // B[p][q]: row = output pixel p, K = target pixels q
                row_b = q / G8;
                kk = (q % G8) * 8;
                p = o0 + row_b;
                qq = k0 + kk;
            } else {  // B[q][p]: rows = output target pixels q, K = source pixels p (one per thread)
                kk = q % KB;
                row_b = (q / KB) * 8;
                p = k0 + kk;
                qq = o0 + row_b;
            }
            float gv[8];
            unpooled8(a, n, p, qq, gv);
            if (a.pass == 0) {
                if constexpr (kSplit) {
                    float hi[8], lo[8];
#pragma unroll
                    for (int i = 0; i < 8; i++) {
                        hi[i] = to_tf32(gv[i]);
                        lo[i] = to_tf32(gv[i] - hi[i]);
                    }
                    *reinterpret_cast<float4*>(sB + sw_off(row_b, kk, 4)) = make_float4(hi[0], hi[1], hi[2], hi[3]);
                    *reinterpret_cast<float4*>(sB + sw_off(row_b, kk + 4, 4)) = make_float4(hi[4], hi[5], hi[6], hi[7]);
                    *reinterpret_cast<float4*>(sBl + sw_off(row_b, kk, 4)) = make_float4(lo[0], lo[1], lo[2], lo[3]);
                    *reinterpret_cast<float4*>(sBl + sw_off(row_b, kk + 4, 4)) = make_float4(lo[4], lo[5], lo[6], lo[7]);
                } else {
                    alignas(16) OpT h[8];
#pragma unroll
                    for (int i = 0; i < 8; i++) h[i] = to_op<OpT>(gv[i]);
                    *reinterpret_cast<uint4*>(sB + sw_off(row_b, kk, EB)) = *reinterpret_cast<const uint4*>(h);
                }
            } else {
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    if constexpr (kSplit) {
                        const float hi = to_tf32(gv[i]);
                        *reinterpret_cast<float*>(sB + sw_off(row_b + i, kk, 4)) = hi;
                        *reinterpret_cast<float*>(sBl + sw_off(row_b + i, kk, 4)) = to_tf32(gv[i] - hi);
                    } else {
                        *reinterpret_cast<OpT*>(sB + sw_off(row_b + i, kk, EB)) = to_op<OpT>(gv[i]);
                    }
                }
            }
        }
        fence_proxy_async();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint64_t da = smem_desc_sw128(sA), db = smem_desc_sw128(sB), dl = smem_desc_sw128(sBl);
#pragma unroll
            for (int ks = 0; ks < 4; ks++) {  // 32 bytes of K per instruction
                const uint64_t o = (uint64_t)(ks * 2);
                const uint32_t acc = (kb | ks) ? 1u : 0u;
                if constexpr (kSplit) {
                    mma_tf32(tmem, da + o, db + o, idesc, acc);
                    mma_tf32(tmem, da + o, dl + o, idesc, 1u);
                } else {
                    mma_f16(tmem, da + o, db + o, idesc, acc);
                }
            }
            mma_commit(&bar[s]);
        }
        committed++;
    }
    if (!fail) {
        const int last = committed - 1;
        if (tid == 0 && !mbar_wait_bounded(&bar[last & 1], (uint32_t)(last >> 1) & 1u, kWaitNs)) fail = 1;
    }
    __syncthreads();
    tc_fence_after();
    if (!fail) {
        if (warp < 4) {
            const int r = 32 * warp + lane;  // accumulator row = channel
            float* orow = a.out + ((size_t)n * C + min(r, C - 1)) * HW + o0;
            for (int c0 = 0; c0 < kTile; c0 += 16) {
                float v[16];
                tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)c0, v);
                tmem_wait_ld();
                if (r < C) {
#pragma unroll
                    for (int j = 0; j < 16; j += 4)
                        *reinterpret_cast<float4*>(orow + c0 + j) =
                            make_float4(v[j] * 0.0625f, v[j + 1] * 0.0625f, v[j + 2] * 0.0625f, v[j + 3] * 0.0625f);
                }
            }
        }
    } else if (tid == 0) {
        atomicOr(a.err, 1);
        // the committed MMAs get one more bounded chance before their tensor memory is freed
        if (committed > 0) mbar_wait_bounded(&bar[(committed - 1) & 1], (uint32_t)((committed - 1) >> 1) & 1u, kWaitNs);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, kTile);
    }
}


// ---------------------------------------------------------------- TMA-fed kernel
//
// The production shapes (16-bit maps and level gradients of one type, W a multiple of 64,
// H and W multiples of 2^(levels-1)) take a warp-specialised persistent kernel whose
// operands arrive by TMA:
//   warp 12 lane 0  TMA: per 64-wide K block, the map tile (channels x 64 K, 128-byte
//                   swizzle), the G_0 tile (output pixels x 64 target pixels; pass 1 two
//                   64-pixel halves x 64 source rows, MN-major) and the G_l tiles that pool
//                   those target pixels (64 >> l cells per row, unswizzled) into a stage;
//   warps 0-7       combine: G_0 += level_sum in place, 16 bytes (8 target pixels of one
//                   image row) per step, rounded once to the operand type;
//   warp 13 lane 0  tcgen05.mma kind::f16, M = 128 channels, N = 128 output pixels, K = 16,
//                   into one of two tensor-memory accumulators (pass 1: B MN-major);
//   warps 8-11      epilogue: tcgen05.ld, x 1/16, FP32 stores; the accumulator is then free.
// Four stages of 46 KB; every G_0 element is read from HBM once per pass, the level tiles
// and the map rows come mostly from L2.

constexpr int kFStages = 4;
constexpr int kFCombineWarps = 8;
constexpr int kFEpiWarp0 = 8;
constexpr int kFTmaWarp = 12, kFMmaWarp = 13;
constexpr int kFThreads = 32 * 14;
constexpr uint32_t kFA = 16384;  // map tile: 128 rows x 128 B
constexpr uint32_t kFG = 16384;  // G_0 tile
// level-l tile bytes (l = 1..3): 128 rows (both halves in pass 1) x (128 >> l) B
__host__ __device__ constexpr uint32_t kFL(int l) { return l == 1 ? 8192u : l == 2 ? 4096u : l == 3 ? 2048u : 0u; }
constexpr uint32_t kFStage = kFA + kFG + 8192 + 4096 + 2048;

struct FastParams {
    float* out;
    int* err;
    int C, W, HW, L, blocks;
    long items;
};

__device__ __forceinline__ uint8_t* fstage(uint8_t* base, int s) { return base + (size_t)s * kFStage; }

template <typename OpT>
__device__ __forceinline__ float2 to_f2(uint32_t v) {
    if constexpr (std::is_same<OpT, __half>::value)
        return __half22float2(*reinterpret_cast<const __half2*>(&v));
    else
        return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&v));
}

template <typename OpT>
__device__ __forceinline__ uint32_t from_f2(float a, float b) {
    if constexpr (std::is_same<OpT, __half>::value) {
        const __half2 h = __floats2half2_rn(a, b);
        return *reinterpret_cast<const uint32_t*>(&h);
    } else {
        const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
        return *reinterpret_cast<const uint32_t*>(&h);
    }
}

// G_0 chunk (8 pixels, 4 pairs) += level_sum per pair, in place (the generic kernel's unpooled8)
template <typename OpT>
__device__ __forceinline__ void combine_chunk(uint4* cp, const uint8_t* l1p, const uint8_t* l2p, const uint8_t* l3p,
                                              int L) {
    uint4 raw = *cp;
    float l1[4], l2[4] = {0.f, 0.f, 0.f, 0.f}, l3 = 0.f;
    {
        const uint2 c1 = *reinterpret_cast<const uint2*>(l1p);
        const float2 a = to_f2<OpT>(c1.x), b = to_f2<OpT>(c1.y);
        l1[0] = a.x; l1[1] = a.y; l1[2] = b.x; l1[3] = b.y;
    }
    if (L > 2) {
        const float2 a = to_f2<OpT>(*reinterpret_cast<const uint32_t*>(l2p));
        l2[0] = l2[1] = a.x;
        l2[2] = l2[3] = a.y;
    }
    if (L > 3) l3 = to_f(*reinterpret_cast<const OpT*>(l3p));
    uint32_t* w = reinterpret_cast<uint32_t*>(&raw);
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const float sk = level_sum(l1[k], l2[k], l3, L);
        const float2 g = to_f2<OpT>(w[k]);
        w[k] = from_f2<OpT>(g.x + sk, g.y + sk);
    }
    *cp = raw;
}

template <typename OpT, int kPass>
__global__ void __launch_bounds__(kFThreads, 1)
    corr_vol_bwd_tma_kernel(const __grid_constant__ CUtensorMap mapF, const __grid_constant__ CUtensorMap mapG0,
                            const __grid_constant__ CUtensorMap mapG1, const __grid_constant__ CUtensorMap mapG2,
                            const __grid_constant__ CUtensorMap mapG3, FastParams a) {
    constexpr int FMT = std::is_same<OpT, __half>::value ? kFmtF16 : kFmtBF16;
    constexpr int R = kPass == 0 ? 128 : 64;  // G rows (K-major rows / MN-major K rows) per half
    extern __shared__ uint8_t sm_raw[];
    __shared__ uint64_t full[kFStages], ready[kFStages], empty[kFStages], accf[2], acce[2];
    __shared__ uint32_t tmem_base;
    __shared__ volatile int fail;
    uint8_t* sm = sm_raw + ((1024u - (smem_u32(sm_raw) & 1023u)) & 1023u);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int W = a.W, HW = a.HW, L = a.L;
    const int nk = HW / 64;
    if (tid == 0) {
        fail = 0;
        for (int s = 0; s < kFStages; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&ready[s], kFCombineWarps);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(&accf[b], 1);
            mbar_init(&acce[b], 4);
        }
        fence_barrier_init();
    }
    if (warp == kFMmaWarp) tmem_alloc(&tmem_base, 2 * kTile);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base;

    if (warp == kFTmaWarp && lane == 0) {
        // ------------------------------------------------ TMA producer
        const CUtensorMap* mg[4] = {&mapG0, &mapG1, &mapG2, &mapG3};
        uint32_t bytes = (uint32_t)min(a.C, kTile) * 128u + kFG;
        for (int l = 1; l < L; l++) bytes += kFL(l);
        uint32_t g = 0;
        for (long item = blockIdx.x; item < a.items && !fail; item += gridDim.x) {
            const int n = (int)(item / a.blocks), o0 = (int)(item % a.blocks) * kTile;
            for (int kb = 0; kb < nk; kb++, g++) {
                const int s = (int)(g % kFStages);
                if (g >= kFStages && !mbar_wait(&empty[s], ((g / kFStages) - 1) & 1, &fail)) break;
                uint8_t* st = fstage(sm, s);
                mbar_expect_tx(&full[s], bytes);
                tma_load_3d(st, &mapF, &full[s], kb * 64, 0, n);
                uint8_t* lv = st + kFA + kFG;
                if (kPass == 0) {
                    // rows o0.. (output pixels), K = target pixels kb*64 .. +63 (one image row)
                    const int q0 = kb * 64, y = q0 / W, x0 = q0 % W;
                    tma_load_2d(st + kFA, mg[0], &full[s], q0, n * HW + o0);
                    for (int l = 1; l < L; l++) {
                        tma_load_2d(lv, mg[l], &full[s], (y >> l) * (W >> l) + (x0 >> l), n * HW + o0);
                        lv += kFL(l);
                    }
                } else {
                    // K rows = source pixels kb*64 .., two 64-pixel halves of the output block
                    for (int h = 0; h < 2; h++) {
                        const int q0 = o0 + 64 * h, y = q0 / W, x0 = q0 % W;
                        tma_load_2d(st + kFA + h * 8192, mg[0], &full[s], q0, n * HW + kb * 64);
                        uint8_t* lh = lv;
                        for (int l = 1; l < L; l++) {
                            tma_load_2d(lh + h * (kFL(l) / 2), mg[l], &full[s], (y >> l) * (W >> l) + (x0 >> l),
                                        n * HW + kb * 64);
                            lh += kFL(l);
                        }
                    }
                }
            }
        }
        if (fail && g > 0) {
            // the loads already issued must land before the CTA exits (bounded)
            const uint64_t t0 = gtimer();
            for (uint32_t k = (g > kFStages ? g - kFStages : 0); k < g; k++)
                while (!mbar_try_wait(&full[k % kFStages], (k / kFStages) & 1) && gtimer() - t0 < kTmaWaitNs) {
                }
        }
    } else if (warp < kFCombineWarps) {
        // ------------------------------------------------ combine: G_0 += level_sum
        // thread tid owns 16-byte chunk j = tid & 7 of rows r0 + 32 m (pass 0) or of row
        // r0 + 32 (m & 1) in half m >> 1 (pass 1); the swizzle phase (r & 7) is fixed per thread
        const int j = tid & 7, r0 = tid >> 3;
        const uint32_t swz = (uint32_t)(((j ^ r0) & 7) << 4);
        uint32_t g = 0;
        for (long item = blockIdx.x; item < a.items && !fail; item += gridDim.x) {
            for (int kb = 0; kb < nk; kb++, g++) {
                const int s = (int)(g % kFStages);
                if (!mbar_wait(&full[s], (g / kFStages) & 1, &fail)) break;
                if (L > 1) {
                    uint8_t* st = fstage(sm, s);
                    const uint8_t* lv1 = st + kFA + kFG;
                    const uint8_t* lv2 = lv1 + kFL(1);
                    const uint8_t* lv3 = lv2 + kFL(2);
#pragma unroll
                    for (int m = 0; m < 4; m++) {
                        const int h = kPass == 0 ? 0 : (m >> 1);
                        const int r = kPass == 0 ? r0 + 32 * m : r0 + 32 * (m & 1);
                        const int hr = h * R + r;  // row in the level tiles
                        uint4* cp = reinterpret_cast<uint4*>(st + kFA + h * 8192 + r * 128 + swz);
                        combine_chunk<OpT>(cp, lv1 + hr * 64 + 8 * j, lv2 + hr * 32 + 4 * j, lv3 + hr * 16 + 2 * j, L);
                    }
                }
                fence_proxy_async();
                __syncwarp();
                if (lane == 0) mbar_arrive(&ready[s]);
            }
        }
    } else if (warp == kFMmaWarp && lane == 0) {
        // ------------------------------------------------ MMA issuer
        const uint32_t idesc = instr_desc(FMT, kTile, kTile) | (kPass == 1 ? (1u << 16) : 0u);
        uint32_t g = 0, t = 0;
        for (long item = blockIdx.x; item < a.items && !fail; item += gridDim.x, t++) {
            const int b = (int)(t & 1);
            if (t >= 2 && !mbar_wait(&acce[b], ((t >> 1) - 1) & 1, &fail)) break;
            tc_fence_after();
            const uint32_t d = tmem + (uint32_t)(b * kTile);
            bool ok = true;
            for (int kb = 0; kb < nk; kb++, g++) {
                const int s = (int)(g % kFStages);
                if (!mbar_wait(&ready[s], (g / kFStages) & 1, &fail)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                uint8_t* st = fstage(sm, s);
                const uint64_t da = smem_desc_sw128(st);
                const uint64_t db = kPass == 0 ? smem_desc_sw128(st + kFA) : smem_desc_sw128_mn(st + kFA, 8192);
                const uint64_t bstep = kPass == 0 ? 2u : (uint64_t)(2048 >> 4);
#pragma unroll
                for (int k = 0; k < 4; k++)
                    mma_f16(d, da + (uint64_t)(2 * k), db + (uint64_t)k * bstep, idesc, (kb | k) ? 1u : 0u);
                mma_commit(&empty[s]);
            }
            if (!ok) break;
            mma_commit(&accf[b]);
        }
        if (fail && g > 0) {
            // the committed MMAs get one more bounded chance before their tensor memory is freed
            const uint32_t k = g - 1;
            mbar_wait_bounded(&empty[k % kFStages], (k / kFStages) & 1, kTmaWaitNs);
        }
    } else if (warp >= kFEpiWarp0 && warp < kFEpiWarp0 + 4) {
        // ------------------------------------------------ epilogue
        const int q = warp & 3;  // tensor-memory lane quarter = channels 32q ..
        const int c = 32 * q + lane;
        uint32_t t = 0;
        for (long item = blockIdx.x; item < a.items && !fail; item += gridDim.x, t++) {
            const int b = (int)(t & 1);
            const int n = (int)(item / a.blocks), o0 = (int)(item % a.blocks) * kTile;
            if (!mbar_wait(&accf[b], (t >> 1) & 1, &fail)) break;
            tc_fence_after();
            float* orow = a.out + ((size_t)n * a.C + min(c, a.C - 1)) * HW + o0;
            for (int c0 = 0; c0 < kTile; c0 += 16) {
                float v[16];
                tmem_ld16(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(b * kTile + c0), v);
                tmem_wait_ld();
                if (c < a.C) {
#pragma unroll
                    for (int jj = 0; jj < 16; jj += 4)
                        *reinterpret_cast<float4*>(orow + c0 + jj) = make_float4(
                            v[jj] * 0.0625f, v[jj + 1] * 0.0625f, v[jj + 2] * 0.0625f, v[jj + 3] * 0.0625f);
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&acce[b]);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (fail && tid == 0) atomicOr(a.err, 1);
    if (warp == kFMmaWarp) {
        tc_fence_after();
        tmem_dealloc(tmem, 2 * kTile);
    }
}

}  // namespace cadj
}  // namespace vipe

using namespace vipe;
using namespace vipe::cadj;

template <typename OpT, typename FT, bool kSplit>
static int launch_vol_bwd(const Params& p, cudaStream_t st) {
    const size_t smem = (size_t)(kSplit ? 3 : 2) * 2 * kOpBytes + 1024;
    VIPE_CUDA_TRY(cudaFuncSetAttribute(corr_vol_bwd_kernel<OpT, FT, kSplit>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    corr_vol_bwd_kernel<OpT, FT, kSplit><<<(unsigned)(p.num * p.blocks), kThreads, smem, st>>>(p);
    VIPE_LAUNCH_CHECK();
    return VIPE_OK;
}

// (rows, cols) 16-bit matrix with row stride `cols`; box (box_cols, box_rows)
static int make_map_2d(CUtensorMap* map, const void* base, CUtensorMapDataType dt, uint64_t rows, uint64_t cols,
                       int box_cols, int box_rows, CUtensorMapSwizzle swz) {
    EncodeTiled enc = get_encode();
    if (!enc) return VIPE_ERR_CUDA;
    const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)cols * 2};
    const cuuint32_t box[2] = {(cuuint32_t)box_cols, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(map, dt, 2, const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, swz,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? VIPE_OK : VIPE_ERR_CUDA;
}

// a feature map (num, C, HW) as dim 0 pixels, dim 1 channels, dim 2 maps; box 64 pixels x C
static int make_fmap_map(CUtensorMap* map, const void* base, CUtensorMapDataType dt, int num, int C, int HW) {
    EncodeTiled enc = get_encode();
    if (!enc) return VIPE_ERR_CUDA;
    const cuuint64_t dims[3] = {(cuuint64_t)HW, (cuuint64_t)C, (cuuint64_t)num};
    const cuuint64_t strides[2] = {(cuuint64_t)HW * 2, (cuuint64_t)C * HW * 2};
    const cuuint32_t box[3] = {64u, (cuuint32_t)C, 1u};
    const cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = enc(map, dt, 3, const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? VIPE_OK : VIPE_ERR_CUDA;
}

static int g_sms = 0;

// one pass of the TMA-fed kernel; returns VIPE_ERR_CUDA when a tensor map does not encode
template <typename OpT>
static int launch_fast(const Params& p, int pass, const void* fmap, float* out, cudaStream_t st) {
    const CUtensorMapDataType dt =
        std::is_same<OpT, __half>::value ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
    const int R = pass == 0 ? 128 : 64;
    const uint64_t rows = (uint64_t)p.num * p.HW;
    CUtensorMap mf, mg[4];
    int rc = make_fmap_map(&mf, fmap, dt, p.num, p.C, p.HW);
    if (rc == VIPE_OK) rc = make_map_2d(&mg[0], p.g[0], dt, rows, (uint64_t)p.HW, 64, R, CU_TENSOR_MAP_SWIZZLE_128B);
    for (int l = 1; l < 4 && rc == VIPE_OK; l++) {
        // levels past num_levels get a valid map of level 0 that the kernel never reads
        if (l < p.L)
            rc = make_map_2d(&mg[l], p.g[l], dt, rows, (uint64_t)(p.HW >> (2 * l)), 64 >> l, R,
                             CU_TENSOR_MAP_SWIZZLE_NONE);
        else
            mg[l] = mg[0];
    }
    if (rc != VIPE_OK) return rc;
    if (g_sms == 0) {
        int dev = 0;
        VIPE_CUDA_TRY(cudaGetDevice(&dev));
        VIPE_CUDA_TRY(cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev));
    }
    FastParams fp{};
    fp.out = out;
    fp.err = p.err;
    fp.C = p.C; fp.W = p.W; fp.HW = p.HW; fp.L = p.L; fp.blocks = p.blocks;
    fp.items = (long)p.num * p.blocks;
    const size_t smem = (size_t)kFStages * kFStage + 1024;
    auto kern = pass == 0 ? corr_vol_bwd_tma_kernel<OpT, 0> : corr_vol_bwd_tma_kernel<OpT, 1>;
    VIPE_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const long grid = std::min<long>(fp.items, (long)g_sms);
    kern<<<(unsigned)grid, kFThreads, smem, st>>>(mf, mg[0], mg[1], mg[2], mg[3], fp);
    VIPE_LAUNCH_CHECK();
    return VIPE_OK;
}

template <typename FT>
static int launch_pass(const Params& p, bool split, cudaStream_t st) {
    if (split) return launch_vol_bwd<float, FT, true>(p, st);
    return launch_vol_bwd<FT, FT, false>(p, st);
}

static int g_force_generic = 0;

// 1: every shape takes the generic (producer-formed) kernel; used by tests to hold the two
// kernels to each other
extern "C" void vipe_corr_volume_backward_force_generic(int on) { g_force_generic = on ? 1 : 0; }

extern "C" int vipe_corr_volume_backward(int map_dtype, int grad_dtype, const void* fmap1, const void* fmap2,
                                         const void* const* level_grads, int num, int C, int H, int W,
                                         int num_levels, float* fmap1_grad_out, float* fmap2_grad_out,
                                         int32_t* dev_status, void* stream) {
    if (map_dtype != VIPE_F16 && map_dtype != VIPE_BF16) return VIPE_ERR_DTYPE;
    if (grad_dtype != VIPE_F16 && grad_dtype != VIPE_BF16 && grad_dtype != VIPE_F32) return VIPE_ERR_DTYPE;
    if (num <= 0 || C <= 0 || C > kTile || H <= 0 || W <= 0 || num_levels < 1 || num_levels > kMaxLevels)
        return VIPE_ERR_ARG;
    const int HW = H * W, span = 1 << (num_levels - 1);
    if (HW % kTile != 0 || W % 8 != 0 || H % span != 0 || W % span != 0) {
        set_last_error("corr volume backward: H*W a multiple of 128, W of 8, H and W of 2^(levels-1)");
        return VIPE_ERR_ARG;
    }
    if (!fmap1 || !fmap2 || !level_grads || !dev_status) return VIPE_ERR_ARG;
    Params p{};
    for (int l = 0; l < num_levels; l++) {
        if (!level_grads[l]) return VIPE_ERR_ARG;
        p.g[l] = level_grads[l];
    }
    p.err = dev_status;
    p.num = num; p.C = C; p.H = H; p.W = W; p.HW = HW; p.L = num_levels; p.gdt = grad_dtype;
    p.blocks = HW / kTile;
    const bool split = grad_dtype == VIPE_F32;
    cudaStream_t st = as_stream(stream);
    VIPE_PROF("corr_volume_bwd", st);
    // TMA-fed kernel: 16-bit operands of one type, 64-pixel K blocks inside one image row, and
    // every level's row stride a multiple of 16 bytes
    const bool fast = grad_dtype == map_dtype && W % 64 == 0 && (HW >> (2 * (num_levels - 1))) % 8 == 0 &&
                      g_force_generic == 0;
    if (fast) {
        for (int pass = 0; pass < 2; pass++) {
            float* out = pass == 0 ? fmap1_grad_out : fmap2_grad_out;
            if (!out) continue;
            const void* fm = pass == 0 ? fmap2 : fmap1;
            const int rc = map_dtype == VIPE_F16 ? launch_fast<__half>(p, pass, fm, out, st)
                                                 : launch_fast<__nv_bfloat16>(p, pass, fm, out, st);
            if (rc != VIPE_OK) return rc;
        }
        return VIPE_OK;
    }
    for (int pass = 0; pass < 2; pass++) {
        float* out = pass == 0 ? fmap1_grad_out : fmap2_grad_out;
        if (!out) continue;
        p.pass = pass;
        p.out = out;
        p.fa = pass == 0 ? fmap2 : fmap1;
        const int rc = map_dtype == VIPE_F16 ? launch_pass<__half>(p, split, st) : launch_pass<__nv_bfloat16>(p, split, st);
        if (rc != VIPE_OK) return rc;
    }
    return VIPE_OK;
}
