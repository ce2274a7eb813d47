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
#include "tcgen05.cuh"

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <type_traits>

namespace vipe {
namespace cadj {

using namespace ::vipe::tc;

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

// Gt[p][q .. q+7] (8 consecutive target pixels in one image row): level 0 as one row chunk,
// level l as the 8 >> l pooled values that cover them, each / 4^l
__device__ __forceinline__ void unpooled8(const Params& a, int n, int p, int q, float* o) {
    const int W = a.W, y = q / W, x = q % W;
    const size_t HW = (size_t)a.HW;
#pragma unroll
    for (int i = 0; i < 8; i++) o[i] = 0.f;
    for (int l = 0; l < a.L; l++) {
        const int Wl = W >> l, HWl = (int)(HW >> (2 * l));
        const size_t row = ((size_t)n * HW + p) * HWl + (size_t)(y >> l) * Wl;
        const float s = 1.f / (float)(1 << (2 * l));
        if (l == 0 && a.gdt == VIPE_F32) {
            const float4* src = reinterpret_cast<const float4*>(static_cast<const float*>(a.g[0]) + row + x);
            const float4 u = src[0], v = src[1];
            o[0] += u.x; o[1] += u.y; o[2] += u.z; o[3] += u.w;
            o[4] += v.x; o[5] += v.y; o[6] += v.z; o[7] += v.w;
        } else if (l == 0) {
            const uint4 raw = *reinterpret_cast<const uint4*>(static_cast<const uint16_t*>(a.g[0]) + row + x);
            const uint16_t* h = reinterpret_cast<const uint16_t*>(&raw);
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const uint16_t b = h[i];
                o[i] += a.gdt == VIPE_F16 ? __half2float(__ushort_as_half(b)) : __bfloat162float(__ushort_as_bfloat16(b));
            }
        } else {
            const int span = 1 << l;
            for (int i = 0; i < 8; i += span) {
                const float v = ld_any(a.g[l], row + ((x + i) >> l), a.gdt) * s;
                for (int u = 0; u < span; u++) o[i + u] += v;
            }
        }
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

template <typename FT>
static int launch_pass(const Params& p, bool split, cudaStream_t st) {
    if (split) return launch_vol_bwd<float, FT, true>(p, st);
    return launch_vol_bwd<FT, FT, false>(p, st);
}

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
