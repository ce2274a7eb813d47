// All-pairs correlation volume + average-pooled pyramid on tcgen05 tensor cores.
//
// Replaces CorrBlock.corr and its pyramid (vipe/slam/networks/droid_net.py:56-69,
// 94-102): for every edge e, V_e = (F1_e / 4)^T (F2_e / 4) over C channels
// (source pixel x target pixel), and level l = avg_pool2d^l(V_e) over the target
// axes (2x2 windows, floor sizes).
//
// Data path (one persistent launch, one CTA per SM):
//   * pack pass: F1, F2 (num, C, H, W) -> K-major BF16/FP16 rows (num, H*W, Kp)
//     scaled by 1/4 (exact), F2's pixels reordered so that 256 consecutive rows
//     are a th x TW block of the target image (8 x 32/16/8, or 4 x 64 for the
//     full-row tiles of 64-wide maps); with 16-bit 64-wide maps only F2 is
//     packed and the A operand is read from F1 itself (MN-major, below);
//   * warp 8 lane 0: TMA loads (SWIZZLE_128B, 64-channel boxes) of the A tile
//     (128 source pixels x Kp, reused for all N tiles of the work item) and of
//     the B tiles (one stage, filled and drained per 64-channel box);
//   * warp 9 lane 0: tcgen05.mma.cta_group::1.kind::f16, M = 128, N = th*TW,
//     K = 16 per instruction, FP32 accumulator in tensor memory, two TMEM
//     accumulator buffers (2 x 256 columns) so the MMA of tile t+1 overlaps the
//     epilogue of tile t;
//   * warps 0-7: epilogue.  tcgen05.ld puts one source pixel's accumulator row
//     in each thread's registers, so the 2x2 / 4x4 average pools close inside
//     the thread; the levels are staged per warp in shared memory and written
//     with 16-byte stores in which consecutive lanes cover contiguous bytes.
//     16-bit output on 64-wide maps (the production shape) uses full-row tiles
//     (4 target rows x 64 columns): each warp owns a column half of all 4 rows,
//     stages levels 0-2 in swizzled boxes and writes them with TMA tensor
//     stores, and pools level 3 from the level-2 rows of two consecutive tiles
//     (the even tile's row carried in registers).  Other 16-bit shapes with
//     32-wide target blocks use
//     the row-split mapping (kR0 below: each warp owns 4 of 8 target rows,
//     16-byte st.global from staging; level 3 pooled afterwards from the stored
//     level 2 by pool_level_kernel); the rest split the tile's columns
//     between warp halves and pool all levels in the epilogue.
// The output write (sum over levels of num*HW*HW/4^l elements) is the HBM
// roofline of this kernel: it is write-only traffic.

// Every mbarrier wait is bounded: on expiry the CTA records an error, stops
// issuing work, drains its in-flight copies (bounded) and frees tensor memory.

#include "common.cuh"
#include "tcgen05.cuh"
#include "tma.cuh"

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <mutex>

namespace vipe {
namespace cbuild {

constexpr int kBM = 128;       // source pixels per tile (TMEM lanes)
constexpr int kTH = 8;         // target rows per N tile
constexpr int kKC = 64;        // channels per TMA box / swizzle row (128 B of 16-bit)
constexpr int kMaxKC = 2;      // up to 128 channels (A + two B stages fit in shared memory)
constexpr int kThreads = 320;  // 8 epilogue warps, 1 TMA warp, 1 MMA warp
constexpr int kEpiWarps = 8;
constexpr int kTmaWarp = 8, kMmaWarp = 9;
constexpr uint64_t kWaitNs = tc::kTmaWaitNs;  // 2 s bound on any mbarrier wait
constexpr int kTmaStage = 12288;  // per-warp staging of the TMA-store epilogue (1024-B aligned; <= Stage::per_warp)

struct Params {
    int num, C, Kp, H, W, HW, TW, N, levels;
    int mtiles, ntiles;
    long items;  // num * mtiles
    int out_dtype;
    void* out[4];
    int* err;
    int rowsplit;  // 1: the row-split epilogue (16-bit output, TW = 32); level 3 by pool_level_kernel
    int tma_store;  // 1: full-row tiles (4 target rows x 64 columns, W = 64) stored by TMA (levels 0-2)
    int th;         // target rows per N tile: 8, or 4 for full-row tiles
    int direct;     // 1: the A operand (source pixels) is loaded by TMA straight from the 16-bit fmap1 (MN-major)
                    // and the product scaled by 1/4 in the epilogue; only fmap2 is packed (full-row tiles only)
};

// ---------------------------------------------------------------- PTX helpers

using namespace ::vipe::tc;

// TMA tensor store of a staged box (3-D map: target columns, source pixels, target
// rows); completion is tracked per thread with bulk groups.  The volume is written once and
// never re-read by this kernel: its lines carry the L2 evict-first policy, so the write stream
// leaves L2 in the order it arrives and the re-read B tiles stay resident (640 edges: 3.95 ->
// 3.73 ms per build, the minimum of alternating runs)
__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, const void* src, int x, int y, int z) {
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    asm volatile(
        "cp.async.bulk.tensor.3d.global.shared::cta.bulk_group.L2::cache_hint [%0, {%2, %3, %4}], [%1], %5;" ::"l"(
            reinterpret_cast<uint64_t>(map)),
        "r"(smem_u32(src)), "r"(x), "r"(y), "r"(z), "l"(pol)
        : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// the staged boxes of every committed store have been read (the buffer may be rewritten)
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// every committed store has completed
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// ---------------------------------------------------------------- output stores

template <typename T>
__device__ __forceinline__ T cvt(float v);
template <>
__device__ __forceinline__ float cvt<float>(float v) { return v; }
template <>
__device__ __forceinline__ __half cvt<__half>(float v) { return __float2half_rn(v); }
template <>
__device__ __forceinline__ __nv_bfloat16 cvt<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }

// Epilogue staging.  Eight epilogue warps: warp w owns TMEM lane quarter
// w % 4 (32 source rows) and half w / 4 of the tile's TW target columns, taken
// in passes of PW columns (16 for 16-bit output, 8 for FP32).  A pass stages,
// per source row: level 0 8 x PW, level 1 4 x PW/2, level 2 2 x PW/4, level 3
// 1 x PW/8 elements; row strides are 16 (mod 128) bytes or odd multiples of 16,
// so each quarter-warp's accesses hit distinct bank groups.  The staged pass is
// then written with 16-byte (level 0/1), 8-byte and 4-byte stores in which
// consecutive lanes cover consecutive bytes of one output row segment.
template <typename T>
struct Stage {
    static constexpr int sz = (int)sizeof(T);
    static constexpr int PW = sz == 4 ? 8 : 16;
    static constexpr int r0 = 8 * PW * sz + 16;         // level 0 row stride (bytes)
    static constexpr int r1 = 4 * (PW / 2) * sz + 16;   // level 1
    static constexpr int r2 = 2 * (PW / 4) * sz + 16;   // level 2
    static constexpr int r3 = 16;                       // level 3
    static constexpr int per_warp = 32 * (r0 + r1 + r2 + r3);
};

// Row-split epilogue (16-bit output, TW = 32): warp (q, rh) owns TMEM lane
// quarter q and target rows 4 rh .. 4 rh + 3 of the 8 x 32 tile, all 32 columns.
// Per source row it stages level 0 as 4 rows of 64 B, level 1 as 2 rows of 32 B
// and level 2 as one 16-byte row, so each level-0 store instruction covers 8
// segments of 64 contiguous bytes, level-1 rows leave as whole 32-byte sectors
// and a level-2 row's two 16-byte halves come from consecutive tiles of the same
// warp.  Level 3 (2x2 of level 2) is pooled afterwards from the stored level 2.
constexpr int kR0 = 4 * 64 + 16, kR1 = 2 * 32 + 16, kR2 = 16 + 16;  // staged row strides (bytes)
static_assert(32 * (kR0 + kR1 + kR2) <= 12800, "row-split staging exceeds the per-warp staging region");

__device__ __forceinline__ float to_float(__half v) { return __half2float(v); }
__device__ __forceinline__ float to_float(__nv_bfloat16 v) { return __bfloat162float(v); }
__device__ __forceinline__ float to_float(float v) { return v; }

template <typename T>
__device__ __forceinline__ uint32_t pack2(float a, float b);
template <>
__device__ __forceinline__ uint32_t pack2<__half>(float a, float b) {
    const __half2 h = __floats2half2_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
}
template <>
__device__ __forceinline__ uint32_t pack2<__nv_bfloat16>(float a, float b) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
}

// store n (= 8, 4, 2 or 1) values of type T at dst with the widest aligned access
template <typename T, int n>
__device__ __forceinline__ void sts_n(uint8_t* dst, const float* v) {
    if constexpr (sizeof(T) == 4) {
        if constexpr (n == 8) {
            reinterpret_cast<float4*>(dst)[0] = make_float4(v[0], v[1], v[2], v[3]);
            reinterpret_cast<float4*>(dst)[1] = make_float4(v[4], v[5], v[6], v[7]);
        } else if constexpr (n == 4) {
            *reinterpret_cast<float4*>(dst) = make_float4(v[0], v[1], v[2], v[3]);
        } else if constexpr (n == 2) {
            *reinterpret_cast<float2*>(dst) = make_float2(v[0], v[1]);
        } else {
            *reinterpret_cast<float*>(dst) = v[0];
        }
    } else {
        if constexpr (n == 8) {
            *reinterpret_cast<uint4*>(dst) =
                make_uint4(pack2<T>(v[0], v[1]), pack2<T>(v[2], v[3]), pack2<T>(v[4], v[5]), pack2<T>(v[6], v[7]));
        } else if constexpr (n == 4) {
            *reinterpret_cast<uint2*>(dst) = make_uint2(pack2<T>(v[0], v[1]), pack2<T>(v[2], v[3]));
        } else if constexpr (n == 2) {
            *reinterpret_cast<uint32_t*>(dst) = pack2<T>(v[0], v[1]);
        } else {
            *reinterpret_cast<T*>(dst) = cvt<T>(v[0]);
        }
    }
}

// pools one 8x8 block and stages all levels at column block cb of the pass
template <typename T>
__device__ __forceinline__ void stage_block(uint8_t* st, int lane, int cb, const float (&blk)[8][8]) {
    using S = Stage<T>;
    uint8_t* s0 = st + lane * S::r0;
    uint8_t* s1 = st + 32 * S::r0 + lane * S::r1;
    uint8_t* s2 = st + 32 * (S::r0 + S::r1) + lane * S::r2;
    uint8_t* s3 = st + 32 * (S::r0 + S::r1 + S::r2) + lane * S::r3;
#pragma unroll
    for (int r = 0; r < 8; r++) sts_n<T, 8>(s0 + (r * S::PW + cb * 8) * S::sz, blk[r]);
    float l1[4][4];
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
        for (int c = 0; c < 4; c++)
            l1[r][c] = 0.25f * ((blk[2 * r][2 * c] + blk[2 * r][2 * c + 1]) + (blk[2 * r + 1][2 * c] + blk[2 * r + 1][2 * c + 1]));
#pragma unroll
    for (int r = 0; r < 4; r++) sts_n<T, 4>(s1 + (r * (S::PW / 2) + cb * 4) * S::sz, l1[r]);
    float l2[2][2];
#pragma unroll
    for (int r = 0; r < 2; r++)
#pragma unroll
        for (int c = 0; c < 2; c++)
            l2[r][c] = 0.25f * ((l1[2 * r][2 * c] + l1[2 * r][2 * c + 1]) + (l1[2 * r + 1][2 * c] + l1[2 * r + 1][2 * c + 1]));
#pragma unroll
    for (int r = 0; r < 2; r++) sts_n<T, 2>(s2 + (r * (S::PW / 4) + cb * 2) * S::sz, l2[r]);
    const float l3 = 0.25f * ((l2[0][0] + l2[0][1]) + (l2[1][0] + l2[1][1]));
    sts_n<T, 1>(s3 + cb * S::sz, &l3);
}

// writes one staged level: per row NSEG segments of SEG bytes (SSTR apart in
// shared memory), copied in CHUNK-byte pieces; lanes walk chunks of one row
// segment consecutively
template <int NSEG, int SEG, int SSTR, int CHUNK>
__device__ __forceinline__ void flush_fixed(const uint8_t* st, int rstride, int nrows, uint8_t* gbase,
                                            uint32_t grow_stride, uint32_t gseg_stride, int lane) {
    constexpr int CPS = SEG / CHUNK;         // chunks per segment
    constexpr int CPR = NSEG * CPS;          // chunks per row
    constexpr int TOTAL = 32 * CPR;
#pragma unroll 4
    for (int j = lane; j < TOTAL; j += 32) {
        const int i = j / CPR;               // compile-time power-of-two divisors
        const int sg = (j / CPS) % NSEG;
        const int k = j % CPS;
        if (i >= nrows) continue;
        const uint8_t* src = st + i * rstride + sg * SSTR + k * CHUNK;
        uint8_t* dst = gbase + (size_t)i * grow_stride + (size_t)sg * gseg_stride + k * CHUNK;
        if constexpr (CHUNK == 16)
            *reinterpret_cast<uint4*>(dst) = *reinterpret_cast<const uint4*>(src);
        else if constexpr (CHUNK == 8)
            *reinterpret_cast<uint2*>(dst) = *reinterpret_cast<const uint2*>(src);
        else if constexpr (CHUNK == 4)
            *reinterpret_cast<uint32_t*>(dst) = *reinterpret_cast<const uint32_t*>(src);
        else
            *reinterpret_cast<uint16_t*>(dst) = *reinterpret_cast<const uint16_t*>(src);
    }
}

// flush a full pass (PW columns) or a half pass (8 columns, only when TW = 8 and PW = 16)
template <typename T, int COLS>
__device__ __forceinline__ void flush_pass(const uint8_t* st, int nrows, uint8_t* const* lvl, const uint32_t* rs,
                                           const uint32_t* ss, int levels, int lane) {
    using S = Stage<T>;
    constexpr int sz = S::sz;
    constexpr int s0 = COLS * sz, s1 = (COLS / 2) * sz, s2 = (COLS / 4) * sz, s3 = (COLS / 8) * sz;
    flush_fixed<8, s0, S::PW * sz, (s0 >= 16 ? 16 : s0)>(st, S::r0, nrows, lvl[0], rs[0], ss[0], lane);
    if (levels > 1)
        flush_fixed<4, s1, (S::PW / 2) * sz, (s1 >= 16 ? 16 : s1)>(st + 32 * S::r0, S::r1, nrows, lvl[1], rs[1], ss[1],
                                                                   lane);
    if (levels > 2)
        flush_fixed<2, s2, (S::PW / 4) * sz, (s2 >= 16 ? 16 : s2)>(st + 32 * (S::r0 + S::r1), S::r2, nrows, lvl[2],
                                                                   rs[2], ss[2], lane);
    if (levels > 3)
        flush_fixed<1, s3, (S::PW / 8) * sz, (s3 >= 16 ? 16 : s3)>(st + 32 * (S::r0 + S::r1 + S::r2), S::r3, nrows,
                                                                   lvl[3], rs[3], ss[3], lane);
}

// ---------------------------------------------------------------- main kernel

// dynamic shared memory: A tile (KC boxes of 128 rows x 128 B) then two B
// stages (KC boxes of N rows x 128 B each); every box starts 1024-B aligned
__host__ __device__ inline size_t a_region(int KC) { return (size_t)KC * kBM * 128; }
__host__ __device__ inline size_t b_box(int N) { return (size_t)N * 128; }

template <typename TOut>
__global__ void __launch_bounds__(kThreads, 1)
    corr_build_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                      const __grid_constant__ CUtensorMap mapO0, const __grid_constant__ CUtensorMap mapO1,
                      const __grid_constant__ CUtensorMap mapO2, Params p, int ab_format) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* sbase = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    __shared__ uint64_t barA_full, barA_empty;
    __shared__ uint64_t barB_full[2], barB_empty[2];
    __shared__ uint64_t barAcc_full[2], barAcc_empty[2];
    __shared__ uint32_t tmem_base;
    __shared__ volatile int fail;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int KC = p.Kp / kKC;
    const int N = p.N;
    auto sa = [&](int kc) { return sbase + (size_t)kc * kBM * 128; };
    auto sb = [&](int st, int kc) { return sbase + a_region(KC) + ((size_t)st * KC + kc) * b_box(N); };
    // One B stage, filled and drained per 64-channel box: box kc of tile t+1 loads as soon as
    // the MMAs of box kc of tile t have read it, so loads overlap the other box's MMAs; the
    // MMA of tile t+1 overlaps the epilogue of tile t through the two TMEM accumulators.
    const int NBS = 1;
    const size_t stage_off = a_region(KC) + (size_t)NBS * KC * b_box(N);

    if (tid == 0) {
        fail = 0;
        mbar_init(&barA_full, 1);
        mbar_init(&barA_empty, 1);
        for (int s = 0; s < 2; s++) {
            mbar_init(&barB_full[s], 1);
            mbar_init(&barB_empty[s], 1);
            mbar_init(&barAcc_full[s], 1);
            mbar_init(&barAcc_empty[s], kEpiWarps);  // one arrive per epilogue warp
        }
        fence_barrier_init();
    }
    if (warp == kMmaWarp) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(&tmem_base)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base;

    const uint32_t a_bytes = (uint32_t)kBM * 128u * KC;
    const uint32_t box_bytes = (uint32_t)N * 128u;  // one 64-channel box of a B tile

    if (warp == kTmaWarp && lane == 0) {
        // ------------------------------------------------ TMA producer
        uint32_t t = 0, it = 0;
        uint32_t issued[kMaxKC] = {0, 0};  // B box loads issued per box slot
        for (long item = blockIdx.x; item < p.items && !fail; item += gridDim.x, it++) {
            const int e = (int)(item / p.mtiles), mt = (int)(item % p.mtiles);
            if (it > 0 && !mbar_wait(&barA_empty, (it - 1) & 1, &fail)) break;
            mbar_expect_tx(&barA_full, a_bytes);
            for (int kc = 0; kc < KC; kc++) {
                if (p.direct) {
                    // two 64-pixel MN atoms of 64 channels each from fmap1 (pixels past H*W read zeros)
                    for (int h = 0; h < kBM / 64; h++)
                        tma_load_3d(sa(kc) + h * 8192, &mapA, &barA_full, mt * kBM + 64 * h, kc * kKC, e);
                } else {
                    tma_load_2d(sa(kc), &mapA, &barA_full, kc * kKC, e * p.HW + mt * kBM);
                }
            }
            for (int nt = 0; nt < p.ntiles && !fail; nt++, t++) {
                // box kc of this tile (barB_full/empty[kc]: one phase per tile)
                for (int kc = 0; kc < KC; kc++) {
                    if (t >= 1 && !mbar_wait(&barB_empty[kc], (t - 1) & 1, &fail)) break;
                    mbar_expect_tx(&barB_full[kc], box_bytes);
                    tma_load_2d(sb(0, kc), &mapB, &barB_full[kc], kc * kKC, e * p.HW + nt * N);
                    issued[kc]++;
                }
            }
        }
        // drain: the last loads issued must land before the CTA exits (bounded; returns at
        // once for a box whose last load already completed)
        if (fail) {
            const uint64_t t0 = gtimer();
            for (int kc = 0; kc < KC; kc++)
                if (issued[kc] > 0)
                    while (!mbar_try_wait(&barB_full[kc], (issued[kc] - 1) & 1) && gtimer() - t0 < kWaitNs) {
                    }
        }
    } else if (warp == kMmaWarp && lane == 0) {
        // ------------------------------------------------ MMA issuer
        // MN-major A (direct loads): transpose bit 15 of the instruction descriptor
        const uint32_t idesc = instr_desc(ab_format, kBM, N) | (p.direct ? (1u << 15) : 0u);
        uint32_t t = 0, it = 0;
        for (long item = blockIdx.x; item < p.items && !fail; item += gridDim.x, it++) {
            if (!mbar_wait(&barA_full, it & 1, &fail)) break;
            tc_fence_after();
            for (int nt = 0; nt < p.ntiles && !fail; nt++, t++) {
                const int acc = t & 1;
                if (t >= 2 && !mbar_wait(&barAcc_empty[acc], ((t >> 1) - 1) & 1, &fail)) break;
                const uint32_t d = tmem + (uint32_t)(acc * 256);
                bool ok = true;
                for (int kc = 0; kc < KC; kc++) {
                    if (!mbar_wait(&barB_full[kc], t & 1, &fail)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint64_t da = p.direct ? smem_desc_sw128_mn(sa(kc), 8192) : smem_desc_sw128(sa(kc));
                    const uint64_t db = smem_desc_sw128(sb(0, kc));
                    // K step of 16 channels: 32 bytes inside the swizzled row (K-major) or 16 rows of
                    // 128 bytes (MN-major A)
                    const uint64_t astep = p.direct ? (uint64_t)(2048 >> 4) : 2u;
#pragma unroll
                    for (int k = 0; k < kKC / 16; k++)
                        mma_f16(d, da + (uint64_t)k * astep, db + (uint64_t)(k * 2), idesc, (kc | k) ? 1u : 0u);
                    mma_commit(&barB_empty[kc]);  // box kc of this tile is read once these MMAs complete
                }
                if (!ok) break;
                mma_commit(&barAcc_full[acc]);
            }
            mma_commit(&barA_empty);
        }
    } else if (warp < kEpiWarps) {
        // ------------------------------------------------ epilogue
        using St = Stage<TOut>;
        constexpr int PW = St::PW;
        const int q = warp & 3, half = warp >> 2;   // TMEM lane quarter, column half
        const uint32_t lane_addr = (uint32_t)(q * 32) << 16;
        const int TW = p.TW, blocks_w = p.W / TW;
        const int col_lo = TW >= 16 ? half * (TW / 2) : 0;
        const int col_hi = TW >= 16 ? col_lo + TW / 2 : (half == 0 ? TW : 0);
        uint8_t* st = sbase + stage_off + (size_t)warp * St::per_warp;
        constexpr int sz = (int)sizeof(TOut);
        const int H = p.H, W = p.W;
        uint32_t rs[4], ss[4];
        for (int l = 0; l < 4; l++) {
            rs[l] = (uint32_t)((H >> l) * (W >> l) * sz);  // one source row of level l
            ss[l] = (uint32_t)((W >> l) * sz);             // one target row of level l
        }
        uint32_t t = 0;
        uint4 l2_carry = make_uint4(0, 0, 0, 0);  // full-row tiles: the previous tile's staged level-2 row
        for (long item = blockIdx.x; item < p.items && !fail; item += gridDim.x) {
            const int e = (int)(item / p.mtiles), mt = (int)(item % p.mtiles);
            const int m0 = mt * kBM + q * 32;               // first source row of this warp
            const int nrows = max(0, min(32, p.HW - m0));
            const long row0 = (long)e * p.HW + m0;
            for (int nt = 0; nt < p.ntiles; nt++, t++) {
                const int acc = t & 1;
                if (!mbar_wait(&barAcc_full[acc], (t >> 1) & 1, &fail)) break;
                tc_fence_after();
                const int hb = nt / blocks_w, wb = nt % blocks_w;
                if (col_lo >= col_hi) {
                    tc_fence_before();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&barAcc_empty[acc]);
                    continue;
                }
                if constexpr (sizeof(TOut) == 2) {
                    if (p.tma_store) {
                        // Full-row tiles (4 target rows x 64 columns): warp (q, ch) owns TMEM lane
                        // quarter q and column half ch, so the two halves of every 128-byte level-0
                        // row leave in the same tile.  Levels 0-2 are staged as the boxes of three
                        // TMA tensor stores (source pixel = lane): level 0 [4 rows][32 px][64 B] with
                        // the 64-byte swizzle (16-byte chunk c of a 64-byte row at c ^ ((px >> 1) & 3)),
                        // level 1 [2][32][32 B] with the 32-byte swizzle (chunk c at
                        // c ^ ((px >> 2) & 1)), level 2 [32][16 B]; the swizzles keep each
                        // quarter-warp's 16-byte stores on distinct bank groups.
                        const int ch = warp >> 2;
                        uint8_t* t0s = sbase + stage_off + (size_t)warp * kTmaStage;
                        uint8_t* t1s = t0s + 8192;
                        uint8_t* t2s = t0s + 10240;
                        if (lane == 0) bulk_wait_read_all();  // the previous tile's boxes have been read
                        __syncwarp();
#pragma unroll 1
                        for (int cb = 0; cb < 4; cb++) {
                            float blk[4][8];
#pragma unroll
                            for (int r = 0; r < 4; r++)
                                tmem_ld8(tmem + lane_addr + (uint32_t)(acc * 256 + r * 64 + ch * 32 + cb * 8), blk[r]);
                            tmem_wait_ld();
                            if (p.direct) {  // fmap1's 1/4 scale (fmap2's is in its pack), applied here (exact)
#pragma unroll
                                for (int r = 0; r < 4; r++)
#pragma unroll
                                    for (int j = 0; j < 8; j++) blk[r][j] *= 0.25f;
                            }
#pragma unroll
                            for (int r = 0; r < 4; r++)
                                sts_n<TOut, 8>(t0s + (r * 32 + lane) * 64 + ((cb ^ ((lane >> 1) & 3)) << 4), blk[r]);
                            float l1[2][4];
#pragma unroll
                            for (int r = 0; r < 2; r++)
#pragma unroll
                                for (int c2 = 0; c2 < 4; c2++)
                                    l1[r][c2] = 0.25f * ((blk[2 * r][2 * c2] + blk[2 * r][2 * c2 + 1]) +
                                                         (blk[2 * r + 1][2 * c2] + blk[2 * r + 1][2 * c2 + 1]));
#pragma unroll
                            for (int r = 0; r < 2; r++)
                                sts_n<TOut, 4>(t1s + (r * 32 + lane) * 32 + (((cb >> 1) ^ ((lane >> 2) & 1)) << 4) +
                                                   (cb & 1) * 8,
                                               l1[r]);
                            float l2[2];
#pragma unroll
                            for (int c2 = 0; c2 < 2; c2++)
                                l2[c2] = 0.25f * ((l1[0][2 * c2] + l1[0][2 * c2 + 1]) + (l1[1][2 * c2] + l1[1][2 * c2 + 1]));
                            sts_n<TOut, 2>(t2s + lane * 16 + cb * 4, l2);
                        }
                        if (p.levels > 3) {
                            // level 3 row hb / 2 pools the level-2 rows of tiles hb - 1 and hb (consecutive
                            // tiles of this warp): even tiles keep their staged row in registers, odd tiles
                            // write 4 values of this lane's column half (the stored FP16 level 2, FP32 sums)
                            const uint4 cur = *reinterpret_cast<const uint4*>(t2s + lane * 16);
                            if ((hb & 1) == 0) {
                                l2_carry = cur;
                            } else if (lane < nrows) {
                                const TOut* a2 = reinterpret_cast<const TOut*>(&l2_carry);
                                const TOut* b2 = reinterpret_cast<const TOut*>(&cur);
                                float l3[4];
#pragma unroll
                                for (int c3 = 0; c3 < 4; c3++)
                                    l3[c3] = 0.25f * ((to_float(a2[2 * c3]) + to_float(a2[2 * c3 + 1])) +
                                                      (to_float(b2[2 * c3]) + to_float(b2[2 * c3 + 1])));
                                uint8_t* g3 = static_cast<uint8_t*>(p.out[3]) +
                                              ((size_t)(row0 + lane) * (size_t)((p.H >> 3) * (p.W >> 3)) +
                                               (size_t)(hb >> 1) * (p.W >> 3) + ch * 4) * sizeof(TOut);
                                *reinterpret_cast<uint2*>(g3) = make_uint2(pack2<TOut>(l3[0], l3[1]),
                                                                           pack2<TOut>(l3[2], l3[3]));
                            }
                        }
                        tc_fence_before();
                        fence_proxy_async();  // generic-proxy staging writes -> the TMA engine
                        __syncwarp();
                        if (lane == 0) mbar_arrive(&barAcc_empty[acc]);
                        if (lane == 0 && nrows > 0) {
                            const int h0 = hb * 4;  // the tile's first target row
                            const int y = (int)row0;
                            tma_store_3d(&mapO0, t0s, ch * 32, y, h0);
                            if (p.levels > 1) tma_store_3d(&mapO1, t1s, ch * 16, y, h0 / 2);
                            if (p.levels > 2) tma_store_3d(&mapO2, t2s, ch * 8, y, h0 / 4);
                            bulk_commit();
                        }
                        __syncwarp();
                        continue;
                    }
                    if (p.rowsplit) {
                        const int rh = warp >> 2;
                        uint8_t* s0 = st;
                        uint8_t* s1 = st + 32 * kR0;
                        uint8_t* s2 = st + 32 * (kR0 + kR1);
#pragma unroll 1
                        for (int cb = 0; cb < 4; cb++) {
                            float blk[4][8];
#pragma unroll
                            for (int r = 0; r < 4; r++)
                                tmem_ld8(tmem + lane_addr + (uint32_t)(acc * 256 + (4 * rh + r) * 32 + cb * 8), blk[r]);
                            tmem_wait_ld();
#pragma unroll
                            for (int r = 0; r < 4; r++) sts_n<TOut, 8>(s0 + lane * kR0 + r * 64 + cb * 16, blk[r]);
                            float l1[2][4];
#pragma unroll
                            for (int r = 0; r < 2; r++)
#pragma unroll
                                for (int c2 = 0; c2 < 4; c2++)
                                    l1[r][c2] = 0.25f * ((blk[2 * r][2 * c2] + blk[2 * r][2 * c2 + 1]) +
                                                         (blk[2 * r + 1][2 * c2] + blk[2 * r + 1][2 * c2 + 1]));
#pragma unroll
                            for (int r = 0; r < 2; r++) sts_n<TOut, 4>(s1 + lane * kR1 + r * 32 + cb * 8, l1[r]);
                            float l2[2];
#pragma unroll
                            for (int c2 = 0; c2 < 2; c2++)
                                l2[c2] = 0.25f * ((l1[0][2 * c2] + l1[0][2 * c2 + 1]) + (l1[1][2 * c2] + l1[1][2 * c2 + 1]));
                            sts_n<TOut, 2>(s2 + lane * kR2 + cb * 4, l2);
                        }
                        // the whole accumulator slice of this warp is read: release TMEM
                        tc_fence_before();
                        __syncwarp();
                        if (lane == 0) mbar_arrive(&barAcc_empty[acc]);
                        __syncwarp();
                        const int h0 = hb * p.th, w0 = wb * TW;
                        {
                            uint8_t* g0 = static_cast<uint8_t*>(p.out[0]) + (size_t)row0 * rs[0] +
                                          ((size_t)(h0 + 4 * rh) * W + w0) * sz;
#pragma unroll 4
                            for (int it = 0; it < 16; it++) {
                                const int j = lane + 32 * it, i = j >> 4, r = (j >> 2) & 3, k = j & 3;
                                if (i < nrows)
                                    *reinterpret_cast<uint4*>(g0 + (size_t)i * rs[0] + (size_t)r * ss[0] + k * 16) =
                                        *reinterpret_cast<const uint4*>(s0 + i * kR0 + r * 64 + k * 16);
                            }
                        }
                        if (p.levels > 1) {
                            uint8_t* g1 = static_cast<uint8_t*>(p.out[1]) + (size_t)row0 * rs[1] +
                                          ((size_t)(h0 / 2 + 2 * rh) * (W / 2) + w0 / 2) * sz;
#pragma unroll
                            for (int it = 0; it < 4; it++) {
                                const int j = lane + 32 * it, i = j >> 2, r = (j >> 1) & 1, k = j & 1;
                                if (i < nrows)
                                    *reinterpret_cast<uint4*>(g1 + (size_t)i * rs[1] + (size_t)r * ss[1] + k * 16) =
                                        *reinterpret_cast<const uint4*>(s1 + i * kR1 + r * 32 + k * 16);
                            }
                        }
                        if (p.levels > 2 && lane < nrows) {
                            uint8_t* g2 = static_cast<uint8_t*>(p.out[2]) + (size_t)row0 * rs[2] +
                                          ((size_t)(h0 / 4 + rh) * (W / 4) + w0 / 4) * sz;
                            *reinterpret_cast<uint4*>(g2 + (size_t)lane * rs[2]) =
                                *reinterpret_cast<const uint4*>(s2 + lane * kR2);
                        }
                        __syncwarp();
                        continue;
                    }
                }
                for (int c = col_lo; c < col_hi; c += PW) {
                    const int pw = min(PW, col_hi - c);  // PW, or 8 when TW = 8
                    for (int cb = 0; cb < pw / 8; cb++) {
                        float blk[8][8];
#pragma unroll
                        for (int r = 0; r < 8; r++)
                            tmem_ld8(tmem + lane_addr + (uint32_t)(acc * 256 + r * TW + c + cb * 8), blk[r]);
                        tmem_wait_ld();
                        stage_block<TOut>(st, lane, cb, blk);
                    }
                    if (c + PW >= col_hi) {
                        // the whole accumulator slice of this warp is read: release TMEM
                        tc_fence_before();
                        __syncwarp();
                        if (lane == 0) mbar_arrive(&barAcc_empty[acc]);
                    }
                    __syncwarp();
                    const int h0 = hb * p.th, w0 = wb * TW + c;
                    uint8_t* lvl[4];
                    for (int l = 0; l < 4; l++)
                        lvl[l] = l < p.levels
                                     ? static_cast<uint8_t*>(p.out[l]) + (size_t)row0 * rs[l] +
                                           ((size_t)(h0 >> l) * (W >> l) + (w0 >> l)) * sz
                                     : nullptr;
                    if (pw == PW)
                        flush_pass<TOut, PW>(st, nrows, lvl, rs, ss, p.levels, lane);
                    else
                        flush_pass<TOut, 8>(st, nrows, lvl, rs, ss, p.levels, lane);
                    __syncwarp();
                }
            }
        }
    }
    // every TMA store of this thread has completed before the CTA exits
    if (p.tma_store && warp < kEpiWarps && lane == 0) bulk_wait_all();
    __syncthreads();
    if (fail && tid == 0) atomicExch(p.err, 1);
    if (warp == kMmaWarp) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem));
    }
}

// ---------------------------------------------------------------- level 3

// out (rows, Hi/2, Wi/2) = 2x2 average of in (rows, Hi, Wi), 16-bit, FP32 sums
// (the row-split epilogue's level 3 from its stored level 2).  One thread per
// output row: two 2*Wi-byte input rows in, one Wi-byte row out, 16-byte accesses
// (Wi = 16: level 2 of a 64-wide map; the host launches it only then).
template <typename T>
__global__ void __launch_bounds__(256) pool_level_kernel(const T* __restrict__ in, T* __restrict__ out, long rows,
                                                         int Hi, int Wi) {
    const int Ho = Hi / 2;
    const long n = rows * Ho;
    for (long idx = (long)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (long)gridDim.x * blockDim.x) {
        const int y = (int)(idx % Ho);
        const long r = idx / Ho;
        const uint4* s0 = reinterpret_cast<const uint4*>(in + (r * Hi + 2 * y) * Wi);
        const uint4* s1 = reinterpret_cast<const uint4*>(in + (r * Hi + 2 * y + 1) * Wi);
        const uint4 a0 = s0[0], a1 = s0[1], b0 = s1[0], b1 = s1[1];
        const T* ra = reinterpret_cast<const T*>(&a0);
        const T* rb = reinterpret_cast<const T*>(&a1);
        const T* sa = reinterpret_cast<const T*>(&b0);
        const T* sb = reinterpret_cast<const T*>(&b1);
        float v[8];
#pragma unroll
        for (int x = 0; x < 8; x++) {
            const T* u = x < 4 ? ra : rb;
            const T* w = x < 4 ? sa : sb;
            const int c = 2 * (x & 3);
            v[x] = 0.25f * ((static_cast<float>(u[c]) + static_cast<float>(u[c + 1])) +
                            (static_cast<float>(w[c]) + static_cast<float>(w[c + 1])));
        }
        *reinterpret_cast<uint4*>(out + (r * Ho + y) * (Wi / 2)) =
            make_uint4(pack2<T>(v[0], v[1]), pack2<T>(v[2], v[3]), pack2<T>(v[4], v[5]), pack2<T>(v[6], v[7]));
    }
}

// ---------------------------------------------------------------- pack pass

// F (num, C, H, W) -> rows (num, HW, Kp) of 16-bit type, scaled by 1/4;
// permute: target-block pixel order (th x TW blocks) for the B operand.  One
// CTA transposes a 64-channel x 128-pixel tile through shared memory with
// 16-byte global loads (along pixels) and 16-byte stores (along channels).
// The tile is held pixel-major (128 rows of 64 channels = 128 B); the 16-byte
// channel chunk c8 of pixel row p sits at chunk c8 ^ ((p >> 3) & 7), so the
// 2-byte stores of 16 lanes with pixels 8 apart spread over 8 bank groups and a
// pixel row's eight chunks are read conflict-free as one 16-byte load each.
template <typename TIn, typename TOp>
__global__ void __launch_bounds__(256) pack_kernel(const TIn* __restrict__ f, TOp* __restrict__ out, int C, int Kp,
                                                   int H, int W, int TW, int th, int permute) {
    constexpr int kPx = 128, kCh = 64;
    __shared__ __align__(16) TOp tile[kPx][kCh];
    const int e = blockIdx.z;
    const int HW = H * W;
    const int p0 = blockIdx.x * kPx;
    const int c0 = blockIdx.y * kCh;
    const TIn* src = f + (size_t)e * C * HW;
    constexpr int V = 16 / (int)sizeof(TIn);  // input elements per 16-byte load
    const bool vec_ok = (HW % V) == 0 && (reinterpret_cast<uintptr_t>(f) % 16) == 0;
    for (int i = threadIdx.x; i < kCh * (kPx / V); i += blockDim.x) {
        const int cc = i / (kPx / V), pv = (i % (kPx / V)) * V;
        const int c = c0 + cc, px = p0 + pv;
        float v[V];
        if (c < C && vec_ok && px + V <= HW) {
            const uint4 raw = __ldg(reinterpret_cast<const uint4*>(src + (size_t)c * HW + px));
            const TIn* rv = reinterpret_cast<const TIn*>(&raw);
#pragma unroll
            for (int k = 0; k < V; k++) v[k] = static_cast<float>(rv[k]);
        } else {
#pragma unroll
            for (int k = 0; k < V; k++)
                v[k] = (c < C && px + k < HW) ? static_cast<float>(src[(size_t)c * HW + px + k]) : 0.f;
        }
#pragma unroll
        for (int k = 0; k < V; k++) {
            const int pp = pv + k;
            tile[pp][(((cc >> 3) ^ ((pp >> 3) & 7)) << 3) | (cc & 7)] = static_cast<TOp>(v[k] * 0.25f);
        }
    }
    __syncthreads();
    // each thread writes 8 consecutive channels (16 bytes) of one pixel
    for (int i = threadIdx.x; i < kPx * (kCh / 8); i += blockDim.x) {
        const int pp = i / (kCh / 8), c8 = i % (kCh / 8), cg = c8 * 8;
        const int px = p0 + pp;
        if (px >= HW || c0 + cg >= Kp) continue;
        int row = px;
        if (permute) {
            const int h = px / W, w = px % W;
            const int hb = h / th, r = h % th, wb = w / TW, c = w % TW;
            row = ((hb * (W / TW) + wb) * th + r) * TW + c;
        }
        *reinterpret_cast<uint4*>(out + ((size_t)e * HW + row) * Kp + c0 + cg) =
            *reinterpret_cast<const uint4*>(&tile[pp][(c8 ^ ((pp >> 3) & 7)) << 3]);
    }
}


// ---------------------------------------------------------------- host side

int make_map(CUtensorMap* map, void* base, CUtensorMapDataType dt, uint64_t rows, int Kp, int box_rows) {
    EncodeTiled enc = get_encode();
    if (!enc) return VIPE_ERR_CUDA;
    const cuuint64_t dims[2] = {(cuuint64_t)Kp, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)Kp * 2};
    const cuuint32_t box[2] = {(cuuint32_t)kKC, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(map, dt, 2, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? VIPE_OK : VIPE_ERR_CUDA;
}

// output level l (16-bit) as a 3-D map: dim 0 target columns (W_l), dim 1 source pixels
// (num * H * W, stride one level plane), dim 2 target rows (H_l, stride one target row);
// box (32 >> l, 32, 4 >> l) = one epilogue warp's rows of one tile
int make_out_map(CUtensorMap* map, void* base, CUtensorMapDataType dt, uint64_t src_rows, int Hl, int Wl, int l,
                 CUtensorMapSwizzle swz) {
    EncodeTiled enc = get_encode();
    if (!enc) return VIPE_ERR_CUDA;
    const cuuint64_t dims[3] = {(cuuint64_t)Wl, (cuuint64_t)src_rows, (cuuint64_t)Hl};
    const cuuint64_t strides[2] = {(cuuint64_t)Hl * Wl * 2, (cuuint64_t)Wl * 2};
    const cuuint32_t box[3] = {(cuuint32_t)(32 >> l), 32u, (cuuint32_t)(4 >> l)};
    const cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = enc(map, dt, 3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, swz,
                     CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? VIPE_OK : VIPE_ERR_CUDA;
}

// a 16-bit feature map (num, C, H*W) as a 3-D map: dim 0 pixels, dim 1 channels, dim 2 maps;
// box 64 pixels x 64 channels (one MN-major 128-byte swizzled operand atom column)
int make_fmap_map(CUtensorMap* map, const void* base, CUtensorMapDataType dt, int HW, int C, int num) {
    EncodeTiled enc = get_encode();
    if (!enc) return VIPE_ERR_CUDA;
    const cuuint64_t dims[3] = {(cuuint64_t)HW, (cuuint64_t)C, (cuuint64_t)num};
    const cuuint64_t strides[2] = {(cuuint64_t)HW * 2, (cuuint64_t)C * HW * 2};
    const cuuint32_t box[3] = {64u, (cuuint32_t)kKC, 1u};
    const cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = enc(map, dt, 3, const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? VIPE_OK : VIPE_ERR_CUDA;
}

int pick_tw(int W) {
    if (W % 32 == 0) return 32;
    if (W % 16 == 0) return 16;
    if (W % 8 == 0) return 8;
    return 0;
}

template <typename T>
size_t smem_bytes(int KC, int N) {
    return a_region(KC) + (size_t)KC * b_box(N) + kEpiWarps * (size_t)Stage<T>::per_warp + 1024;
}

bool g_attr_set[64] = {false};

}  // namespace cbuild
}  // namespace vipe

using namespace vipe;
using namespace vipe::cbuild;

extern "C" size_t vipe_corr_volume_workspace_size(int num, int C, int ht, int wd) {
    if (num <= 0 || C <= 0 || ht <= 0 || wd <= 0) return 0;
    const size_t Kp = (size_t)((C + kKC - 1) / kKC) * kKC;
    const size_t rows = (size_t)num * ht * wd;
    // error word + two packed operands (16-bit)
    return 256 + 2 * (((rows * Kp * 2) + 255) & ~size_t(255));
}

extern "C" int vipe_corr_volume_build(int in_dtype, int out_dtype, const void* fmap1, const void* fmap2, int num,
                                      int C, int ht, int wd, int num_levels, void* const* level_out, void* workspace,
                                      size_t workspace_bytes, void* stream) {
    if (num <= 0 || C <= 0 || ht <= 0 || wd <= 0 || num_levels < 1 || num_levels > 4) return VIPE_ERR_ARG;
    if (!fmap1 || !fmap2 || !level_out || !workspace) return VIPE_ERR_ARG;
    for (int l = 0; l < num_levels; l++)
        if (!level_out[l]) return VIPE_ERR_ARG;
    int TW = pick_tw(wd);
    if (TW == 0 || ht % kTH != 0) return VIPE_ERR_CAPACITY;  // fused pooling needs 8 x 8 closable blocks
    const int Kp = ((C + kKC - 1) / kKC) * kKC;
    if (Kp / kKC > kMaxKC) return VIPE_ERR_CAPACITY;
    if (in_dtype != VIPE_F16 && in_dtype != VIPE_BF16 && in_dtype != VIPE_F32) return VIPE_ERR_DTYPE;
    if (out_dtype != VIPE_F32 && out_dtype != VIPE_F16 && out_dtype != VIPE_BF16) return VIPE_ERR_DTYPE;
    if (workspace_bytes < vipe_corr_volume_workspace_size(num, C, ht, wd)) return VIPE_ERR_WORKSPACE;
    cudaStream_t st = as_stream(stream);
    const int HW = ht * wd;
    const size_t rows = (size_t)num * HW;
    const size_t op_bytes = ((rows * Kp * 2) + 255) & ~size_t(255);
    // workspace: [error word, 256 B][packed F1][packed F2]
    char* ws = static_cast<char*>(workspace);
    int* err = reinterpret_cast<int*>(ws);
    void* pa = ws + 256;
    void* pb = ws + 256 + op_bytes;
    VIPE_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(int), st));

    // epilogue mode, decided before the pack (it fixes the B pixel order): 16-bit 64-wide maps
    // use full-row tiles (4 x 64) stored by TMA when the output maps encode; other 16-bit
    // shapes with 32-wide blocks the row-split epilogue; the rest the column-half epilogue
    bool al16 = true;
    for (int l = 0; l < num_levels; l++) al16 &= (reinterpret_cast<uintptr_t>(level_out[l]) % 16) == 0;
    // (level 3 of the row-split and full-row paths is pooled by a 16-byte-row kernel for 64-wide maps)
    const int rowsplit = (out_dtype != VIPE_F32 && TW == 32 && al16 && (num_levels < 4 || wd == 64)) ? 1 : 0;
    CUtensorMap mO[3];
    int tma_store = 0, th = kTH;
    if (rowsplit && wd == 64 && HW % 32 == 0) {
        const CUtensorMapDataType odt =
            out_dtype == VIPE_F16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
        const CUtensorMapSwizzle swz[3] = {CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_SWIZZLE_32B,
                                           CU_TENSOR_MAP_SWIZZLE_NONE};
        bool ok = true;
        const int nl = std::min(num_levels, 3);
        for (int l = 0; l < 3 && ok; l++) {
            const int ll = l < nl ? l : 0;  // unused maps repeat level 0 (never issued)
            ok = make_out_map(&mO[l], level_out[ll], odt, (uint64_t)num * HW, ht >> ll, wd >> ll, ll, swz[ll]) ==
                 VIPE_OK;
        }
        if (ok) {
            tma_store = 1;
            TW = 64;
            th = 4;
        }
    }

    // operand type: FP16 inputs stay FP16, others go to BF16
    const int op_fmt = (in_dtype == VIPE_F16) ? 0 : 1;
    const CUtensorMapDataType dt = op_fmt == 0 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
    // Full-row tiles of 16-bit maps with whole 64-channel boxes load the A operand (read once per
    // work item) straight from fmap1 (num, C, H*W): for a fixed channel the pixels are contiguous,
    // which is the MN-major operand layout.  The B operand, re-read by every work item of its edge,
    // stays packed K-major (contiguous 128-byte rows load faster than 64 strided ones).
    CUtensorMap mA, mB;
    int direct = 0;
    if (tma_store && in_dtype != VIPE_F32 && C == Kp && (HW % 8) == 0 && reinterpret_cast<uintptr_t>(fmap1) % 16 == 0)
        direct = make_fmap_map(&mA, fmap1, dt, HW, C, num) == VIPE_OK;
    dim3 pg(ceil_div(HW, 128), Kp / kKC, num);
    {
        VIPE_PROF("corr_pack", st);
        for (int side = direct ? 1 : 0; side < 2; side++) {
            const void* src = side == 0 ? fmap1 : fmap2;
            void* dst = side == 0 ? pa : pb;
            const int perm = side;
            if (in_dtype == VIPE_F16)
                pack_kernel<__half, __half><<<pg, 256, 0, st>>>(static_cast<const __half*>(src),
                                                                static_cast<__half*>(dst), C, Kp, ht, wd, TW, th, perm);
            else if (in_dtype == VIPE_BF16)
                pack_kernel<__nv_bfloat16, __nv_bfloat16><<<pg, 256, 0, st>>>(
                    static_cast<const __nv_bfloat16*>(src), static_cast<__nv_bfloat16*>(dst), C, Kp, ht, wd, TW, th, perm);
            else
                pack_kernel<float, __nv_bfloat16><<<pg, 256, 0, st>>>(static_cast<const float*>(src),
                                                                      static_cast<__nv_bfloat16*>(dst), C, Kp, ht,
                                                                      wd, TW, th, perm);
            VIPE_LAUNCH_CHECK();
        }
    }
    const int N = th * TW;
    int rc;
    if (!direct && (rc = make_map(&mA, pa, dt, rows, Kp, kBM)) != VIPE_OK) return rc;
    if ((rc = make_map(&mB, pb, dt, rows, Kp, N)) != VIPE_OK) return rc;

    Params p;
    p.num = num; p.C = C; p.Kp = Kp; p.H = ht; p.W = wd; p.HW = HW; p.TW = TW; p.N = N; p.levels = num_levels;
    p.mtiles = (HW + kBM - 1) / kBM;
    p.ntiles = HW / N;
    p.items = (long)num * p.mtiles;
    p.out_dtype = out_dtype;
    for (int l = 0; l < 4; l++) p.out[l] = l < num_levels ? level_out[l] : nullptr;
    p.err = err;
    p.rowsplit = rowsplit;
    p.tma_store = tma_store;
    p.th = th;
    p.direct = direct;
    if (!p.tma_store) mO[0] = mO[1] = mO[2] = mA;  // placeholders, never used

    int dev = 0, sms = 148;
    VIPE_CUDA_TRY(cudaGetDevice(&dev));
    VIPE_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    size_t smem;
    if (out_dtype == VIPE_F32)
        smem = smem_bytes<float>(Kp / kKC, N);
    else
        smem = smem_bytes<__half>(Kp / kKC, N);
    if (dev < 64 && !g_attr_set[dev]) {
        VIPE_CUDA_TRY(cudaFuncSetAttribute(corr_build_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem_bytes<float>(kMaxKC, 256)));
        VIPE_CUDA_TRY(cudaFuncSetAttribute(corr_build_kernel<__half>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem_bytes<__half>(kMaxKC, 256)));
        VIPE_CUDA_TRY(cudaFuncSetAttribute(corr_build_kernel<__nv_bfloat16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem_bytes<__nv_bfloat16>(kMaxKC, 256)));
        g_attr_set[dev] = true;
    }
    const int grid = (int)std::min<long>(p.items, (long)sms);
    {
        VIPE_PROF("corr_build", st);
        if (out_dtype == VIPE_F32)
            corr_build_kernel<float><<<grid, kThreads, smem, st>>>(mA, mB, mO[0], mO[1], mO[2], p, op_fmt);
        else if (out_dtype == VIPE_F16)
            corr_build_kernel<__half><<<grid, kThreads, smem, st>>>(mA, mB, mO[0], mO[1], mO[2], p, op_fmt);
        else
            corr_build_kernel<__nv_bfloat16><<<grid, kThreads, smem, st>>>(mA, mB, mO[0], mO[1], mO[2], p, op_fmt);
    }
    VIPE_LAUNCH_CHECK();
    if (p.rowsplit && num_levels > 3 && !p.tma_store) {  // (full-row tiles pool level 3 in the epilogue)
        if (wd != 64) {
            set_last_error("corr_volume_build: level 3 of the row-split path expects 64-wide maps");
            return VIPE_ERR_CAPACITY;
        }
        const long rows = (long)num * HW;
        const long n3 = rows * (ht / 8);
        const unsigned pgrid = (unsigned)std::min<long>((n3 + 255) / 256, (long)sms * 16);
        VIPE_PROF("corr_pool_level", st);
        if (out_dtype == VIPE_F16)
            pool_level_kernel<__half><<<pgrid, 256, 0, st>>>(static_cast<const __half*>(level_out[2]),
                                                               static_cast<__half*>(level_out[3]), rows, ht / 4,
                                                               wd / 4);
        else
            pool_level_kernel<__nv_bfloat16><<<pgrid, 256, 0, st>>>(
                static_cast<const __nv_bfloat16*>(level_out[2]), static_cast<__nv_bfloat16*>(level_out[3]), rows,
                ht / 4, wd / 4);
        VIPE_LAUNCH_CHECK();
    }
    return VIPE_OK;
}
