// TMA (cp.async.bulk.tensor) helpers shared by the tensor-core kernels (sm_100a): tiled
// loads into shared memory completing on an mbarrier, the MN-major 128-byte-swizzled
// operand descriptor, a bounded mbarrier wait that also gives up when another role of
// the CTA has failed, and the host-side tensor-map encoder (driver entry point).
#pragma once

#include "common.cuh"
#include "tcgen05.cuh"

#include <cuda.h>

#include <mutex>

namespace vipe {
namespace tc {

constexpr uint64_t kTmaWaitNs = 2000000000ull;  // 2 s bound on any mbarrier wait

// bounded wait; returns false (and flags the CTA) when 2 s pass or another role already failed
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* fail) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = gtimer();
    while (true) {
        if (mbar_try_wait(bar, parity)) return true;
        if (*fail) return false;
        if (gtimer() - t0 > kTmaWaitNs) break;
    }
    *fail = 1;
    return false;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y, int z) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
        : "memory");
}

// Shared-memory descriptor of an MN-major, 128-byte swizzled 16-bit operand: 64-element MN
// atoms (128-byte rows, one per K index) `atom_bytes` apart, 8-row K groups 1024 B apart.
__device__ __forceinline__ uint64_t smem_desc_sw128_mn(const void* base, uint32_t atom_bytes) {
    const uint64_t addr = smem_u32(base);
    uint64_t d = 0;
    d |= (addr >> 4) & 0x3FFFull;                       // start address
    d |= (uint64_t)((atom_bytes >> 4) & 0x3FFF) << 16;  // leading byte offset: next MN atom
    d |= (uint64_t)(1024 >> 4) << 32;                   // stride byte offset: next 8 K rows
    d |= (uint64_t)1 << 46;                             // descriptor version (sm100)
    d |= (uint64_t)2 << 61;                             // SWIZZLE_128B
    return d;
}

// ---------------------------------------------------------------- host side

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// cuTensorMapEncodeTiled through the runtime's driver entry point (no -lcuda); null if absent
inline EncodeTiled get_encode() {
    static EncodeTiled fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiled>(p);
    });
    return fn;
}

}  // namespace tc
}  // namespace vipe
