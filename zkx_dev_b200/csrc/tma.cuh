// Tensor-memory-accelerator (TMA) helpers for sm_100a: 2-D tiled bulk loads into
// shared memory completed on an mbarrier.  Single-GPU loads only: no cluster
// multicast is ever used.
//
// Every wait on an mbarrier is bounded (about one second of SM clocks); a CTA whose
// copy does not complete in time records an error code in the library's device error
// word and leaves instead of spinning forever.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>

namespace zkx {

// Error codes a kernel can leave in the device error word.
enum KernelError : int { kKernelOk = 0, kKernelTmaTimeout = 1 };

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase)
{
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
    return done != 0;
}

// Bounded wait: true when the phase completed, false after `limit` SM clocks (by default
// 2^31, about one second).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t phase, long long limit = 1LL << 31)
{
    const long long start = clock64();
    while (!mbar_try_wait(bar, phase)) {
        if (clock64() - start > limit) return false;
    }
    return true;
}

// 2-D tiled load of one box at element coordinates (x inner, y outer) into dst.
// x * element size must be a multiple of 16 bytes (callers pass 32-float steps).
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y,
                                            uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// 1-D bulk copy of `bytes` (a multiple of 16, both addresses 16-byte aligned) into
// shared memory, completing on `bar`.
__device__ __forceinline__ void bulk_load_1d(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// Asynchronous prefetch of [src, src + bytes) from global memory into L2 (no completion
// signal; src 16-byte aligned, bytes a multiple of 16).
__device__ __forceinline__ void bulk_prefetch_l2(const void* src, uint32_t bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

// Orders this thread's earlier generic-proxy shared-memory accesses before later
// async-proxy (bulk copy) writes to the same memory.
__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Host: encode a row-major 2-D FP32 tensor [outer, inner] with the given row pitch
// (bytes, a multiple of 16) and box (inner x outer elements).  Returns false when the
// driver entry point is unavailable or the encoding is rejected.
bool encode_tensor_map_2d_f32(CUtensorMap* map, const void* base, uint64_t inner, uint64_t outer,
                              uint64_t row_pitch_bytes, uint32_t box_inner, uint32_t box_outer);

}  // namespace zkx
