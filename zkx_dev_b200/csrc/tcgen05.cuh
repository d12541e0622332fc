// tcgen05 building blocks for sm_100a: tensor-memory allocation, the kind::f16 MMA with
// shared-memory operands, commit to an mbarrier, tensor-memory loads, the shared-memory
// and instruction descriptors, the canonical K-major operand layout, and the hi + lo
// FP16 / BF16 operand split used by the split-precision kernels.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "tma.cuh"  // smem_u32, mbarriers

namespace zkx {



__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t columns)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 ::"r"(smem_u32(slot)), "r"(columns) : "memory");
}
__device__ __forceinline__ void tmem_relinquish()
{
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t columns)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(columns)
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// D[tmem] (+)= A[smem] * B[smem]^T, kind::f16 (FP16 or BF16 operands, FP32 accumulate).
__device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc,
                                        uint32_t idesc, uint32_t accumulate)
{
    const uint32_t mask = 0;  // no disabled output lanes
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        ::"r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate),
          "r"(mask), "r"(mask), "r"(mask), "r"(mask)
        : "memory");
}

// Arrives on the mbarrier once every MMA this thread issued before has completed.
__device__ __forceinline__ void mma_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 ::"r"(smem_u32(bar)) : "memory");
}

// 32 consecutive FP32 columns of this thread's tensor-memory lane.
__device__ __forceinline__ void tmem_load32(uint32_t taddr, float* v)
{
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
        "%12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, "
        "%30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
          "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
          "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_load() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Shared-memory matrix descriptor, K-major, no swizzle: 8-row x 16-byte core matrices,
// `lbo` bytes between the two K halves of one MMA, `sbo` bytes between 8-row groups.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version of sm_100
    return d;
}

// Instruction descriptor of kind::f16: FP32 accumulator, A and B of format `fmt`
// (0 = FP16, 1 = BF16), both K-major, M x N.
constexpr uint32_t mma_idesc(int fmt, int m, int n)
{
    return (1u << 4) | ((uint32_t)fmt << 7) | ((uint32_t)fmt << 10) | ((uint32_t)(n >> 3) << 17) |
           ((uint32_t)(m >> 4) << 24);
}

// Byte offset of element (row, kk) of a K-major operand with `rows` rows: K blocks of 16
// (one MMA each) of rows x 16 elements; inside, 8-row groups of two 8 x 8 core matrices.
__device__ __forceinline__ uint32_t operand_offset(int rows, int row, int kk)
{
    return (uint32_t)(((kk >> 4) * (rows * 16) + (row >> 3) * 128 + ((kk & 15) >> 3) * 64 +
                       (row & 7) * 8 + (kk & 7)) * 2);
}
constexpr uint32_t kLbo = 128, kSbo = 256;

// ------------------------------------------------------------------ split formats

template <int FMT>
__device__ __forceinline__ void split_pair(float2 v, uint32_t& hi, uint32_t& lo)
{
    if constexpr (FMT == 0) {
        const __half2 h = __floats2half2_rn(v.x, v.y);
        const float2 hf = __half22float2(h);
        const __half2 l = __floats2half2_rn(v.x - hf.x, v.y - hf.y);
        hi = *reinterpret_cast<const uint32_t*>(&h);
        lo = *reinterpret_cast<const uint32_t*>(&l);
    } else {
        const __nv_bfloat162 h = __floats2bfloat162_rn(v.x, v.y);
        const float2 hf = __bfloat1622float2(h);
        const __nv_bfloat162 l = __floats2bfloat162_rn(v.x - hf.x, v.y - hf.y);
        hi = *reinterpret_cast<const uint32_t*>(&h);
        lo = *reinterpret_cast<const uint32_t*>(&l);
    }
}

template <int FMT>
__device__ __forceinline__ uint16_t split_one(float v, uint16_t& lo)
{
    if constexpr (FMT == 0) {
        const __half h = __float2half_rn(v);
        const __half l = __float2half_rn(v - __half2float(h));
        lo = *reinterpret_cast<const uint16_t*>(&l);
        return *reinterpret_cast<const uint16_t*>(&h);
    } else {
        const __nv_bfloat16 h = __float2bfloat16_rn(v);
        const __nv_bfloat16 l = __float2bfloat16_rn(v - __bfloat162float(h));
        lo = *reinterpret_cast<const uint16_t*>(&l);
        return *reinterpret_cast<const uint16_t*>(&h);
    }
}


// 16 consecutive FP32 columns of this thread's tensor-memory lane.
__device__ __forceinline__ void tmem_load16(uint32_t taddr, float* v)
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
        "%12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Stores 16 FP32 words into consecutive columns of this thread's tensor-memory lane
// (warp-collective); tmem_wait_store makes them visible to this thread's later loads.
__device__ __forceinline__ void tmem_store16(uint32_t taddr, const float* v)
{
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
        "%12, %13, %14, %15, %16};"
        ::"r"(taddr), "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
          "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
          "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])), "r"(__float_as_uint(v[8])),
          "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])), "r"(__float_as_uint(v[11])),
          "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])), "r"(__float_as_uint(v[14])),
          "r"(__float_as_uint(v[15]))
        : "memory");
}
__device__ __forceinline__ void tmem_wait_store() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// Exponent e such that max * 2^e lies below 2^14 (0 for an all-zero pulse), clamped to
// the range of normal FP32 powers of two.
__device__ __forceinline__ int range_exponent(float max_abs)
{
    if (!(max_abs > 0.f)) return 0;
    int e;
    frexpf(max_abs, &e);  // max_abs < 2^e
    return max(-126, min(126, 14 - e));
}
// 2^e for -126 <= e <= 127, exactly.
__device__ __forceinline__ float pow2(int e) { return __int_as_float((e + 127) << 23); }

}  // namespace zkx
