// Range compression with the DFT stages on the 5th-generation tensor cores (tcgen05),
// split hi + lo FP16 or BF16 operands accumulated in FP32: the precision path beside the
// plain FP32 shared-memory FFT (radar.cu).
//
// A transform of N = R1 * R2 * R3 points (4096 = 16*16*16, 8192 = 32*16*16,
// 16384 = 32*32*16) runs as three Stockham passes.  Pass i treats the N values as
// G = N / R groups of R values; the groups are the rows of A (G x 2R, real and imaginary
// parts interleaved along K) and one pass is the product D = A * B^T with B the
// real-embedded R-point DFT matrix (2R x 2R):
//
//   D[g][2k]   = sum_j Re u_j cos(2 pi jk/R) + Im u_j sin(2 pi jk/R)   (Re of output k)
//   D[g][2k+1] = sum_j Im u_j cos(2 pi jk/R) - Re u_j sin(2 pi jk/R)   (Im of output k)
//
// A and B are split into hi = fmt(v) and lo = fmt(v - hi) and D accumulates
// A_hi B_hi + A_hi B_lo + A_lo B_hi in FP32 in tensor memory (the lo*lo term is below the
// FP32 rounding of the sum).  One thread issues the M = 128 MMAs of a pass and commits
// them to an mbarrier; then every thread loads one D row (one group) from tensor memory,
// applies the Stockham twiddle W_Mprev^(n k) and the pass scale 1/R in FP32 and writes the
// outputs, split again, to the A rows of the next pass.  The inverse transform runs the
// same forward passes on conjugated data.  FP16 operands are kept in range by power-of-two
// scales chosen per pulse from the largest magnitude at the two entry points (the input
// and the spectrum product); all scales are exact and undone at the output.
//
// Shared memory: A_hi, A_lo (4N bytes each, the canonical K-major no-swizzle layout of
// 8-row x 16-byte core matrices) and the hi/lo DFT matrices; tensor memory: the FP32
// accumulators of one pass (2N / 128 columns).  One persistent 512-thread CTA per SM.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <type_traits>

#include "fft_core.cuh"
#include "tcgen05.cuh"
#include "tma.cuh"
#include "zkx_internal.h"

namespace zkx {
namespace {

constexpr int kTcThreads = 512;

// --------------------------------------------------------------------- the plan

template <int N>
struct TcPlan {
    static constexpr int R1 = N >= 8192 ? 32 : 16;
    static constexpr int R2 = N >= 16384 ? 32 : 16;
    static constexpr int R3 = 16;
    static_assert(R1 * R2 * R3 == N, "supported lengths: 4096, 8192, 16384");
    static constexpr int radix(int i) { return i == 0 ? R1 : i == 1 ? R2 : R3; }
    // sub-transform length before pass i (M_0 = N)
    static constexpr int mprev(int i) { return i == 0 ? N : i == 1 ? N / R1 : N / (R1 * R2); }
    static constexpr int COLUMNS = 2 * N / 128;  // tensor-memory columns of one pass
    static constexpr int TMEM_COLS = COLUMNS < 32 ? 32 : COLUMNS;
    static constexpr int A_BYTES = 4 * N;        // one of A_hi / A_lo
    static constexpr int B32_BYTES = 64 * 64 * 2, B16_BYTES = 32 * 32 * 2;
    static constexpr int SMEM = 2 * A_BYTES + 2 * B32_BYTES + 2 * B16_BYTES + 256;
};

struct TcShared {
    uint64_t bar;
    uint32_t tmem;
    int abort;
    float red[kTcThreads / 32];
};

// Position p of a buffer whose sub-transforms have length mbuf -> (group, slot) of the next
// pass with radix rn.
__device__ __forceinline__ void next_slot(int p, int mbuf, int rn, int& g, int& k)
{
    const int mn = mbuf / rn;
    const int s = p / mbuf, rem = p - s * mbuf;
    k = rem / mn;
    g = s * mn + (rem - k * mn);
}

template <int FMT>
__device__ __forceinline__ void store_split(uint8_t* a_hi, uint8_t* a_lo, int rows, int g, int k, float2 v)
{
    uint32_t hi, lo;
    split_pair<FMT>(v, hi, lo);
    const uint32_t off = operand_offset(rows, g, 2 * k);
    *reinterpret_cast<uint32_t*>(a_hi + off) = hi;
    *reinterpret_cast<uint32_t*>(a_lo + off) = lo;
}

// Largest |component| over the CTA (every thread passes its local maximum).
__device__ __forceinline__ float block_max(float m, TcShared* sh)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    __syncthreads();  // previous readers of red[] are done
    if ((threadIdx.x & 31) == 0) sh->red[threadIdx.x >> 5] = m;
    __syncthreads();
    float r = 0.f;
#pragma unroll
    for (int i = 0; i < kTcThreads / 32; ++i) r = fmaxf(r, sh->red[i]);
    return r;
}

// The real-embedded R-point DFT matrix, split, in the K-major operand layout (2R rows).
template <int R, int FMT>
__device__ void build_dft(uint8_t* b_hi, uint8_t* b_lo, const float2* __restrict__ tw)
{
    constexpr int ROWS = 2 * R;
    for (int i = threadIdx.x; i < ROWS * ROWS; i += blockDim.x) {
        const int n = i / ROWS, kk = i - n * ROWS;
        const int k = n >> 1, j = kk >> 1;
        const float2 w = tw[((j * k) % R) * (kTwiddleSize / R)];  // exp(-2 pi i jk / R)
        // row 2k (Re of output k) over (Re u_j, Im u_j): [w.x, -w.y]; row 2k+1: [w.y, w.x]
        float val;
        if ((n & 1) == 0) val = (kk & 1) == 0 ? w.x : -w.y;
        else val = (kk & 1) == 0 ? w.y : w.x;
        uint16_t lo;
        const uint16_t hi = split_one<FMT>(val, lo);
        const uint32_t off = operand_offset(ROWS, n, kk);
        *reinterpret_cast<uint16_t*>(b_hi + off) = hi;
        *reinterpret_cast<uint16_t*>(b_lo + off) = lo;
    }
}

template <int N, int FMT>
__global__ void __launch_bounds__(kTcThreads, 1)
tc_compression_kernel(const float2* __restrict__ x, int pulses, int samples,
                      const float2* __restrict__ spectrum, float2* __restrict__ y,
                      const float2* __restrict__ tw, int* err)
{
    using PL = TcPlan<N>;
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* a_hi = smem;
    uint8_t* a_lo = a_hi + PL::A_BYTES;
    uint8_t* b32_hi = a_lo + PL::A_BYTES;
    uint8_t* b32_lo = b32_hi + PL::B32_BYTES;
    uint8_t* b16_hi = b32_lo + PL::B32_BYTES;
    uint8_t* b16_lo = b16_hi + PL::B16_BYTES;
    TcShared* sh = reinterpret_cast<TcShared*>(b16_lo + PL::B16_BYTES);
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;

    if (PL::R1 == 32 || PL::R2 == 32) build_dft<32, FMT>(b32_hi, b32_lo, tw);
    build_dft<16, FMT>(b16_hi, b16_lo, tw);
    if (t == 0) {
        mbar_init(&sh->bar, 1);
        sh->abort = 0;
    }
    if (warp == 0) {
        tmem_alloc(&sh->tmem, PL::TMEM_COLS);
        tmem_relinquish();
    }
    fence_proxy_async_smem();  // DFT matrices written by the generic proxy, read by MMAs
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = sh->tmem;
    uint32_t phase = 0;
    bool ok = true;

    // One pass: MMAs of every row block, then each thread's D rows through `consume`.
    auto run_pass = [&](auto RADIX, auto consume) {
        constexpr int R = decltype(RADIX)::value;
        constexpr int G = N / R, BLOCKS = G / 128, KSTEPS = 2 * R / 16;
        constexpr uint32_t idesc = mma_idesc(FMT, 128, 2 * R);
        uint8_t* bh = R == 32 ? b32_hi : b16_hi;
        uint8_t* bl = R == 32 ? b32_lo : b16_lo;
        fence_proxy_async_smem();  // this thread's A stores -> visible to the MMAs
        tc_fence_before();
        __syncthreads();
        if (t == 0) {
            tc_fence_after();
            const uint32_t ah = smem_u32(a_hi), al = smem_u32(a_lo);
            const uint32_t bhs = smem_u32(bh), bls = smem_u32(bl);
#pragma unroll 1
            for (int b = 0; b < BLOCKS; ++b) {
#pragma unroll
                for (int j = 0; j < KSTEPS; ++j) {
                    const uint32_t aoff = (uint32_t)(j * G * 32 + b * 4096);
                    const uint32_t boff = (uint32_t)(j * 2 * R * 32);
                    const uint32_t d = tmem + (uint32_t)(b * 2 * R);
                    mma_f16(d, smem_desc(ah + aoff, kLbo, kSbo), smem_desc(bhs + boff, kLbo, kSbo), idesc, j > 0);
                    mma_f16(d, smem_desc(ah + aoff, kLbo, kSbo), smem_desc(bls + boff, kLbo, kSbo), idesc, 1);
                    mma_f16(d, smem_desc(al + aoff, kLbo, kSbo), smem_desc(bhs + boff, kLbo, kSbo), idesc, 1);
                }
            }
            mma_commit(&sh->bar);
        }
        const bool done = mbar_wait_bounded(&sh->bar, phase);
        phase ^= 1u;
        if (__syncthreads_or(!done)) {
            ok = false;
            return;
        }
        tc_fence_after();
        const int q = warp & 3, wc = warp >> 2;
        constexpr int MINE = (BLOCKS + kTcThreads / 128 - 1) / (kTcThreads / 128);
#pragma unroll
        for (int i = 0; i < MINE; ++i) {
            const int b = wc + (kTcThreads / 128) * i;
            if (b < BLOCKS) {
                float d[2 * R];
                const uint32_t taddr = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(b * 2 * R);
                tmem_load32(taddr, d);
                if constexpr (R == 32) tmem_load32(taddr + 32, d + 32);
                tmem_wait_load();
                consume(b * 128 + 32 * q + lane, d, i);
            }
        }
    };

    // Middle pass output: twiddle W_mprev^(n k), scale 1/R, store to the next pass's A.
    auto stockham_out = [&](auto PASS) {
        constexpr int I = decltype(PASS)::value;
        constexpr int R = PL::radix(I), MP = PL::mprev(I), MI = MP / R, PP = N / MP;
        constexpr int RN = PL::radix(I + 1), GN = N / RN;
        return [=](int g, const float* d, int) {
            const int s = g / MI, n = g - (g / MI) * MI;
#pragma unroll
            for (int k = 0; k < R; ++k) {
                float2 v = make_float2(d[2 * k] * (1.0f / R), d[2 * k + 1] * (1.0f / R));
                if (n != 0 && k != 0) v = cmul(v, __ldg(&tw[((n * k) & (MP - 1)) * (kTwiddleSize / MP)]));
                int g2, k2;
                next_slot((s + PP * k) * MI + n, MI, RN, g2, k2);
                store_split<FMT>(a_hi, a_lo, GN, g2, k2, v);
            }
        };
    };

    constexpr int R3 = PL::R3, G3 = N / R3, BL3 = G3 / 128;
    constexpr int MINE3 = (BL3 + 3) / 4;  // last-pass row blocks per thread
#pragma unroll 1
    for (int pulse = blockIdx.x; pulse < pulses && ok; pulse += gridDim.x) {
        // ---- input: zero-padded/truncated pulse, scaled into FP16 range, to A of pass 1
        const float2* xr = x + (size_t)pulse * samples;
        constexpr int PER = N / kTcThreads;
        float2 in[PER];
        float m = 0.f;
#pragma unroll
        for (int i = 0; i < PER; ++i) {
            const int e = t + kTcThreads * i;
            in[i] = e < samples ? __ldcs(&xr[e]) : make_float2(0.f, 0.f);
            m = fmaxf(m, fmaxf(fabsf(in[i].x), fabsf(in[i].y)));
        }
        const int e_in = range_exponent(block_max(m, sh));
        const float sc_in = pow2(e_in);
#pragma unroll
        for (int i = 0; i < PER; ++i) {
            int g, k;
            next_slot(t + kTcThreads * i, N, PL::R1, g, k);
            store_split<FMT>(a_hi, a_lo, N / PL::R1, g, k, make_float2(in[i].x * sc_in, in[i].y * sc_in));
        }
        // ---- forward passes 1, 2
        run_pass(std::integral_constant<int, PL::R1>{}, stockham_out(std::integral_constant<int, 0>{}));
        if (!ok) break;
        run_pass(std::integral_constant<int, PL::R2>{}, stockham_out(std::integral_constant<int, 1>{}));
        if (!ok) break;
        // ---- forward pass 3: bins g + (N/R3) k; product with the spectrum, kept in registers
        float2 z[MINE3][R3];
        int zg[MINE3];
#pragma unroll
        for (int i = 0; i < MINE3; ++i) zg[i] = -1;
        float zm = 0.f;
        run_pass(std::integral_constant<int, R3>{}, [&](int g, const float* d, int i) {
#pragma unroll
            for (int k = 0; k < R3; ++k) {
                const float2 v = make_float2(d[2 * k] * (1.0f / R3), d[2 * k + 1] * (1.0f / R3));
                const float2 p = cmul(v, __ldg(&spectrum[g + G3 * k]));
                z[i][k] = p;
                zm = fmaxf(zm, fmaxf(fabsf(p.x), fabsf(p.y)));
            }
            zg[i] = g;
        });
        if (!ok) break;
        const int e_mid = range_exponent(block_max(zm, sh));
        const float sc_mid = pow2(e_mid);
        // conjugated product -> A of inverse pass 1 (forward passes on conjugated data)
#pragma unroll
        for (int i = 0; i < MINE3; ++i) {
            if (zg[i] >= 0) {
#pragma unroll
                for (int k = 0; k < R3; ++k) {
                    int g, kk;
                    next_slot(zg[i] + G3 * k, N, PL::R1, g, kk);
                    store_split<FMT>(a_hi, a_lo, N / PL::R1, g, kk,
                                     make_float2(z[i][k].x * sc_mid, -z[i][k].y * sc_mid));
                }
            }
        }
        // ---- inverse passes 1, 2, 3
        run_pass(std::integral_constant<int, PL::R1>{}, stockham_out(std::integral_constant<int, 0>{}));
        if (!ok) break;
        run_pass(std::integral_constant<int, PL::R2>{}, stockham_out(std::integral_constant<int, 1>{}));
        if (!ok) break;
        // y = conj(result) * N^2 / (2^e_in 2^e_mid): every factor a power of two, applied as
        // two exact scalings so that no intermediate factor leaves the FP32 range
        constexpr int LOGN = ilog2(N), LOGR3 = ilog2(R3);
        const int e_out = 2 * LOGN - LOGR3 - e_in - e_mid;
        const int e1 = max(-126, min(126, e_out)), e2 = max(-126, min(126, e_out - e1));
        const float f1 = pow2(e1), f2 = pow2(e2);
        float2* yr = y + (size_t)pulse * N;
        run_pass(std::integral_constant<int, R3>{}, [&](int g, const float* d, int) {
#pragma unroll
            for (int k = 0; k < R3; ++k)
                yr[g + G3 * k] = make_float2(d[2 * k] * f1 * f2, -d[2 * k + 1] * f1 * f2);
        });
    }
    if (!ok && t == 0) atomicCAS(err, 0, (int)kKernelTmaTimeout);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, PL::TMEM_COLS);
    }
}

template <int N, int FMT>
int tc_impl(const float2* x, int pulses, int samples, const float2* spectrum, float2* y,
            cudaStream_t s)
{
    using PL = TcPlan<N>;
    auto k = tc_compression_kernel<N, FMT>;
    ZKX_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, PL::SMEM));
    int dev = 0, sms = 0;
    ZKX_CUDA(cudaGetDevice(&dev));
    ZKX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int grid = std::max(1, std::min(pulses, sms));
    k<<<grid, kTcThreads, PL::SMEM, s>>>(x, pulses, samples, spectrum, y, twiddle_table(),
                                          kernel_error_word());
    ZKX_LAUNCHED("tc_compression_kernel");
    return ZKX_SUCCESS;
}

}  // namespace

int launch_pulse_compression_tc(const float2* x, int pulses, int samples, int nfft,
                                const float2* spectrum, float2* y, int precision,
                                cudaStream_t stream)
{
    if (!twiddle_table()) return fail(ZKX_INTERNAL_ERROR, "twiddle table not initialised on this device");
    const int fmt = precision == ZKX_PRECISION_TC_F16 ? 0 : 1;
    switch (nfft) {
    case 4096: return fmt == 0 ? tc_impl<4096, 0>(x, pulses, samples, spectrum, y, stream)
                               : tc_impl<4096, 1>(x, pulses, samples, spectrum, y, stream);
    case 8192: return fmt == 0 ? tc_impl<8192, 0>(x, pulses, samples, spectrum, y, stream)
                               : tc_impl<8192, 1>(x, pulses, samples, spectrum, y, stream);
    case 16384: return fmt == 0 ? tc_impl<16384, 0>(x, pulses, samples, spectrum, y, stream)
                                : tc_impl<16384, 1>(x, pulses, samples, spectrum, y, stream);
    default:
        return fail(ZKX_UNSUPPORTED_OPERATION,
                    "tensor-core pulse_compression: nfft must be 4096, 8192 or 16384");
    }
}

}  // namespace zkx
