// Long causal FIR filters as overlap-save convolutions on the library's Stockham transforms.
//
// Two real lines a, b form one complex signal z = x_a + i x_b.  The taps are real, so
// IFFT(FFT(z) . FFT(h)) carries the two convolutions in its real and imaginary parts.  A
// block of N samples (N = 1024 up to 384 taps, 4096 up to 512, 8192 / 16384 for longer filters) yields
// its last N - (nb - 1) outputs, the ones whose window lies inside the block; block j
// starts nb - 1 samples before its first output, so the blocks tile the line with zero
// extension before sample 0 (the causal definition of filtering_typed.cpp:1545-1590).
// Each block is one CTA-resident transform pair: load, forward FFT, product with the tap
// spectrum (scaled by 1/N), inverse FFT, store -- one HBM pass, about 2 x 5 log2 N flops per
// complex sample instead of 2 nb per real output.
#include "fft_core.cuh"
#include "zkx_internal.h"

namespace zkx {
namespace {

// H = FFT(b zero-padded to N) / N in one CTA (real taps, imaginary parts zero).
template <int N>
__global__ void __launch_bounds__(FftPlan<N, elems_for(N)>::T)
fir_spectrum_kernel(const float* __restrict__ b, int nb, float2* __restrict__ H, const float2* __restrict__ tw)
{
    using PL = FftPlan<N, elems_for(N)>;
    extern __shared__ float2 sm[];
    const int t = threadIdx.x;
    constexpr float scale = 1.0f / (float)N;  // exact: N is a power of two
    float2 v[PL::E];
#pragma unroll
    for (int r = 0; r < PL::E; ++r) {
        const int e = t + PL::T * r;
        v[r] = make_float2(e < nb ? b[e] * scale : 0.f, 0.f);
    }
    fft_block<PL, -1, 1>(v, sm, t, tw);
#pragma unroll
    for (int r = 0; r < PL::E; ++r) H[t + PL::T * r] = v[r];
}

// CTAs per SM the register budget is sized for: four 128-thread CTAs for 1024 points (128
// registers, 47.5 us against 51.5 us with three at 168 registers and 53.6 us with five,
// which spill; 127 taps on 16 x 2^20); two for the other 32-value plans (three would cap
// them at 80 registers and spill); three of up to 256 threads otherwise.
template <int N, int G>
constexpr int fir_fft_min_blocks()
{
    return N == 1024 ? 4
         : G * FftPlan<N, elems_for(N)>::T > 256 ? 1
         : elems_for(N) >= 32 ? 2 : 3;
}

template <int N, int G>
__global__ void __launch_bounds__(G * FftPlan<N, elems_for(N)>::T, (fir_fft_min_blocks<N, G>()))
fir_fft_kernel(const float* __restrict__ x, int lines, int n, int nb, const float2* __restrict__ H,
               const float* __restrict__ zi, float* __restrict__ y, const float2* __restrict__ tw)
{
    using PL = FftPlan<N, elems_for(N)>;
    extern __shared__ float2 sm[];
    const int g = threadIdx.x / PL::T;
    const int t = threadIdx.x - g * PL::T;
    float2* smg = sm + g * PL::smem_elems();
    const int hist = nb - 1;
    const int step = N - hist;                         // outputs per block
    const long long block = (long long)blockIdx.x * G + g;
    const long long out0 = block * step;               // first output of the block
    const long long s0 = out0 - hist;                  // first input sample of the block
    const int la = 2 * blockIdx.y, lb = la + 1;
    const bool has_b = lb < lines;
    const bool active = out0 < n;
    const float* xa = x + (size_t)la * n;
    const float* xb = x + (size_t)(has_b ? lb : la) * n;
    float2 v[PL::E];
    // blocks wholly inside the line (all but the first and last of each line) load at
    // constant offsets from the block's first sample, without per-sample range checks
    if (active && s0 >= 0 && s0 + N <= n) {
        const float* pa = xa + s0 + t;
        const float* pb = xb + s0 + t;
#pragma unroll
        for (int r = 0; r < PL::E; ++r) {
            const float a = __ldcs(pa + PL::T * r);
            const float b = __ldcs(pb + PL::T * r);
            v[r] = make_float2(a, has_b ? b : 0.f);
        }
    } else {
#pragma unroll
        for (int r = 0; r < PL::E; ++r) {
            const long long s = s0 + t + PL::T * r;
            const bool in = active && s >= 0 && s < n;
            v[r] = make_float2(in ? __ldcs(&xa[s]) : 0.f, (in && has_b) ? __ldcs(&xb[s]) : 0.f);
        }
    }
    fft_block<PL, -1, 1>(v, smg, t, tw);
#pragma unroll
    for (int r = 0; r < PL::E; ++r) v[r] = cmul(v[r], __ldg(&H[t + PL::T * r]));
    if constexpr (PL::PASSES > 1) __syncthreads();
    fft_block<PL, 1, 1>(v, smg, t, tw);
    if (!active) return;
    float* ya = y + (size_t)la * n;
    float* yb = y + (size_t)lb * n;
    // every output of an interior block exists and none lies within the zi history
    if (s0 >= 0 && out0 + step <= n) {
        float* qa = ya + s0 + t;
        float* qb = yb + s0 + t;
#pragma unroll
        for (int r = 0; r < PL::E; ++r) {
            if (t + PL::T * r >= hist) {
                qa[PL::T * r] = v[r].x;  // stays in L2 for the next stage
                if (has_b) qb[PL::T * r] = v[r].y;
            }
        }
        return;
    }
#pragma unroll
    for (int r = 0; r < PL::E; ++r) {
        const int e = t + PL::T * r;
        const long long o = s0 + e;
        if (e >= hist && o < n) {
            float va = v[r].x, vb = v[r].y;
            if (zi && o < hist) {
                va += zi[(size_t)la * hist + o];
                if (has_b) vb += zi[(size_t)lb * hist + o];
            }
            ya[o] = va;  // stays in L2 for the next stage
            if (has_b) yb[o] = vb;
        }
    }
}

template <int N>
int fir_fft_impl(const float* b, int nb, const float* x, int lines, int n, const float* zi, float* y,
                 cudaStream_t s)
{
    if (!twiddle_table()) return fail(ZKX_INTERNAL_ERROR, "twiddle table not initialised on this device");
    using PL = FftPlan<N, elems_for(N)>;
    StreamWorkspace ws;
    ws.stream = s;
    ZKX_TRY(stream_workspace((size_t)N * sizeof(float2), s, &ws.ptr));
    float2* H = static_cast<float2*>(ws.ptr);
    const size_t spec_smem = (size_t)PL::smem_elems() * sizeof(float2);
    ZKX_CUDA(cudaFuncSetAttribute(fir_spectrum_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)spec_smem));
    fir_spectrum_kernel<N><<<1, PL::T, spec_smem, s>>>(b, nb, H, twiddle_table());
    ZKX_LAUNCHED("fir_spectrum_kernel");
    constexpr int G = rows_per_cta(N);
    const size_t smem = (size_t)G * PL::smem_elems() * sizeof(float2);
    auto k = fir_fft_kernel<N, G>;
    ZKX_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const long long step = N - (nb - 1);
    const long long blocks = (n + step - 1) / step;
    const dim3 grid((unsigned)((blocks + G - 1) / G), (unsigned)((lines + 1) / 2));
    k<<<grid, G * PL::T, smem, s>>>(x, lines, n, nb, H, zi, y, twiddle_table());
    ZKX_LAUNCHED("fir_fft_kernel");
    return ZKX_SUCCESS;
}

}  // namespace

int launch_fir_fft(const float* b, int nb, const float* x, int lines, int n, const float* zi, float* y,
                   cudaStream_t stream)
{
    if ((lines + 1) / 2 > 65535) return fail(ZKX_UNSUPPORTED_OPERATION, "firfilter: more than 131070 lines");
    // measured on 16 x 2^20 samples: 1024 points (two radix-32 passes) beat 4096 (three
    // radix-16 passes) up to 383 taps (51.4 against 67.8 us at 127 taps, 61.9 against
    // 69.9 at 383) and tie at 511; 2048 points were never the fastest
    if (nb <= 384) return fir_fft_impl<1024>(b, nb, x, lines, n, zi, y, stream);
    if (nb <= 512) return fir_fft_impl<4096>(b, nb, x, lines, n, zi, y, stream);
    if (nb <= 1024) return fir_fft_impl<8192>(b, nb, x, lines, n, zi, y, stream);
    if (nb <= 4096) return fir_fft_impl<16384>(b, nb, x, lines, n, zi, y, stream);
    return fail(ZKX_UNSUPPORTED_OPERATION, "firfilter: more than 4096 taps");
}

}  // namespace zkx
