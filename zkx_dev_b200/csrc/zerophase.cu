// Zero-phase FIR filtering (firfilter2) and the analytic signal (hilbert) along the last
// axis of row-major [lines, n] float32 data.
//
// firfilter2 (filtering_typed.cpp:1226-1302 layout, 1631-1730 algorithm): each line is
// extended by `edge` samples on both sides (odd / even / constant reflection, or none),
// filtered forward with the steady-state initial condition (the FIR state for a constant
// input equal to the first extended sample: the same as extending the line to the left
// by that sample), then filtered again backwards with the same rule (extending the
// forward output to the right by its last value), and cropped back to n samples:
//
//   f[i] = sum_k b[k] E(i - k),   E(i < 0) = E(0)
//   y[m] = sum_k b[k] F(edge + m + k),   F(i >= ne - 1) = f[ne - 1],   ne = n + 2 edge.
//
// One CTA produces 16 (256 s - nbp / 16) outputs of one line (s sweeps, nbp = nb rounded up to
// 16) in a single HBM pass: the extended input
// window (with both halos) is built in shared memory straight from x, the forward pass
// writes the f window next to it, the backward pass reads it with the taps reversed.
// Both passes use the blocked register FIR of the causal filter (16 consecutive outputs
// per thread, 16-tap chunks, skewed shared blocks).  4 B in + 4 B out per sample, 4·nb
// FLOP per sample plus the halo (nbp / 4096).
//
// hilbert (filtering_typed.cpp:500-562 layout, 1813-1872 algorithm): x zero-padded or
// truncated to N along the axis, DFT, bins 1..ceil(N/2)-1 doubled, bin N/2 (N even) kept,
// the upper half zeroed, inverse DFT.  For N a power of two up to 16384 one kernel does
// load, forward FFT, mask, inverse FFT and store per line (4 B in, 8 B out per sample);
// other lengths run the library's batched transforms in place in the output.
#include <cuda_fp16.h>

#include <climits>

#include "fft_core.cuh"
#include "zkx_internal.h"

namespace zkx {
namespace {

constexpr int kZpThreads = 256;
constexpr int kZpPer = 16;
constexpr int kMaxZpTaps = 4096;
// With padding at least as long as the filter the one-convolution FFT path beats the two direct
// passes at every length measured: 16 x 2^20 samples, 7 taps 99 against 121 us, 127 taps 100
// against 250 us, 511 taps 117 against 757 us.
constexpr int kZpFftMinTaps = 1;

__host__ __device__ __forceinline__ int zp_word(int block) { return 20 * block; }  // 16 samples + 4 pad words

// 2 * endpoint - reflected with the rounding of the reference's padded element type:
// float arithmetic (ZKX_PAD_ROUND_F32), the same rounded to half (F16), or the integer
// wrap of an 8/16/32-bit element (filtering_typed.cpp:1597-1620).
__device__ __forceinline__ float odd_reflect(float endpoint, float reflected, int rounding)
{
    if (rounding == ZKX_PAD_ROUND_F16) {
        const float doubled = __half2float(__float2half_rn(__fmul_rn(2.0f, endpoint)));
        return __half2float(__float2half_rn(__fsub_rn(doubled, reflected)));
    }
    if (rounding == ZKX_PAD_ROUND_I8 || rounding == ZKX_PAD_ROUND_I16 || rounding == ZKX_PAD_ROUND_I32) {
        const int bits = rounding == ZKX_PAD_ROUND_I8 ? 8 : rounding == ZKX_PAD_ROUND_I16 ? 16 : 32;
        const long long modulus = 1LL << bits, sign = modulus / 2;
        long long v = 2LL * (long long)endpoint - (long long)reflected;
        v %= modulus;
        if (v < 0) v += modulus;
        if (v >= sign) v -= modulus;
        return (float)v;
    }
    return __fsub_rn(__fmul_rn(2.0f, endpoint), reflected);
}

// Extended sample i of a line (0 <= i < n + 2 edge; i < 0 reads sample 0).
__device__ __forceinline__ float extended_sample(const float* __restrict__ xl, int n, int edge, int padtype,
                                                 int rounding, long long i)
{
    if (i < 0) i = 0;
    if (i >= edge && i < (long long)edge + n) return xl[i - edge];
    if (i < edge) {
        const float endpoint = xl[0];
        if (padtype == ZKX_PAD_CONSTANT) return endpoint;
        const float r = xl[edge - i];
        return padtype == ZKX_PAD_EVEN ? r : odd_reflect(endpoint, r, rounding);
    }
    const int right = (int)(i - edge - n);
    const float endpoint = xl[n - 1];
    if (padtype == ZKX_PAD_CONSTANT) return endpoint;
    const float r = xl[n - 2 - right];
    return padtype == ZKX_PAD_EVEN ? r : odd_reflect(endpoint, r, rounding);
}

// acc[q] = sum_{k < nbp} taps[k] src[16 ob + q - k + nbp - 1] over skewed 16-sample blocks.
__device__ __forceinline__ void fir16(const float* __restrict__ taps, const float* __restrict__ src, int ob,
                                      int chunks, float (&acc)[kZpPer])
{
#pragma unroll
    for (int q = 0; q < kZpPer; ++q) acc[q] = 0.f;
    for (int c = 0; c < chunks; ++c) {
        float bv[16];
        const float4* tp = reinterpret_cast<const float4*>(taps + 16 * c);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const float4 t4 = tp[u];
            bv[4 * u] = t4.x; bv[4 * u + 1] = t4.y; bv[4 * u + 2] = t4.z; bv[4 * u + 3] = t4.w;
        }
        const int blk = ob + chunks - 1 - c;
        float xw[32];
        const float4* w0 = reinterpret_cast<const float4*>(src + zp_word(blk));
        const float4* w1 = reinterpret_cast<const float4*>(src + zp_word(blk + 1));
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const float4 a = w0[u], d = w1[u];
            xw[4 * u] = a.x; xw[4 * u + 1] = a.y; xw[4 * u + 2] = a.z; xw[4 * u + 3] = a.w;
            xw[16 + 4 * u] = d.x; xw[17 + 4 * u] = d.y; xw[18 + 4 * u] = d.z; xw[19 + 4 * u] = d.w;
        }
#pragma unroll
        for (int kk = 0; kk < 16; ++kk) {
#pragma unroll
            for (int q = 0; q < kZpPer; ++q) acc[q] = fmaf(bv[kk], xw[q - kk + 15], acc[q]);
        }
    }
}

// The F window is fb = 256 * sweeps blocks of 16, one block per thread per sweep, and the
// CTA's outputs are the tb = fb - nbp / 16 blocks whose backward taps it covers, so both
// passes keep every thread busy.  Shared layout (floats): taps[nbp] | reversed taps[nbp] |
// E window (fb + nbp / 16 blocks) | F window (fb blocks).  E block j holds
// E(o0 - nbp + 1 + 16 j + s), F block j holds F(o0 + 16 j + s), o0 = edge + 16 tb blockIdx.x.
__global__ void __launch_bounds__(kZpThreads, 4)
firfilter2_kernel(const float* __restrict__ b, int nb, int nbp, int sweeps, const float* __restrict__ x,
                  int lines, int n, int edge, int padtype, int rounding, float* __restrict__ y)
{
    extern __shared__ __align__(16) float zsm[];
    const int chunks = nbp >> 4;
    const int fb = kZpThreads * sweeps;
    const int tb = fb - chunks;
    float* taps = zsm;
    float* rtaps = zsm + nbp;
    float* es = rtaps + nbp;
    float* fs = es + zp_word(fb + chunks);
    __shared__ float f_last;
    const int hist = nbp - 1;
    const long long ne = (long long)n + 2LL * edge;
    for (int k = threadIdx.x; k < nbp; k += kZpThreads) {
        taps[k] = k < nb ? b[k] : 0.f;
        rtaps[k] = (hist - k) < nb ? b[hist - k] : 0.f;
    }
    for (int line = blockIdx.y; line < lines; line += gridDim.y) {
        const float* xl = x + (size_t)line * n;
        const long long o0 = edge + (long long)blockIdx.x * 16 * tb;
        const int espan = 16 * (fb + chunks);
        for (int j = threadIdx.x; j < espan; j += kZpThreads) {
            const long long i = o0 - hist + j;
            es[zp_word(j >> 4) + (j & 15)] = i < ne ? extended_sample(xl, n, edge, padtype, rounding, i) : 0.f;
        }
        if (threadIdx.x < 32 && o0 + 16LL * fb >= ne) {
            // f[ne - 1], the value the backward pass extends the forward output with (only
            // the CTAs whose F window reaches the end of the line read it)
            float v = 0.f;
            for (int k = threadIdx.x; k < nb; k += 32)
                v = fmaf(b[k], extended_sample(xl, n, edge, padtype, rounding, ne - 1 - k), v);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (threadIdx.x == 0) f_last = v;
        }
        __syncthreads();
        float acc[kZpPer];
        for (int ob = threadIdx.x; ob < fb; ob += kZpThreads) {
            fir16(taps, es, ob, chunks, acc);
            // window positions at or past ne - 1 hold f[ne - 1]
            const long long past = ne - 1 - o0 - 16LL * ob;
            const int first = past < 0 ? 0 : (past > kZpPer ? kZpPer : (int)past);
#pragma unroll
            for (int q = 0; q < kZpPer; ++q) fs[zp_word(ob) + q] = q >= first ? f_last : acc[q];
        }
        __syncthreads();
        float* yl = y + (size_t)line * n;
        for (int ob = threadIdx.x; ob < tb; ob += kZpThreads) {
            fir16(rtaps, fs, ob, chunks, acc);
            const long long m0 = (long long)blockIdx.x * 16 * tb + 16LL * ob;
            if (m0 + kZpPer <= n && (reinterpret_cast<uintptr_t>(yl + m0) & 15) == 0) {
                float4* yp = reinterpret_cast<float4*>(yl + m0);
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    __stcs(&yp[u], make_float4(acc[4 * u], acc[4 * u + 1], acc[4 * u + 2], acc[4 * u + 3]));
            } else {
#pragma unroll
                for (int q = 0; q < kZpPer; ++q)
                    if (m0 + q < n) yl[m0 + q] = acc[q];
            }
        }
        __syncthreads();  // the windows are rebuilt for the next line
    }
}

// ------------------------------------------------ firfilter2 by one convolution
//
// When the padding is at least as long as the filter (edge >= nb; the default padlen is 3 nb),
// neither initial condition reaches an output: every output is
//
//   y[m] = sum_{|d| < nb} c[d] E(edge + m + d),   c[d] = sum_k b[k] b[k - d],
//
// one symmetric convolution of the extended line with the taps' autocorrelation, whose
// spectrum is |FFT(b)|^2.  Overlap-save as for the causal FIR: two lines per complex
// transform (c is real), blocks of N extended samples giving their N - 2 (nb - 1) central
// outputs, the padded samples built on the fly.

// P = (|FFT(b zero-padded)|^2 / N, 0), one CTA.
template <int N>
__global__ void __launch_bounds__(FftPlan<N, elems_for(N)>::T)
autocorr_spectrum_kernel(const float* __restrict__ b, int nb, float2* __restrict__ P,
                         const float2* __restrict__ tw)
{
    using PL = FftPlan<N, elems_for(N)>;
    extern __shared__ float2 hsm[];
    const int t = threadIdx.x;
    float2 v[PL::E];
#pragma unroll
    for (int r = 0; r < PL::E; ++r) {
        const int e = t + PL::T * r;
        v[r] = make_float2(e < nb ? b[e] : 0.f, 0.f);
    }
    fft_block<PL, -1, 1>(v, hsm, t, tw);
    constexpr float inv = 1.0f / (float)N;  // exact: N is a power of two
#pragma unroll
    for (int r = 0; r < PL::E; ++r)
        P[t + PL::T * r] = make_float2(fmaf(v[r].x, v[r].x, v[r].y * v[r].y) * inv, 0.f);
}

// Three CTAs of up to 256 threads per SM, two for the 32-value plans (three would cap them
// at 80 registers and spill), one above 256 threads.
template <int N, int G>
constexpr int zp_fft_min_blocks()
{
    return G * FftPlan<N, elems_for(N)>::T > 256 ? 1 : elems_for(N) >= 32 ? 2 : 3;
}

template <int N, int G>
__global__ void __launch_bounds__(G * FftPlan<N, elems_for(N)>::T, (zp_fft_min_blocks<N, G>()))
firfilter2_fft_kernel(const float* __restrict__ x, int lines, int n, int nb, int edge, int padtype, int rounding,
                      const float2* __restrict__ P, float* __restrict__ y, const float2* __restrict__ tw)
{
    using PL = FftPlan<N, elems_for(N)>;
    extern __shared__ float2 hsm[];
    const int g = threadIdx.x / PL::T;
    const int t = threadIdx.x - g * PL::T;
    float2* smg = hsm + g * PL::smem_elems();
    const int hist = nb - 1;
    const int step = N - 2 * hist;                    // outputs per block
    const long long out0 = ((long long)blockIdx.x * G + g) * step;
    const long long s0 = edge + out0 - hist;          // extended index of the block's first sample
    const long long ne = (long long)n + 2LL * edge;
    const int la = 2 * blockIdx.y, lb = la + 1;
    const bool has_b = lb < lines;
    const bool active = out0 < n;
    const float* xa = x + (size_t)la * n;
    const float* xb = x + (size_t)(has_b ? lb : la) * n;
    float2 v[PL::E];
    if (active && s0 >= edge && s0 + N <= (long long)edge + n) {
        // a block wholly inside the line: extended sample i is x[i - edge], read at
        // constant offsets without the padding logic
        const float* pa = xa + (s0 - edge) + t;
        const float* pb = xb + (s0 - edge) + t;
#pragma unroll
        for (int r = 0; r < PL::E; ++r) {
            const float a = __ldcs(pa + PL::T * r);
            const float b = __ldcs(pb + PL::T * r);
            v[r] = make_float2(a, has_b ? b : 0.f);
        }
    } else {
#pragma unroll
        for (int r = 0; r < PL::E; ++r) {
            const long long i = s0 + t + PL::T * r;
            const bool in = active && i < ne;
            v[r] = make_float2(in ? extended_sample(xa, n, edge, padtype, rounding, i) : 0.f,
                               (in && has_b) ? extended_sample(xb, n, edge, padtype, rounding, i) : 0.f);
        }
    }
    fft_block<PL, -1, 1>(v, smg, t, tw);
#pragma unroll
    for (int r = 0; r < PL::E; ++r) {
        const float p = __ldg(&P[t + PL::T * r]).x;
        v[r] = make_float2(v[r].x * p, v[r].y * p);
    }
    if constexpr (PL::PASSES > 1) __syncthreads();
    fft_block<PL, 1, 1>(v, smg, t, tw);
    if (!active) return;
    float* ya = y + (size_t)la * n;
    float* yb = y + (size_t)lb * n;
    if (out0 + step <= n) {
        // every output of the block exists: store at constant offsets from the first
        float* qa = ya + out0 - hist + t;
        float* qb = yb + out0 - hist + t;
#pragma unroll
        for (int r = 0; r < PL::E; ++r) {
            const int e = t + PL::T * r;
            if (e >= hist && e < hist + step) {
                __stcs(qa + PL::T * r, v[r].x);
                if (has_b) __stcs(qb + PL::T * r, v[r].y);
            }
        }
        return;
    }
#pragma unroll
    for (int r = 0; r < PL::E; ++r) {
        const int e = t + PL::T * r;
        const long long m = out0 + e - hist;
        if (e >= hist && e < hist + step && m < n) {
            __stcs(&ya[m], v[r].x);
            if (has_b) __stcs(&yb[m], v[r].y);
        }
    }
}

template <int N>
int firfilter2_fft_impl(const float* b, int nb, const float* x, int lines, int n, int edge, int padtype,
                        int rounding, float* y, cudaStream_t s)
{
    if (!twiddle_table()) return fail(ZKX_INTERNAL_ERROR, "twiddle table not initialised on this device");
    using PL = FftPlan<N, elems_for(N)>;
    StreamWorkspace ws;
    ws.stream = s;
    ZKX_TRY(stream_workspace((size_t)N * sizeof(float2), s, &ws.ptr));
    float2* P = static_cast<float2*>(ws.ptr);
    const size_t spec_smem = (size_t)PL::smem_elems() * sizeof(float2);
    ZKX_CUDA(cudaFuncSetAttribute(autocorr_spectrum_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)spec_smem));
    autocorr_spectrum_kernel<N><<<1, PL::T, spec_smem, s>>>(b, nb, P, twiddle_table());
    ZKX_LAUNCHED("autocorr_spectrum_kernel");
    constexpr int G = rows_per_cta(N);
    const size_t smem = (size_t)G * PL::smem_elems() * sizeof(float2);
    auto k = firfilter2_fft_kernel<N, G>;
    ZKX_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const long long step = N - 2LL * (nb - 1);
    const long long blocks = (n + step - 1) / step;
    const dim3 grid((unsigned)((blocks + G - 1) / G), (unsigned)((lines + 1) / 2));
    k<<<grid, G * PL::T, smem, s>>>(x, lines, n, nb, edge, padtype, rounding, P, y, twiddle_table());
    ZKX_LAUNCHED("firfilter2_fft_kernel");
    return ZKX_SUCCESS;
}

// ------------------------------------------------------------------ hilbert

// Weight of bin k of an N-point analytic-signal mask (filtering_typed.cpp:1798-1803).
__device__ __forceinline__ float hilbert_weight(int k, int N)
{
    if (k == 0 || ((N & 1) == 0 && k == N / 2)) return 1.f;
    return k < (N + 1) / 2 ? 2.f : 0.f;
}

template <int N, int G>
__global__ void __launch_bounds__(G * FftPlan<N, elems_for(N)>::T)
hilbert_kernel(const float* __restrict__ x, int lines, int n, float2* __restrict__ y,
               const float2* __restrict__ tw)
{
    using PL = FftPlan<N, elems_for(N)>;
    extern __shared__ float2 sm[];
    const int g = threadIdx.x / PL::T;
    const int t = threadIdx.x - g * PL::T;
    const int line = blockIdx.x * G + g;
    const bool active = line < lines;
    float2* smg = sm + g * PL::smem_elems();
    const float* xl = active ? x + (size_t)line * n : nullptr;
    float2 v[PL::E];
#pragma unroll
    for (int r = 0; r < PL::E; ++r) {
        const int e = t + PL::T * r;
        v[r] = make_float2((active && e < n) ? __ldcs(&xl[e]) : 0.f, 0.f);
    }
    fft_block<PL, -1, 1>(v, smg, t, tw);
    constexpr float inv = 1.0f / (float)N;  // exact: N is a power of two
#pragma unroll
    for (int r = 0; r < PL::E; ++r) {
        const float w = hilbert_weight(t + PL::T * r, N) * inv;
        v[r] = make_float2(v[r].x * w, v[r].y * w);
    }
    if constexpr (PL::PASSES > 1) __syncthreads();
    fft_block<PL, 1, 1>(v, smg, t, tw);
    if (active) {
        float2* yl = y + (size_t)line * N;
#pragma unroll
        for (int r = 0; r < PL::E; ++r) __stcs(&yl[t + PL::T * r], v[r]);
    }
}

template <int N>
int hilbert_fused(const float* x, int lines, int n, float2* y, cudaStream_t s)
{
    if (!twiddle_table()) return fail(ZKX_INTERNAL_ERROR, "twiddle table not initialised on this device");
    using PL = FftPlan<N, elems_for(N)>;
    constexpr int G = rows_per_cta(N);
    const size_t smem = (size_t)G * PL::smem_elems() * sizeof(float2);
    auto k = hilbert_kernel<N, G>;
    ZKX_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k<<<(lines + G - 1) / G, G * PL::T, smem, s>>>(x, lines, n, y, twiddle_table());
    ZKX_LAUNCHED("hilbert_kernel");
    return ZKX_SUCCESS;
}

// y[line][k] = (k < n ? x[line][k] : 0) + 0i, rows of N
__global__ void hilbert_pack_kernel(const float* __restrict__ x, int lines, int n, int N, float2* __restrict__ y)
{
    const long long total = (long long)lines * N;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int line = (int)(e / N), k = (int)(e - (long long)line * N);
        y[e] = make_float2(k < n ? x[(size_t)line * n + k] : 0.f, 0.f);
    }
}

__global__ void hilbert_mask_kernel(float2* __restrict__ y, int lines, int N)
{
    const long long total = (long long)lines * N;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const float w = hilbert_weight((int)(e % N), N);
        const float2 v = y[e];
        y[e] = make_float2(v.x * w, v.y * w);
    }
}

unsigned grid_for(long long elems)
{
    const long long b = (elems + 255) / 256;
    return (unsigned)(b < 1 ? 1 : (b < 148LL * 16 ? b : 148LL * 16));
}

}  // namespace

int launch_firfilter2(const float* b, int nb, const float* x, int lines, int n, int edge, int padtype,
                      int rounding, float* y, cudaStream_t stream, int method)
{
    if (nb > kMaxZpTaps) return fail(ZKX_UNSUPPORTED_OPERATION, "firfilter2: more than 4096 coefficients");
    const bool fft_ok = edge >= nb && (lines + 1) / 2 <= 65535;
    if (method == ZKX_FIR_FFT && !fft_ok)
        return fail(ZKX_UNSUPPORTED_OPERATION, "firfilter2: the FFT method needs padlen >= the number of taps");
    if (method == ZKX_FIR_FFT || (method == ZKX_FIR_AUTO && fft_ok && nb >= kZpFftMinTaps)) {
        if (nb <= 1024) return firfilter2_fft_impl<4096>(b, nb, x, lines, n, edge, padtype, rounding, y, stream);
        if (nb <= 2048) return firfilter2_fft_impl<8192>(b, nb, x, lines, n, edge, padtype, rounding, y, stream);
        return firfilter2_fft_impl<16384>(b, nb, x, lines, n, edge, padtype, rounding, y, stream);
    }
    const int nbp = (nb + 15) & ~15;
    const int chunks = nbp / 16;
    const int sweeps = (chunks + 64 + kZpThreads - 1) / kZpThreads;  // at least 64 output blocks per CTA
    const int fb = kZpThreads * sweeps, tb = fb - chunks;
    const size_t smem = (2 * (size_t)nbp + zp_word(fb + chunks) + zp_word(fb)) * sizeof(float);
    ZKX_CUDA(cudaFuncSetAttribute(firfilter2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const long long per_cta = 16LL * tb;
    const dim3 grid((unsigned)((n + per_cta - 1) / per_cta), (unsigned)(lines < 65535 ? lines : 65535));
    firfilter2_kernel<<<grid, kZpThreads, smem, stream>>>(b, nb, nbp, sweeps, x, lines, n, edge, padtype, rounding,
                                                          y);
    ZKX_LAUNCHED("firfilter2_kernel");
    return ZKX_SUCCESS;
}

int launch_hilbert(const float* x, int lines, int n, int nfft, float2* y, cudaStream_t stream)
{
    if (is_pow2(nfft) && nfft <= (1 << kMaxSmemFftLog)) {
        switch (ilog2_host(nfft)) {
        case 0: return hilbert_fused<1>(x, lines, n, y, stream);
        case 1: return hilbert_fused<2>(x, lines, n, y, stream);
        case 2: return hilbert_fused<4>(x, lines, n, y, stream);
        case 3: return hilbert_fused<8>(x, lines, n, y, stream);
        case 4: return hilbert_fused<16>(x, lines, n, y, stream);
        case 5: return hilbert_fused<32>(x, lines, n, y, stream);
        case 6: return hilbert_fused<64>(x, lines, n, y, stream);
        case 7: return hilbert_fused<128>(x, lines, n, y, stream);
        case 8: return hilbert_fused<256>(x, lines, n, y, stream);
        case 9: return hilbert_fused<512>(x, lines, n, y, stream);
        case 10: return hilbert_fused<1024>(x, lines, n, y, stream);
        case 11: return hilbert_fused<2048>(x, lines, n, y, stream);
        case 12: return hilbert_fused<4096>(x, lines, n, y, stream);
        case 13: return hilbert_fused<8192>(x, lines, n, y, stream);
        default: return hilbert_fused<16384>(x, lines, n, y, stream);
        }
    }
    const long long total = (long long)lines * nfft;
    hilbert_pack_kernel<<<grid_for(total), 256, 0, stream>>>(x, lines, n, nfft, y);
    ZKX_LAUNCHED("hilbert_pack_kernel");
    ZKX_TRY(launch_fft_rows(y, lines, nfft, 0, y, stream));
    hilbert_mask_kernel<<<grid_for(total), 256, 0, stream>>>(y, lines, nfft);
    ZKX_LAUNCHED("hilbert_mask_kernel");
    return launch_fft_rows(y, lines, nfft, 1, y, stream);
}

}  // namespace zkx

// ------------------------------------------------------------------ C ABI

using namespace zkx;

extern "C" int zkx_firfilter2_f32(const float* b, int nb, const float* x, int lines, int n, int padtype,
                                  int has_padlen, int padlen, int pad_rounding, float* y, zkx_stream_t stream)
{
    return zkx_firfilter2_ex_f32(b, nb, x, lines, n, padtype, has_padlen, padlen, pad_rounding, y, ZKX_FIR_AUTO,
                                 stream);
}

extern "C" int zkx_firfilter2_ex_f32(const float* b, int nb, const float* x, int lines, int n, int padtype,
                                     int has_padlen, int padlen, int pad_rounding, float* y, int method,
                                     zkx_stream_t stream)
{
    // filtering_typed.cpp:1226-1302
    if (method < ZKX_FIR_AUTO || method > ZKX_FIR_FFT) return fail(ZKX_INVALID_ARGUMENT, "firfilter2: unknown method");
    if (nb < 1) return fail(ZKX_INVALID_ARGUMENT, "firfilter2 coefficients");
    if (padtype < ZKX_PAD_ODD || padtype > ZKX_PAD_NONE) return fail(ZKX_INVALID_ARGUMENT, "firfilter2 padtype");
    if (pad_rounding < ZKX_PAD_ROUND_F32 || pad_rounding > ZKX_PAD_ROUND_I32)
        return fail(ZKX_INVALID_ARGUMENT, "firfilter2 pad rounding");
    if (lines < 0 || n < 1 || (long long)lines * n > INT_MAX) return fail(ZKX_INVALID_SHAPE, "firfilter2 input shape");
    long long requested = 0;
    if (padtype != ZKX_PAD_NONE) requested = has_padlen ? (long long)padlen : 3LL * nb;
    if (n <= requested) return fail(ZKX_INVALID_SHAPE, "firfilter2 input axis must exceed padlen");
    const long long edge = requested > 0 ? requested : 0;
    if ((long long)lines * (n + 2 * edge) > INT_MAX)
        return fail(ZKX_INVALID_SHAPE, "firfilter2 extended input exceeds int indexing");
    if (!b || !x || !y) return fail(ZKX_INVALID_ARGUMENT, "firfilter2: null pointer");
    if (lines == 0) return ZKX_SUCCESS;
    ZKX_TRY(ensure_device_ready());
    return launch_firfilter2(b, nb, x, lines, n, (int)edge, padtype, pad_rounding, y, stream, method);
}

extern "C" int zkx_hilbert_f32(const float* x, int lines, int n, int nfft, void* y, zkx_stream_t stream)
{
    // filtering_typed.cpp:500-562
    if (nfft == -1) nfft = n;
    if (lines < 0 || n < 0) return fail(ZKX_INVALID_SHAPE, "hilbert input shape");
    if (nfft < 1) return fail(ZKX_INVALID_ARGUMENT, "hilbert N must be positive");
    if ((long long)lines * nfft > INT_MAX || (long long)lines * n > INT_MAX)
        return fail(ZKX_INVALID_SHAPE, "hilbert output exceeds int indexing");
    if (nfft > (1 << 16) || (!is_pow2(nfft) && nfft > kMaxBluesteinLength))
        return fail(ZKX_UNSUPPORTED_OPERATION, "hilbert: N must be at most 32768, or a power of two up to 65536");
    if ((n > 0 && !x) || !y) return fail(ZKX_INVALID_ARGUMENT, "hilbert: null pointer");
    if (lines == 0) return ZKX_SUCCESS;
    ZKX_TRY(ensure_device_ready());
    return launch_hilbert(x, lines, n, nfft, static_cast<float2*>(y), stream);
}
