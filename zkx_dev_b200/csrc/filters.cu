// Front-end filters for sm_100a: causal FIR (firfilter) and polyphase
// upfirdn / resample_poly, both along the last axis of row-major [lines, n] data.
//
// FIR: a CTA computes 4096 outputs of one line with 256 threads x 16 consecutive
// outputs.  The input block plus its (nb - 1)-sample history and the taps are
// staged in shared memory; every thread keeps a 16-value sliding window of inputs
// in registers, so each tap costs one shared load, one broadcast tap load and 16
// FMAs.  The staged input is skewed (one pad word per 16) so the 32 threads of a
// warp, whose windows start 16 samples apart, read 32 different banks.
// Algorithmic traffic: 4 B in + 4 B out per sample; 2*nb FLOP per sample.
//
// Polyphase: output m uses phase ph = (m*down + offset) mod up and the taps
// h[ph], h[ph+up], ... against x[q], x[q-1], ... with q = floor((m*down+offset)/up),
// the reference's causal zero-extended definition (filtering_typed.cpp:2585-2612,
// 2656-2684) without visiting the taps of other phases.  Taps are regrouped per
// phase in shared memory; the input span of the CTA's outputs is staged once.
#include "fft_core.cuh"
#include "zkx_internal.h"

namespace zkx {
namespace {

constexpr int kFirThreads = 256;
constexpr int kFirPerThread = 16;
constexpr int kFirBlock = kFirThreads * kFirPerThread;  // outputs per CTA

__host__ __device__ __forceinline__ int fir_skew(int j) { return j + (j >> 4); }

__global__ void __launch_bounds__(kFirThreads)
fir_kernel(const float* __restrict__ b, int nb, const float* __restrict__ x, int n,
           const float* __restrict__ zi, float* __restrict__ y)
{
    extern __shared__ float sm[];
    float* taps = sm;                       // nb
    float* xs = sm + ((nb + 3) & ~3);       // skewed input, kFirBlock + nb - 1 samples
    const int line = blockIdx.y;
    const long long n0 = (long long)blockIdx.x * kFirBlock;
    const float* xl = x + (size_t)line * n;
    const int hist = nb - 1;
    for (int k = threadIdx.x; k < nb; k += kFirThreads) taps[k] = b[k];
    const int span = kFirBlock + hist;
    for (int j = threadIdx.x; j < span; j += kFirThreads) {
        const long long src = n0 - hist + j;
        xs[fir_skew(j)] = (src >= 0 && src < n) ? __ldcs(&xl[src]) : 0.f;
    }
    __syncthreads();

    // outputs n0 + o + q, q < 16, with o = 16 * tid; x[i - k] sits at xs[i - n0 + hist - k]
    const int o = threadIdx.x * kFirPerThread;
    float acc[kFirPerThread];
    float win[kFirPerThread];
#pragma unroll
    for (int q = 0; q < kFirPerThread; ++q) {
        acc[q] = 0.f;
        win[q] = xs[fir_skew(o + hist + q)];
    }
    // win[q] = x[n0 + o + q - k] at step k; unrolling by 16 turns the shifts into
    // register renames
#pragma unroll 16
    for (int k = 0; k < nb; ++k) {
        const float bk = taps[k];
#pragma unroll
        for (int q = 0; q < kFirPerThread; ++q) acc[q] = fmaf(bk, win[q], acc[q]);
#pragma unroll
        for (int q = kFirPerThread - 1; q > 0; --q) win[q] = win[q - 1];
        const int j = o + hist - k - 1;
        win[0] = j >= 0 ? xs[fir_skew(j)] : 0.f;
    }
    float* yl = y + (size_t)line * n;
#pragma unroll
    for (int q = 0; q < kFirPerThread; ++q) {
        const long long i = n0 + o + q;
        if (i < n) {
            float v = acc[q];
            if (zi && i < hist) v += zi[(size_t)line * hist + i];
            __stcs(&yl[i], v);
        }
    }
}

// Final state: zf[j] = sum_k b[k] x[n + j - k] (valid terms) + zi[n + j] when n + j < nb - 1
// (filtering_typed.cpp:1560-1588 evaluates the full convolution at n + j).
__global__ void fir_state_kernel(const float* __restrict__ b, int nb, const float* __restrict__ x,
                                 int n, const float* __restrict__ zi, float* __restrict__ zf,
                                 int lines)
{
    const int hist = nb - 1;
    const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= (long long)lines * hist) return;
    const int line = (int)(id / hist), j = (int)(id % hist);
    const long long full = (long long)n + j;
    float v = 0.f;
    for (int k = 0; k < nb; ++k) {
        const long long s = full - k;
        if (s >= 0 && s < n) v = fmaf(b[k], x[(size_t)line * n + s], v);
    }
    if (zi && full < hist) v += zi[(size_t)line * hist + full];
    zf[(size_t)line * hist + j] = v;
}

__device__ __forceinline__ long long floor_div(long long a, long long b)
{
    long long q = a / b;
    if ((a % b != 0) && ((a < 0) != (b < 0))) --q;
    return q;
}

constexpr int kPolyThreads = 256;

__global__ void __launch_bounds__(kPolyThreads)
polyphase_kernel(const float* __restrict__ h, int nh, int up, int down, long long offset,
                 const float* __restrict__ x, int n, float* __restrict__ y, int nout, int block,
                 int jmax, int span_cap)
{
    extern __shared__ float sm[];
    float* hp = sm;                               // [up][jmax] phase-major taps
    float* xs = sm + ((up * jmax + 3) & ~3);      // input span
    const int line = blockIdx.y;
    const long long m0 = (long long)blockIdx.x * block;
    const long long mlast = m0 + block - 1 < nout - 1 ? m0 + block - 1 : nout - 1;
    const long long qlo = floor_div(m0 * down + offset, up) - (jmax - 1);
    const long long qhi = floor_div(mlast * down + offset, up);
    const int span = (int)(qhi - qlo + 1);
    const float* xl = x + (size_t)line * n;
    for (int i = threadIdx.x; i < up * jmax; i += kPolyThreads) {
        const int ph = i / jmax, j = i % jmax;
        const int k = ph + j * up;
        hp[i] = k < nh ? h[k] : 0.f;
    }
    for (int i = threadIdx.x; i < span && i < span_cap; i += kPolyThreads) {
        const long long s = qlo + i;
        xs[i] = (s >= 0 && s < n) ? __ldcs(&xl[s]) : 0.f;
    }
    __syncthreads();
    float* yl = y + (size_t)line * nout;
    for (long long m = m0 + threadIdx.x; m <= mlast; m += kPolyThreads) {
        const long long tt = m * down + offset;
        const long long q = floor_div(tt, up);
        const int ph = (int)(tt - q * up);
        const float* hrow = hp + ph * jmax;
        const int base = (int)(q - qlo);
        float acc = 0.f;
        for (int j = 0; j < jmax; ++j) acc = fmaf(hrow[j], xs[base - j], acc);
        __stcs(&yl[m], acc);
    }
}

}  // namespace

int launch_fir(const float* b, int nb, const float* x, int lines, int n, const float* zi,
               float* y, float* zf, cudaStream_t stream)
{
    if (lines > 65535) return fail(ZKX_UNSUPPORTED_OPERATION, "firfilter: more than 65535 lines");
    const int span = kFirBlock + nb - 1;
    const size_t smem = ((size_t)((nb + 3) & ~3) + (size_t)fir_skew(span) + 1) * sizeof(float);
    if (smem > 200 * 1024) return fail(ZKX_UNSUPPORTED_OPERATION, "firfilter: too many taps for the shared-memory kernel");
    ZKX_CUDA(cudaFuncSetAttribute(fir_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dim3 grid((unsigned)((n + kFirBlock - 1) / kFirBlock), (unsigned)lines);
    fir_kernel<<<grid, kFirThreads, smem, stream>>>(b, nb, x, n, zi, y);
    ZKX_LAUNCHED("fir_kernel");
    if (zf && nb > 1) {
        const long long total = (long long)lines * (nb - 1);
        fir_state_kernel<<<(unsigned)((total + 255) / 256), 256, 0, stream>>>(b, nb, x, n, zi, zf, lines);
        ZKX_LAUNCHED("fir_state_kernel");
    }
    return ZKX_SUCCESS;
}

int launch_polyphase(const float* taps, int ntaps, int up, int down, long long offset,
                     const float* x, int lines, int n, float* y, int nout, cudaStream_t stream)
{
    if (nout <= 0 || lines <= 0) return ZKX_SUCCESS;
    if (lines > 65535) return fail(ZKX_UNSUPPORTED_OPERATION, "upfirdn: more than 65535 lines");
    const int jmax = (ntaps + up - 1) / up;
    // outputs per CTA: keep the staged input span within 12K samples
    long long block = 2048;
    while (block > kPolyThreads && (block * down) / up + jmax + 2 > 12288) block /= 2;
    const int span_cap = (int)((block * down) / up + jmax + 2);
    const size_t smem = ((size_t)((up * jmax + 3) & ~3) + (size_t)span_cap) * sizeof(float);
    if (smem > 200 * 1024) return fail(ZKX_UNSUPPORTED_OPERATION, "upfirdn: filter too long for the shared-memory kernel");
    ZKX_CUDA(cudaFuncSetAttribute(polyphase_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dim3 grid((unsigned)((nout + block - 1) / block), (unsigned)lines);
    polyphase_kernel<<<grid, kPolyThreads, smem, stream>>>(taps, ntaps, up, down, offset, x, n, y,
                                                           nout, (int)block, jmax, span_cap);
    ZKX_LAUNCHED("polyphase_kernel");
    return ZKX_SUCCESS;
}

}  // namespace zkx
