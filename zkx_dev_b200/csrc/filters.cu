// Front-end filters for sm_100a: causal FIR (firfilter) and polyphase
// upfirdn / resample_poly, both along the last axis of row-major [lines, n] data.
//
// FIR: a CTA computes 4096 outputs of one line with 256 threads x 16 consecutive
// outputs.  The input block plus its history and the taps (zero-padded to a multiple
// of 16) are staged in shared memory.  Per 16-tap chunk a thread loads the 16 taps
// (4 broadcast 128-bit loads) and the 31 input samples its outputs touch (8 128-bit
// loads) and performs 256 register FMAs: about 1.05 instructions per multiply-add.
// Algorithmic traffic: 4 B in + 4 B out per sample; 2*nb FLOP per sample.
//
// Polyphase: output m uses phase ph = (m*down + offset) mod up and the taps
// h[ph], h[ph+up], ... against x[q], x[q-1], ... with q = floor((m*down+offset)/up),
// the reference's causal zero-extended definition (filtering_typed.cpp:2585-2612,
// 2656-2684) without visiting the taps of other phases.  Taps are regrouped per
// phase in shared memory; the input span of the CTA's outputs is staged once.
#include "fft_core.cuh"
#include "tma.cuh"
#include "zkx_internal.h"

namespace zkx {
namespace {

constexpr int kFirThreads = 256;
// From this many taps the overlap-save FFT path (firfft.cu) beats the direct sums: on
// 16 x 2^20 samples 15 taps take 48.0 us direct and 49.4 us by FFT, 31 taps 55.2 and 49.5,
// 63 taps 70.4 and 51.4, 127 taps 106.4 and 51.4 (the FFT path stays within 48-72 us up
// to 511 taps).
constexpr int kFirFftMinTaps = 20;
constexpr int kFirPerThread = 16;
constexpr int kFirBlock = kFirThreads * kFirPerThread;  // outputs per CTA

// Shared layout of the staged input: samples in 16-sample blocks, block b at word 20*b
// (4 pad words per block), so the 128-bit loads of 8 threads whose windows start 16
// samples apart land on 32 distinct banks.
__host__ __device__ __forceinline__ int fir_block_word(int b) { return 20 * b; }

// y[n0 + o + q] = sum_{k < nbp} b[k] x[n0 + o + q - k], o = 16*tid, q < 16, with the taps
// zero-padded to nbp (a multiple of 16).  Relative sample index j = i - n0 + nbp - 1; for
// tap chunk c the 31 samples a thread needs are blocks tid + nbp/16 - 1 - c and the next.
__global__ void __launch_bounds__(kFirThreads)
fir_kernel(const float* __restrict__ b, int nb, int nbp, const float* __restrict__ x, int n,
           const float* __restrict__ zi, float* __restrict__ y)
{
    extern __shared__ __align__(16) float sm[];
    float* taps = sm;                        // nbp
    float* xs = sm + nbp;                    // skewed blocks
    const int line = blockIdx.y;
    const long long n0 = (long long)blockIdx.x * kFirBlock;
    const float* xl = x + (size_t)line * n;
    const int hist = nbp - 1;
    for (int k = threadIdx.x; k < nbp; k += kFirThreads) taps[k] = k < nb ? b[k] : 0.f;
    const int span = kFirBlock + hist;       // samples n0 - hist .. n0 + kFirBlock - 1
    // 8 loads in flight per thread before their shared stores
    for (int j0 = 0; j0 < span; j0 += 8 * kFirThreads) {
        float tmp[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int j = j0 + u * kFirThreads + threadIdx.x;
            const long long src = n0 - hist + j;
            tmp[u] = (j < span && src >= 0 && src < n) ? __ldcs(&xl[src]) : 0.f;
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int j = j0 + u * kFirThreads + threadIdx.x;
            if (j < span) xs[fir_block_word(j >> 4) + (j & 15)] = tmp[u];
        }
    }
    __syncthreads();

    float acc[kFirPerThread];
#pragma unroll
    for (int q = 0; q < kFirPerThread; ++q) acc[q] = 0.f;
    const int chunks = nbp >> 4;
    for (int c = 0; c < chunks; ++c) {
        float bv[16];
        const float4* tp = reinterpret_cast<const float4*>(taps + 16 * c);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const float4 t4 = tp[u];
            bv[4 * u] = t4.x; bv[4 * u + 1] = t4.y; bv[4 * u + 2] = t4.z; bv[4 * u + 3] = t4.w;
        }
        const int blk = threadIdx.x + chunks - 1 - c;
        float xw[32];
        const float4* w0 = reinterpret_cast<const float4*>(xs + fir_block_word(blk));
        const float4* w1 = reinterpret_cast<const float4*>(xs + fir_block_word(blk + 1));
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const float4 a = w0[u], d = w1[u];
            xw[4 * u] = a.x; xw[4 * u + 1] = a.y; xw[4 * u + 2] = a.z; xw[4 * u + 3] = a.w;
            xw[16 + 4 * u] = d.x; xw[17 + 4 * u] = d.y; xw[18 + 4 * u] = d.z; xw[19 + 4 * u] = d.w;
        }
        // tap 16c + kk on output q reads window position q - kk + 15
#pragma unroll
        for (int kk = 0; kk < 16; ++kk) {
#pragma unroll
            for (int q = 0; q < kFirPerThread; ++q) acc[q] = fmaf(bv[kk], xw[q - kk + 15], acc[q]);
        }
    }
    float* yl = y + (size_t)line * n;
    const int zhist = nb - 1;
    const long long ob = n0 + threadIdx.x * kFirPerThread;
    if (ob + kFirPerThread <= n && !(zi && ob < zhist) &&
        ((reinterpret_cast<uintptr_t>(yl + ob) & 15) == 0)) {
        float4* yp = reinterpret_cast<float4*>(yl + ob);
#pragma unroll
        for (int u = 0; u < 4; ++u)
            yp[u] = make_float4(acc[4 * u], acc[4 * u + 1], acc[4 * u + 2], acc[4 * u + 3]);
    } else {
#pragma unroll
        for (int q = 0; q < kFirPerThread; ++q) {
            const long long i = ob + q;
            if (i < n) {
                float v = acc[q];
                if (zi && i < zhist) v += zi[(size_t)line * zhist + i];
                yl[i] = v;
            }
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

// Generic polyphase kernel: each thread walks Q consecutive outputs, tracking the
// phase and input index incrementally in 32-bit arithmetic (one division per thread).
template <int Q>
__global__ void __launch_bounds__(kPolyThreads)
polyphase_kernel(const float* __restrict__ h, int nh, int up, int down, long long offset,
                 const float* __restrict__ x, int n, float* __restrict__ y, int nout, int jmax,
                 int span_cap)
{
    extern __shared__ float sm[];
    float* hp = sm;                               // [up][jmax] phase-major taps
    float* xs = sm + ((up * jmax + 3) & ~3);      // input span
    constexpr int block = kPolyThreads * Q;
    const int line = blockIdx.y;
    const long long m0 = (long long)blockIdx.x * block;
    const long long base = m0 * down + offset;    // filter time of the CTA's first output
    const long long qb = floor_div(base, up);
    const int rb = (int)(base - qb * up);
    const long long qlo = qb - (jmax - 1);
    const float* xl = x + (size_t)line * n;
    for (int i = threadIdx.x; i < up * jmax; i += kPolyThreads) {
        const int ph = i / jmax, j = i - ph * jmax;
        const int k = ph + j * up;
        hp[i] = k < nh ? h[k] : 0.f;
    }
    for (int i0 = 0; i0 < span_cap; i0 += 8 * kPolyThreads) {
        float tmp[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int i = i0 + u * kPolyThreads + threadIdx.x;
            const long long s = qlo + i;
            tmp[u] = (i < span_cap && s >= 0 && s < n) ? __ldcs(&xl[s]) : 0.f;
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int i = i0 + u * kPolyThreads + threadIdx.x;
            if (i < span_cap) xs[i] = tmp[u];
        }
    }
    __syncthreads();
    // first output of this thread: d = tid * Q, filter time rb + d * down (32-bit)
    const int d0 = threadIdx.x * Q;
    const int t0 = rb + d0 * down;
    int q = t0 / up + (jmax - 1);                 // index into xs of the newest sample
    int ph = t0 - (t0 / up) * up;
    const int dq = down / up, dr = down - dq * up;
    float* yl = y + (size_t)line * nout;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const long long m = m0 + d0 + i;
        if (m < nout) {
            const float* hrow = hp + ph * jmax;
            float acc = 0.f;
            for (int j = 0; j < jmax; ++j) acc = fmaf(hrow[j], xs[q - j], acc);
            __stcs(&yl[m], acc);
        }
        ph += dr;
        q += dq;
        if (ph >= up) {
            ph -= up;
            ++q;
        }
    }
}

// Register-blocked polyphase for fixed (UP, DOWN, J): thread (g, r) computes the Q
// outputs m = m0 + g*UP*Q + r + UP*i, which share one phase, so its J taps and the
// J + DOWN*(Q-1) input samples they touch are read from shared memory once each (each
// sample is reused by up to J/DOWN outputs).  G groups of UP threads with G*UP*Q a
// multiple of 4, so a CTA's outputs start on a 16-byte boundary of an aligned row.
// The input span arrives as one bulk copy (from the 4-sample boundary at or below its
// first sample) wherever it lies inside the line and the line is 16-byte aligned;
// spans that reach past either end are gathered with zero fill.  Outputs are staged
// in shared memory and stored as 128-bit words.
template <int UP, int Q>
constexpr int poly_groups()
{
    int g = kPolyThreads / UP;
    while ((g * UP * Q) % 4 != 0) --g;
    return g;
}

template <int UP, int DOWN, int J, int Q>
struct PolyBlockGeom {
    static constexpr int NT = poly_groups<UP, Q>() * UP;
    static constexpr int BLOCK = NT * Q;                         // outputs per CTA
    static constexpr int HW = (UP * J + 3) & ~3;                 // phase-major taps
    // samples from floor(qlo) needed by the CTA: newest index (rb + (BLOCK-1)*DOWN)/UP
    // + J - 1 relative to qlo, plus up to 3 of alignment, rounded to 4
    static constexpr int SPAN = ((BLOCK * DOWN) / UP + J + 2 + 3 + 3) & ~3;
    static constexpr size_t smem_bytes() { return (size_t)(4 + HW + BLOCK + SPAN) * sizeof(float); }
};

template <int UP, int DOWN, int J, int Q>
__global__ void __launch_bounds__(PolyBlockGeom<UP, DOWN, J, Q>::NT)
polyphase_blocked_kernel(const float* __restrict__ h, int nh, long long offset,
                         const float* __restrict__ x, int n, float* __restrict__ y, int nout,
                         int aligned, int* err)
{
    using PG = PolyBlockGeom<UP, DOWN, J, Q>;
    constexpr int NT = PG::NT, BLOCK = PG::BLOCK, SPAN = PG::SPAN;
    extern __shared__ __align__(16) float sm[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm);
    float* hp = sm + 4;                          // [UP][J]
    float* ys = hp + PG::HW;                     // BLOCK staged outputs
    float* xs = ys + BLOCK;                      // xs[k] = sample qa + k
    const int line = blockIdx.y;
    const long long m0 = (long long)blockIdx.x * BLOCK;
    const long long base = m0 * DOWN + offset;
    const long long qb = floor_div(base, UP);
    const int rb = (int)(base - qb * UP);
    const long long qlo = qb - (J - 1);
    const long long qa = qlo & ~3LL;             // 4-sample boundary at or below qlo
    const int shift = (int)(qlo - qa);
    const float* xl = x + (size_t)line * n;
    const bool bulk = (aligned & 1) && qa >= 0 && qa + SPAN <= n;
    if (bulk && threadIdx.x == 0) {
        mbar_init(bar, 1);
        mbar_arrive_expect_tx(bar, (uint32_t)(SPAN * sizeof(float)));
        bulk_load_1d(xs, xl + qa, (uint32_t)(SPAN * sizeof(float)), bar);
    }
    for (int i = threadIdx.x; i < UP * J; i += NT) {
        const int ph = i / J, j = i - ph * J;
        const int k = ph + j * UP;
        hp[i] = k < nh ? h[k] : 0.f;
    }
    if (!bulk) {
        for (int i0 = 0; i0 < SPAN; i0 += 8 * NT) {
            float tmp[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int i = i0 + u * NT + threadIdx.x;
                const long long s = qa + i;
                tmp[u] = (i < SPAN && s >= 0 && s < n) ? __ldcs(&xl[s]) : 0.f;
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int i = i0 + u * NT + threadIdx.x;
                if (i < SPAN) xs[i] = tmp[u];
            }
        }
    }
    __syncthreads();
    if (bulk) {
        const bool ok = mbar_wait_bounded(bar, 0);
        if (__syncthreads_or(!ok)) {
            if (threadIdx.x == 0) atomicCAS(err, 0, (int)kKernelTmaTimeout);
            return;
        }
    }
    const int g = threadIdx.x / UP, r = threadIdx.x - (threadIdx.x / UP) * UP;
    const int d0 = g * UP * Q + r;
    const int t0 = rb + d0 * DOWN;
    const int q0 = t0 / UP;                      // newest sample of output 0, relative to qb
    const int ph = t0 - q0 * UP;
    float hreg[J];
#pragma unroll
    for (int j = 0; j < J; ++j) hreg[j] = hp[ph * J + j];
    constexpr int W = J + DOWN * (Q - 1);
    float xw[W];                                 // xw[w] = sample qb + q0 - (J-1) + w
#pragma unroll
    for (int w = 0; w < W; ++w) xw[w] = xs[shift + q0 + w];
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        float acc = 0.f;
#pragma unroll
        for (int j = 0; j < J; ++j) acc = fmaf(hreg[j], xw[J - 1 + DOWN * i - j], acc);
        ys[d0 + UP * i] = acc;
    }
    __syncthreads();
    float* yl = y + (size_t)line * nout;
    if ((aligned & 2) && m0 + BLOCK <= nout) {
        float4* yp = reinterpret_cast<float4*>(yl + m0);
        const float4* ysp = reinterpret_cast<const float4*>(ys);
        for (int i = threadIdx.x; i < BLOCK / 4; i += NT) __stcs(&yp[i], ysp[i]);
    } else {
        for (int i = threadIdx.x; i < BLOCK; i += NT) {
            const long long m = m0 + i;
            if (m < nout) __stcs(&yl[m], ys[i]);
        }
    }
}

template <int UP, int DOWN, int J, int Q>
int polyphase_blocked_launch(const float* taps, int ntaps, long long offset, const float* x,
                             int lines, int n, float* y, int nout, cudaStream_t stream)
{
    using PG = PolyBlockGeom<UP, DOWN, J, Q>;
    const size_t smem = PG::smem_bytes();
    const int aligned = (((n & 3) == 0 && (reinterpret_cast<uintptr_t>(x) & 15) == 0) ? 1 : 0) |
                        (((nout & 3) == 0 && (reinterpret_cast<uintptr_t>(y) & 15) == 0) ? 2 : 0);
    auto k = polyphase_blocked_kernel<UP, DOWN, J, Q>;
    ZKX_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dim3 grid((unsigned)((nout + PG::BLOCK - 1) / PG::BLOCK), (unsigned)lines);
    k<<<grid, PG::NT, smem, stream>>>(taps, ntaps, offset, x, n, y, nout, aligned, kernel_error_word());
    ZKX_LAUNCHED("polyphase_blocked_kernel");
    return ZKX_SUCCESS;
}

}  // namespace

int launch_fir(const float* b, int nb, const float* x, int lines, int n, const float* zi,
               float* y, float* zf, cudaStream_t stream, int method)
{
    if (method == ZKX_FIR_FFT || (method == ZKX_FIR_AUTO && nb >= kFirFftMinTaps && nb <= 4096)) {
        ZKX_TRY(launch_fir_fft(b, nb, x, lines, n, zi, y, stream));
        if (zf && nb > 1) {
            const long long total = (long long)lines * (nb - 1);
            fir_state_kernel<<<(unsigned)((total + 255) / 256), 256, 0, stream>>>(b, nb, x, n, zi, zf, lines);
            ZKX_LAUNCHED("fir_state_kernel");
        }
        return ZKX_SUCCESS;
    }
    if (lines > 65535) return fail(ZKX_UNSUPPORTED_OPERATION, "firfilter: more than 65535 lines");
    const int nbp = (nb + 15) & ~15;
    const int span = kFirBlock + nbp - 1;
    const size_t smem = ((size_t)nbp + (size_t)fir_block_word((span + 15) >> 4)) * sizeof(float);
    if (smem > 200 * 1024) return fail(ZKX_UNSUPPORTED_OPERATION, "firfilter: too many taps for the shared-memory kernel");
    ZKX_CUDA(cudaFuncSetAttribute(fir_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dim3 grid((unsigned)((n + kFirBlock - 1) / kFirBlock), (unsigned)lines);
    fir_kernel<<<grid, kFirThreads, smem, stream>>>(b, nb, nbp, x, n, zi, y);
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
    // register-blocked kernels for the common rational factors with designed filters
    if (up == 3 && down == 2 && jmax == 21) return polyphase_blocked_launch<3, 2, 21, 7>(taps, ntaps, offset, x, lines, n, y, nout, stream);
    if (up == 2 && down == 1 && jmax == 21) return polyphase_blocked_launch<2, 1, 21, 8>(taps, ntaps, offset, x, lines, n, y, nout, stream);
    if (up == 2 && down == 3 && jmax == 31) return polyphase_blocked_launch<2, 3, 31, 5>(taps, ntaps, offset, x, lines, n, y, nout, stream);
    if (up == 1 && down == 2 && jmax == 41) return polyphase_blocked_launch<1, 2, 41, 4>(taps, ntaps, offset, x, lines, n, y, nout, stream);
    constexpr int Q = 8;
    constexpr long long block = (long long)kPolyThreads * Q;
    // span: floor((block-1)*down/up) + 1 + jmax samples, plus slack for the remainder
    const long long span_ll = (block * down) / up + jmax + 2;
    if (up > 4096 || down > 4096 || span_ll > 48 * 1024)
        return fail(ZKX_UNSUPPORTED_OPERATION, "upfirdn: factors too large for the shared-memory kernel");
    const int span_cap = (int)span_ll;
    const size_t smem = ((size_t)((up * jmax + 3) & ~3) + (size_t)span_cap) * sizeof(float);
    if (smem > 200 * 1024) return fail(ZKX_UNSUPPORTED_OPERATION, "upfirdn: filter too long for the shared-memory kernel");
    ZKX_CUDA(cudaFuncSetAttribute(polyphase_kernel<Q>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dim3 grid((unsigned)((nout + block - 1) / block), (unsigned)lines);
    polyphase_kernel<Q><<<grid, kPolyThreads, smem, stream>>>(taps, ntaps, up, down, offset, x, n, y,
                                                             nout, jmax, span_cap);
    ZKX_LAUNCHED("polyphase_kernel");
    return ZKX_SUCCESS;
}

}  // namespace zkx
