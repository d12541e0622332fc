// Range compression (fused FFT x conj(replica spectrum) x IFFT per pulse) and the
// Doppler transform (windowed FFT across pulses, optional |.|^2) for sm_100a.
//
// Layout in HBM: a CPI is row-major [pulses, range samples] complex64; the
// compressed cube keeps that layout ([pulses, range_nfft]); the range-Doppler map
// and power are [doppler_nfft, range_nfft] (Doppler bin major), the reference's
// output layout (radartools_typed.cu:241-243).
//
// Range compression reads each pulse once and writes it once: 16 B per cell of
// compulsory HBM traffic.  The Doppler kernel reads the compressed cube once and
// writes the map (8 B) and the power (4 B): 20 B per cell.
#include <algorithm>

#include "fft_core.cuh"
#include "fft_local.cuh"
#include "rows.cuh"
#include "tcgen05.cuh"
#include "tma.cuh"
#include "window.cuh"
#include "zkx_internal.h"

namespace zkx {
namespace {

// ------------------------------------------------------------ replica spectrum

// spectrum[k] = conj(FFT(w h / ||w h||, N))[k] / N; one CTA.  The norm runs over all
// `length` template samples (radartools_typed.cpp:639-648) in FP64.
template <int N>
__global__ void __launch_bounds__(FftPlan<N, elems_for(N)>::T)
replica_spectrum_kernel(const float2* __restrict__ h, int length, int normalize, int window_kind,
                        const float* __restrict__ explicit_window, float2* __restrict__ spectrum,
                        const float2* __restrict__ tw)
{
    using PL = FftPlan<N, elems_for(N)>;
    extern __shared__ float2 sm[];
    __shared__ double partial[PL::T];
    const int t = threadIdx.x;
    double acc = 0.0;
    for (int i = t; i < length; i += PL::T) {
        const double w = window_value(window_kind, explicit_window, i, length);
        const float2 v = h[i];
        const double re = (double)v.x * w, im = (double)v.y * w;
        acc += re * re + im * im;
    }
    partial[t] = acc;
    __syncthreads();
    if (t == 0) {
        double total = 0.0;
        for (int i = 0; i < PL::T; ++i) total += partial[i];
        partial[0] = total;
    }
    __syncthreads();
    const double norm = normalize ? sqrt(partial[0]) : 1.0;
    const float scale = (float)(1.0 / (norm * (double)N));
    float2 v[PL::E];
#pragma unroll
    for (int r = 0; r < PL::E; ++r) {
        const int e = t + PL::T * r;
        float2 x = make_float2(0.f, 0.f);
        if (e < length) {
            const float w = window_value(window_kind, explicit_window, e, length);
            const float2 hv = h[e];
            x = make_float2(hv.x * w, hv.y * w);
        }
        v[r] = x;
    }
    fft_block<PL, -1, 1>(v, sm, t, tw);
#pragma unroll
    for (int r = 0; r < PL::E; ++r) {
        const float2 s = v[r];
        spectrum[t + PL::T * r] = make_float2(s.x * scale, -s.y * scale);
    }
}

// ------------------------------------------------------------ range compression

// Range compression lengths with a persistent kernel (N >= 4096) and a three-pass plan
// read the second-pass twiddles from a shared table in both compression kernels.
template <int N>
constexpr bool compression_mid_table()
{
    return N >= 4096 && mid_table_elems<FftPlan<N, elems_for(N)>>() > 0;
}

// G pulses per CTA; each pulse: load (zero-pad/truncate to N), forward FFT, multiply
// by the replica spectrum, inverse FFT, store.  The cube crosses HBM once each way.
template <int N, int G, class Src>
__global__ void __launch_bounds__(G * FftPlan<N, elems_for(N)>::T)
pulse_compression_kernel(const Src src, int pulses, int samples,
                         const float2* __restrict__ spectrum, float2* __restrict__ y,
                         const float2* __restrict__ tw)
{
    using PL = FftPlan<N, elems_for(N)>;
    extern __shared__ float2 sm[];
    const int g = threadIdx.x / PL::T;
    const int t = threadIdx.x - g * PL::T;
    const int pulse = blockIdx.x * G + g;
    const bool active = pulse < pulses;
    float2* smg = sm + g * PL::smem_elems();
    // lengths that also have the persistent kernel take its second-pass twiddle table,
    // so both kernels round identically and the tuning choice never changes a result
    float2* mid = compression_mid_table<N>() ? sm + G * PL::smem_elems() : nullptr;
    if (mid) fill_mid_table<PL>(mid, threadIdx.x, G * PL::T, tw);
    const float2* xr = active ? src.row(pulse) : nullptr;
    float2 v[PL::E];
#pragma unroll
    for (int r = 0; r < PL::E; ++r) {
        const int e = t + PL::T * r;
        v[r] = (active && e < samples) ? __ldcs(&xr[e]) : make_float2(0.f, 0.f);
    }
    fft_block<PL, -1, 1>(v, smg, t, tw, mid);
#pragma unroll
    for (int r = 0; r < PL::E; ++r) v[r] = cmul(v[r], __ldg(&spectrum[t + PL::T * r]));
    if constexpr (PL::PASSES > 1) __syncthreads();
    fft_block<PL, 1, 1>(v, smg, t, tw, mid);
    if (active) {
        float2* yr = y + (size_t)pulse * N;
#pragma unroll
        for (int r = 0; r < PL::E; ++r) yr[t + PL::T * r] = v[r];  // stays in L2 for the next stage
    }
}

// Persistent variant for long pulses (one 512-thread CTA per SM holds a whole
// transform in shared memory, so CTAs cannot overlap each other's memory phases).
// Each CTA walks pulses blockIdx.x, +gridDim.x, ...; as soon as the inverse transform
// of one pulse has read the exchange buffer for the last time, one thread issues bulk
// copies of the CTA's next pulse into that buffer, so the load streams in while the
// current results are being stored.  Pulses are read from the staged copy
// (unpadded, element e at sm[e]), zero beyond `samples`.
template <int N, class Src>
__global__ void __launch_bounds__(FftPlan<N, elems_for(N)>::T)
pulse_compression_persistent_kernel(const Src src, int pulses, int samples,
                                    const float2* __restrict__ spectrum, float2* __restrict__ y,
                                    const float2* __restrict__ tw, int* err)
{
    using PL = FftPlan<N, elems_for(N)>;
    extern __shared__ __align__(128) float2 sm[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + PL::smem_elems());
    // second-pass twiddles, the same for every pulse the CTA transforms
    float2* mid = mid_table_elems<PL>() > 0 ? sm + PL::smem_elems() + 2 : nullptr;
    const int t = threadIdx.x;
    if (mid) fill_mid_table<PL>(mid, t, PL::T, tw);
    // first-pass twiddle bases, the same for every pulse and both directions: each
    // thread keeps its own in shared memory at an odd pitch of float2 (the 64-bit reads
    // of 16 lanes then land on distinct bank pairs)
    constexpr int LOGE = ilog2(PL::E);
    float2* first = sm + PL::smem_elems() + 2 + mid_table_elems<PL>() + t * (LOGE | 1);
    {
        float2 wb[LOGE];
        load_twiddle_bases<PL::E, PL::LOGN>(wb, t, tw);
#pragma unroll
        for (int b = 0; b < LOGE; ++b) first[b] = wb[b];
    }
    const int copy = samples < N ? samples : N;                 // elements staged per pulse
    const uint32_t bytes = (uint32_t)copy * (uint32_t)sizeof(float2);
    constexpr uint32_t kChunk = 32768;                          // bytes per bulk copy
    auto issue = [&](int pulse) {
        mbar_arrive_expect_tx(bar, bytes);
        const char* from = reinterpret_cast<const char*>(src.row(pulse));
        char* dst = reinterpret_cast<char*>(sm);
        for (uint32_t off = 0; off < bytes; off += kChunk)
            bulk_load_1d(dst + off, from + off, bytes - off < kChunk ? bytes - off : kChunk, bar);
    };
    if (t == 0) mbar_init(bar, 1);
    __syncthreads();
    int pulse = blockIdx.x;
    if (t == 0 && pulse < pulses) issue(pulse);
    uint32_t phase = 0;
    for (; pulse < pulses; pulse += gridDim.x) {
        const bool ok = mbar_wait_bounded(bar, phase);
        if (__syncthreads_or(!ok)) {
            if (t == 0) atomicCAS(err, 0, (int)kKernelTmaTimeout);
            return;
        }
        phase ^= 1u;
        // the next pulse can only be copied into shared memory once this one's exchanges
        // are done; pull it into L2 now so that copy reads L2 instead of HBM
        if (t == 0 && pulse + (int)gridDim.x < pulses) {
            const char* from = reinterpret_cast<const char*>(src.row(pulse + gridDim.x));
            for (uint32_t off = 0; off < bytes; off += kChunk)
                bulk_prefetch_l2(from + off, bytes - off < kChunk ? bytes - off : kChunk);
        }
        float2 v[PL::E];
#pragma unroll
        for (int r = 0; r < PL::E; ++r) {
            const int e = t + PL::T * r;
            v[r] = e < copy ? sm[e] : make_float2(0.f, 0.f);
        }
        __syncthreads();
        fft_block<PL, -1, 1>(v, sm, t, tw, mid, first);
#pragma unroll
        for (int r = 0; r < PL::E; ++r) v[r] = cmul(v[r], __ldg(&spectrum[t + PL::T * r]));
        __syncthreads();
        fft_block<PL, 1, 1>(v, sm, t, tw, mid, first);
        // every thread is done with the exchange buffer; order those accesses before the
        // bulk copy that overwrites it
        fence_proxy_async_smem();
        __syncthreads();
        const int next = pulse + gridDim.x;
        if (t == 0 && next < pulses) issue(next);
        float2* yr = y + (size_t)pulse * N;
#pragma unroll
        for (int r = 0; r < PL::E; ++r) yr[t + PL::T * r] = v[r];  // stays in L2 for the next stage
    }
}

// Persistent compression with the four-step ordering of fft_local.cuh (N = 4096, 8192,
// 16384): the same pulse loop, bulk-copy staging, L2 prefetch and pass-1 twiddle bases as
// the kernel above, but each direction synchronises the CTA twice instead of three or four
// times.  The forward transform leaves each thread the spectrum bins of a fixed
// digit-reversed set, so each thread writes its 2E spectrum words once, at the start, into
// its own tensor-memory lane (tcgen05.st) and reads them back per pulse (tcgen05.ld): no
// spectrum traffic from L2 per pulse (read at those bins from global memory, each warp
// load would touch 16 sectors).  Warp w uses lanes 32 (w % 4) .. +31 and columns
// (w / 4) 2E .. +2E-1 of the CTA's allocation, T / 128 * 2E columns: 256 at N = 16384
// (one CTA per SM), 128 at 8192 (two), 64 at 4096 (four).  (Keeping the pass-1 twiddles
// there as well, instead of forming them from bases, measured slower: 271.6 against
// 265.8 us for the 1024 x 16384 chain.)
template <int N>
constexpr int local_tmem_columns()
{
    using LP = LocalPlan<N>;
    constexpr int c = (LP::T / 128) * 2 * LP::E;
    return c < 32 ? 32 : c;
}

// PAIRS (y 16-byte aligned): lanes t and t^1 swap one value per register pair, so each
// thread stores two adjacent outputs with one 128-bit store (half the store instructions;
// 118.8 -> 115.0 us at 1024 x 16384, the same bits).
template <int N, class Src, bool PAIRS>
__global__ void __launch_bounds__(LocalPlan<N>::T)
pulse_compression_local_kernel(const Src src, int pulses, int samples, const float2* __restrict__ spectrum,
                               float2* __restrict__ y, const float2* __restrict__ tw, int* err)
{
    using LP = LocalPlan<N>;
    constexpr int LOGE = ilog2(LP::E);
    constexpr uint32_t kCols = local_tmem_columns<N>();
    static_assert(LP::T % 128 == 0 && (2 * LP::E) % 16 == 0, "tensor-memory slice layout");
    extern __shared__ __align__(128) float2 sm[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + LP::EXCHANGE);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + LP::EXCHANGE + 1);
    float2* tab = sm + LP::EXCHANGE + 2;
    const int t = threadIdx.x;
    const int warp = t >> 5;
    if (warp == 0) {
        tmem_alloc(tmem_slot, kCols);
        tmem_relinquish();
    }
    // pass-2 twiddles and this thread's pass-1 twiddle bases, the same for every pulse
    float2* first = tab + LP::TABLE + t * (LOGE | 1);
    fill_local_table<LP>(tab, t, LP::T, tw);
    {
        float2 wb[LOGE];
        load_twiddle_bases<LP::E, LP::LOGN>(wb, t, tw);
#pragma unroll
        for (int b = 0; b < LOGE; ++b) first[b] = wb[b];
    }
    if (t == 0) mbar_init(bar, 1);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;
    const uint32_t spec_cols = tmem_base + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(warp >> 2) * (2 * LP::E);
    spectrum_to_tmem<LP>(spectrum, t, spec_cols);
    auto twiddle = [&](float2(&x)[LP::E]) { apply_twiddles_from<LP::E, -1>(x, first); };
    auto twiddle_conj = [&](float2(&x)[LP::E]) { apply_twiddles_from<LP::E, 1>(x, first); };

    const int copy = samples < N ? samples : N;
    const uint32_t bytes = (uint32_t)copy * (uint32_t)sizeof(float2);
    constexpr uint32_t kChunk = 32768;
    auto issue = [&](int pulse) {
        mbar_arrive_expect_tx(bar, bytes);
        const char* from = reinterpret_cast<const char*>(src.row(pulse));
        char* dst = reinterpret_cast<char*>(sm);
        for (uint32_t off = 0; off < bytes; off += kChunk)
            bulk_load_1d(dst + off, from + off, bytes - off < kChunk ? bytes - off : kChunk, bar);
    };
    int pulse = blockIdx.x;
    if (t == 0 && pulse < pulses) issue(pulse);
    uint32_t phase = 0;
    bool timed_out = false;
    for (; pulse < pulses; pulse += gridDim.x) {
        const bool ok = mbar_wait_bounded(bar, phase);
        if (__syncthreads_or(!ok)) {
            if (t == 0) atomicCAS(err, 0, (int)kKernelTmaTimeout);
            timed_out = true;
            break;
        }
        phase ^= 1u;
        if (t == 0 && pulse + (int)gridDim.x < pulses) {
            const char* from = reinterpret_cast<const char*>(src.row(pulse + gridDim.x));
            for (uint32_t off = 0; off < bytes; off += kChunk)
                bulk_prefetch_l2(from + off, bytes - off < kChunk ? bytes - off : kChunk);
        }
        float2 v[LP::E];
#pragma unroll
        for (int r = 0; r < LP::E; ++r) {
            const int e = t + LP::T * r;
            v[r] = e < copy ? sm[e] : make_float2(0.f, 0.f);
        }
        __syncthreads();
        local_fft_forward<LP>(v, sm, t, twiddle, tab);
        tmem_multiply<LP::E, false>(v, spec_cols);
        local_fft_inverse<LP>(v, sm, t, twiddle_conj, tab);
        fence_proxy_async_smem();
        __syncthreads();
        const int next = pulse + gridDim.x;
        if (t == 0 && next < pulses) issue(next);
        float2* yr = y + (size_t)pulse * N;
#pragma unroll
        for (int r = 0; r < LP::E; r += 2) {  // outputs stay in L2 for the next stage
            if constexpr (PAIRS) {
                const bool even = (t & 1) == 0;
                const float2 send = even ? v[r + 1] : v[r];
                float2 recv;
                recv.x = __shfl_xor_sync(0xffffffffu, send.x, 1);
                recv.y = __shfl_xor_sync(0xffffffffu, send.y, 1);
                const float4 pair = even ? make_float4(v[r].x, v[r].y, recv.x, recv.y)
                                         : make_float4(recv.x, recv.y, v[r + 1].x, v[r + 1].y);
                const int e = even ? t + LP::T * r : (t - 1) + LP::T * (r + 1);
                *reinterpret_cast<float4*>(yr + e) = pair;
            } else {
                yr[t + LP::T * r] = v[r];
                yr[t + LP::T * (r + 1)] = v[r + 1];
            }
        }
    }
    // every warp is done with tensor memory (on the timeout path too): release it.  A
    // timed-out CTA waits (bounded) for its copy still in flight before leaving.
    if (timed_out && t == 0) (void)mbar_wait_bounded(bar, phase);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem_base, kCols);
    }
}

// Batched C2C transform of contiguous rows: forward unnormalised, inverse scaled by 1/N
// (the convention of the reference's FFTInterface, fft_interface.h:39-42).  Each row is
// held in registers before any store, so in-place calls (x == y) are safe.
template <int N, int G, int DIR>
__global__ void __launch_bounds__(G * FftPlan<N, elems_for(N)>::T)
fft_rows_kernel(const float2* x, int rows, float2* y, const float2* __restrict__ tw)
{
    using PL = FftPlan<N, elems_for(N)>;
    extern __shared__ float2 sm[];
    const int g = threadIdx.x / PL::T;
    const int t = threadIdx.x - g * PL::T;
    const int row = blockIdx.x * G + g;
    const bool active = row < rows;
    constexpr int S = PL::smem_elems() % 16 == 0 && PL::T < 16 ? PL::smem_elems() + 8 : PL::smem_elems();
    float2* smg = sm + g * S;
    const float2* xr = x + (size_t)row * N;
    float2 v[PL::E];
#pragma unroll
    for (int r = 0; r < PL::E; ++r) v[r] = active ? xr[t + PL::T * r] : make_float2(0.f, 0.f);
    fft_block<PL, DIR, 1>(v, smg, t, tw);
    if (active) {
        float2* yr = y + (size_t)row * N;
        constexpr float scale = DIR > 0 ? 1.0f / (float)N : 1.0f;
#pragma unroll
        for (int r = 0; r < PL::E; ++r) {
            float2 o = v[r];
            if (DIR > 0) {
                o.x *= scale;
                o.y *= scale;
            }
            yr[t + PL::T * r] = o;
        }
    }
}

// ------------------------------------------------------------------- Doppler

// Range columns per Doppler CTA: 16 (128-byte row segments per warp load, a
// conflict-free interleave without padding) while the CTA stays within 1024 threads,
// fewer with the padded exchange for the longest transforms.  The loads of a CTA are
// row-strided, so throughput follows the bytes per request: 8 columns (64-byte
// segments) measured half the bandwidth of 16.  Both layouts were checked
// conflict-free for every supported length by simulating the exchange addresses.
constexpr int doppler_columns(int n)
{
    const int t = n / elems_for(n);
    return t <= 64 ? 16 : 1024 / t;
}

// CTA = C consecutive range columns x all pulses.  Thread (t, c) with c fastest, so
// each warp touches C*8-byte row segments.  Columns are interleaved in shared memory
// (element e of column c at e*C + c); with C = 16 every half-warp lands on distinct
// banks without padding, smaller C uses the per-pass padding.
template <int N>
__global__ void __launch_bounds__(doppler_columns(N) * FftPlan<N, elems_for(N)>::T)
pulse_doppler_kernel(const float2* __restrict__ x, int pulses, int samples,
                     const float* __restrict__ window, float2* __restrict__ out,
                     float* __restrict__ power, const float2* __restrict__ tw)
{
    using PL = FftPlan<N, elems_for(N)>;
    constexpr int C = doppler_columns(N);
    constexpr bool PAD = C < 16;
    extern __shared__ float2 sm[];
    const int c = threadIdx.x % C;
    const int t = threadIdx.x / C;
    const int col = blockIdx.x * C + c;
    const bool active = col < samples;
    (void)PAD;
    // CPI of a stacked batch
    x += (size_t)blockIdx.y * pulses * samples;
    if (out) out += (size_t)blockIdx.y * N * samples;
    if (power) power += (size_t)blockIdx.y * N * samples;
    float2 v[PL::E];
#pragma unroll
    for (int r = 0; r < PL::E; ++r) {
        const int e = t + PL::T * r;
        float2 a = make_float2(0.f, 0.f);
        if (active && e < pulses) {
            a = __ldcs(&x[(size_t)e * samples + col]);
            if (window) {
                const float w = __ldg(&window[e]);
                a.x *= w;
                a.y *= w;
            }
        }
        v[r] = a;
    }
    fft_block<PL, -1, C, PAD>(v, sm + c, t, tw);
    if (active) {
#pragma unroll
        for (int r = 0; r < PL::E; ++r) {
            const size_t o = (size_t)(t + PL::T * r) * samples + col;
            if (out) __stcs(&out[o], v[r]);
            if (power) power[o] = fmaf(v[r].x, v[r].x, v[r].y * v[r].y);  // read next by CFAR
        }
    }
}

// TMA-fed variant (16 columns): one thread issues the tile's 2-D bulk copies
// (boxes of 16 columns x up to 256 pulses, pulses beyond the input zero-filled by the
// copy engine) and the CTA waits on an mbarrier.  Row-strided tiles reach much higher
// bandwidth this way than with per-thread loads, whose throughput is bounded by the
// requests a thread can keep in flight.  The tile buffer doubles as the exchange
// buffer once every thread has read its values.
template <int N, int C>
__global__ void __launch_bounds__(C * FftPlan<N, elems_for(N)>::T)
pulse_doppler_tma_kernel(const __grid_constant__ CUtensorMap tmap, int pulses, int samples,
                         const float* __restrict__ window, float2* __restrict__ out,
                         float* __restrict__ power, const float2* __restrict__ tw, int* err)
{
    using PL = FftPlan<N, elems_for(N)>;
    constexpr int BOXH = N < 256 ? N : 256;
    extern __shared__ __align__(128) float2 sm[];
    // the exchange of a narrower tile is padded and can outgrow the landed tile
    constexpr int SPAN = C < 16 && C * PL::smem_elems(true) > N * C ? C * PL::smem_elems(true) : N * C;
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + SPAN);
    const int c = threadIdx.x % C;
    const int t = threadIdx.x / C;
    const int col0 = blockIdx.x * C;
    const int cpi = blockIdx.y;  // CPI of a stacked batch: rows cpi*pulses .. +pulses-1
    if (out) out += (size_t)cpi * N * samples;
    if (power) power += (size_t)cpi * N * samples;
    if (threadIdx.x == 0) mbar_init(bar, 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        mbar_arrive_expect_tx(bar, (uint32_t)(N * C * sizeof(float2)));
#pragma unroll
        for (int b = 0; b < N / BOXH; ++b)
            tma_load_2d(sm + b * BOXH * C, &tmap, 2 * col0, cpi * pulses + b * BOXH, bar);
    }
    // the window weights and the first pass's twiddle bases arrive while the tile is
    // in flight
    float wv[PL::E];
#pragma unroll
    for (int r = 0; r < PL::E; ++r) {
        const int e = t + PL::T * r;
        wv[r] = (window && e < pulses) ? __ldg(&window[e]) : 1.f;
    }
    float2 wb[ilog2(PL::E) > 0 ? ilog2(PL::E) : 1];
    if constexpr (PL::PASSES > 1) load_twiddle_bases<PL::E, PL::LOGN>(wb, t, tw);
    const bool ok = mbar_wait_bounded(bar, 0);
    if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0) atomicCAS(err, 0, (int)kKernelTmaTimeout);
        return;
    }
    const int col = col0 + c;
    const bool active = col < samples;
    float2 v[PL::E];
#pragma unroll
    for (int r = 0; r < PL::E; ++r) {
        const int e = t + PL::T * r;
        // rows past this CPI's pulses (zero padding to nfft) may hold the next CPI's data
        float2 a = e < pulses ? sm[e * C + c] : make_float2(0.f, 0.f);
        if (window && e < pulses) {
            a.x *= wv[r];
            a.y *= wv[r];
        }
        v[r] = a;
    }
    __syncthreads();
    fft_block<PL, -1, C, (C < 16)>(v, sm + c, t, tw, nullptr, PL::PASSES > 1 ? wb : nullptr);
    if (active) {
#pragma unroll
        for (int r = 0; r < PL::E; ++r) {
            const size_t o = (size_t)(t + PL::T * r) * samples + col;
            if (out) __stcs(&out[o], v[r]);
            if (power) power[o] = fmaf(v[r].x, v[r].x, v[r].y * v[r].y);  // read next by CFAR
        }
    }
}

__global__ void doppler_window_kernel(int pulses, int kind, const float* explicit_window,
                                      float* out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < pulses) out[i] = window_value(kind, explicit_window, i, pulses);
}

// --------------------------------------------------------------- dispatchers

template <int N>
int replica_impl(const float2* h, int length, int normalize, int kind, const float* w,
                 float2* spectrum, cudaStream_t s)
{
    if (!twiddle_table()) return fail(ZKX_INTERNAL_ERROR, "twiddle table not initialised on this device");
    using PL = FftPlan<N, elems_for(N)>;
    const size_t smem = (size_t)PL::smem_elems() * sizeof(float2);
    auto k = replica_spectrum_kernel<N>;
    ZKX_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k<<<1, PL::T, smem, s>>>(h, length, normalize, kind, w, spectrum, twiddle_table());
    ZKX_LAUNCHED("replica_spectrum_kernel");
    return ZKX_SUCCESS;
}

template <int N>
constexpr size_t local_compression_smem()
{
    using LP = LocalPlan<N>;
    return ((size_t)LP::EXCHANGE + 2 + LP::TABLE + (size_t)LP::T * (ilog2(LP::E) | 1)) * sizeof(float2);
}

// CTAs of the four-step compression kernel resident on the whole GPU at once.
template <int N>
int local_compression_slots(int* slots)
{
    using LP = LocalPlan<N>;
    int dev = 0, sms = 0, per_sm = 0;
    ZKX_CUDA(cudaGetDevice(&dev));
    ZKX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    auto k = pulse_compression_local_kernel<N, RowsContiguous, true>;
    const size_t smem = local_compression_smem<N>();
    ZKX_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    ZKX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, LP::T, smem));
    *slots = sms * std::max(per_sm, 1);
    return ZKX_SUCCESS;
}

// The default kernel for the four-step lengths: the persistent kernel once every resident
// CTA gets at least four pulses (its set-up per CTA and its pipelining then pay off), the
// one-launch-per-pulse kernel below that (measured: 1024 x 16384 265.8 vs 278.5 us for the
// chain; 256 x 16384 91.1 vs 83.8; 512 x 8192 90.3 vs 85.7; 1024 x 4096 91.9 vs 81.7).
int default_variant_for(int pulses, int slots)
{
    return pulses >= 4 * slots ? ZKX_COMPRESSION_LOCAL : ZKX_COMPRESSION_PLAIN;
}

template <int N, class Src>
int compression_impl(const Src& x, bool aligned16, int pulses, int samples, const float2* spectrum,
                     float2* y, int variant, cudaStream_t s)
{
    if (!twiddle_table()) return fail(ZKX_INTERNAL_ERROR, "twiddle table not initialised on this device");
    using PL = FftPlan<N, elems_for(N)>;
    if constexpr (local_fft_for(N)) {
        if (variant == ZKX_COMPRESSION_DEFAULT) {
            int slots = 0;
            ZKX_TRY(local_compression_slots<N>(&slots));
            variant = default_variant_for(pulses, slots);
        }
        if (aligned16 && variant == ZKX_COMPRESSION_LOCAL) {
            using LP = LocalPlan<N>;
            int slots = 0;
            ZKX_TRY(local_compression_slots<N>(&slots));
            const size_t smem = local_compression_smem<N>();
            const bool pairs = (reinterpret_cast<uintptr_t>(y) & 15) == 0;
            auto k = pairs ? pulse_compression_local_kernel<N, Src, true> : pulse_compression_local_kernel<N, Src, false>;
            ZKX_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            const int grid = std::max(1, std::min(pulses, slots));
            k<<<grid, LP::T, smem, s>>>(x, pulses, samples, spectrum, y, twiddle_table(), kernel_error_word());
            ZKX_LAUNCHED("pulse_compression_local_kernel");
            return ZKX_SUCCESS;
        }
    }
    if constexpr (N >= 4096) {
        // persistent bulk-copy pipeline: 16-byte aligned pulses (even length, aligned bases);
        // variant ZKX_COMPRESSION_PLAIN keeps the one-launch-per-pulse-group kernel
        if (aligned16 && variant != ZKX_COMPRESSION_PLAIN) {
            int dev = 0, sms = 0;
            ZKX_CUDA(cudaGetDevice(&dev));
            ZKX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
            const size_t smem = ((size_t)PL::smem_elems() + 2 + mid_table_elems<PL>() +
                                 (size_t)PL::T * (ilog2(PL::E) | 1)) * sizeof(float2);
            auto k = pulse_compression_persistent_kernel<N, Src>;
            ZKX_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            int per_sm = 0;
            ZKX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, PL::T, smem));
            const int grid = std::max(1, std::min(pulses, sms * std::max(per_sm, 1)));
            k<<<grid, PL::T, smem, s>>>(x, pulses, samples, spectrum, y, twiddle_table(),
                                        kernel_error_word());
            ZKX_LAUNCHED("pulse_compression_persistent_kernel");
            return ZKX_SUCCESS;
        }
    }
    constexpr int G = rows_per_cta(N);
    const size_t smem = ((size_t)G * PL::smem_elems() +
                         (compression_mid_table<N>() ? mid_table_elems<PL>() : 0)) * sizeof(float2);
    auto k = pulse_compression_kernel<N, G, Src>;
    ZKX_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int blocks = (pulses + G - 1) / G;
    k<<<blocks, G * PL::T, smem, s>>>(x, pulses, samples, spectrum, y, twiddle_table());
    ZKX_LAUNCHED("pulse_compression_kernel");
    return ZKX_SUCCESS;
}

template <int N, int CT>
int doppler_tma(const CUtensorMap& map, int pulses, int samples, const float* window, float2* out,
                float* power, int batch, cudaStream_t s)
{
    using PL = FftPlan<N, elems_for(N)>;
    constexpr int SPAN = CT < 16 && CT * PL::smem_elems(true) > N * CT ? CT * PL::smem_elems(true) : N * CT;
    const size_t smem = (size_t)SPAN * sizeof(float2) + 16;
    auto k = pulse_doppler_tma_kernel<N, CT>;
    ZKX_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const dim3 tiles((samples + CT - 1) / CT, batch);
    k<<<tiles, CT * PL::T, smem, s>>>(map, pulses, samples, window, out, power, twiddle_table(),
                                      kernel_error_word());
    ZKX_LAUNCHED("pulse_doppler_tma_kernel");
    return ZKX_SUCCESS;
}

template <int N>
int doppler_impl(const float2* x, int pulses, int samples, const float* window, float2* out,
                 float* power, int batch, int columns, cudaStream_t s)
{
    if (!twiddle_table()) return fail(ZKX_INTERNAL_ERROR, "twiddle table not initialised on this device");
    using PL = FftPlan<N, elems_for(N)>;
    constexpr int C = doppler_columns(N);
    const dim3 blocks((samples + C - 1) / C, batch);
    if (batch > 65535) return launch_doppler_any(x, pulses, samples, N, window, out, power, batch, s);
    if constexpr (C == 16) {
        // TMA path: rows must be 16-byte multiples and the base 16-byte aligned
        if ((samples & 1) == 0 && (reinterpret_cast<uintptr_t>(x) & 15) == 0) {
            CUtensorMap map;
            constexpr int BOXH = N < 256 ? N : 256;
            // columns per CTA on the bulk-copy path: 8 (two tiles of 64 KB per SM overlap
            // each other's copy, transform and stores) measured faster from 512 pulses up,
            // 16 below; `columns` overrides (the autotuner's choice)
            const int ct = columns == 8 || columns == 16 ? columns : (N >= 512 ? 8 : 16);
            if (encode_tensor_map_2d_f32(&map, x, 2ull * samples, (uint64_t)pulses * batch,
                                         (uint64_t)samples * sizeof(float2), 2 * ct, BOXH))
                return ct == 8 ? doppler_tma<N, 8>(map, pulses, samples, window, out, power, batch, s)
                               : doppler_tma<N, 16>(map, pulses, samples, window, out, power, batch, s);
        }
    }
    const size_t smem = (size_t)C * PL::smem_elems(C < 16) * sizeof(float2);
    if (smem > 227 * 1024)  // the column tile does not fit: transposed row passes instead
        return launch_doppler_any(x, pulses, samples, N, window, out, power, batch, s);
    auto k = pulse_doppler_kernel<N>;
    ZKX_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k<<<blocks, C * PL::T, smem, s>>>(x, pulses, samples, window, out, power, twiddle_table());
    ZKX_LAUNCHED("pulse_doppler_kernel");
    return ZKX_SUCCESS;
}

template <int N>
int fft_rows_impl(const float2* x, int rows, int inverse, float2* y, cudaStream_t s)
{
    if (!twiddle_table()) return fail(ZKX_INTERNAL_ERROR, "twiddle table not initialised on this device");
    using PL = FftPlan<N, elems_for(N)>;
    constexpr int G = rows_per_cta(N);
    constexpr int S = PL::smem_elems() % 16 == 0 && PL::T < 16 ? PL::smem_elems() + 8 : PL::smem_elems();
    const size_t smem = (size_t)G * S * sizeof(float2);
    const int blocks = (rows + G - 1) / G;
    if (inverse) {
        auto k = fft_rows_kernel<N, G, 1>;
        ZKX_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k<<<blocks, G * PL::T, smem, s>>>(x, rows, y, twiddle_table());
    } else {
        auto k = fft_rows_kernel<N, G, -1>;
        ZKX_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k<<<blocks, G * PL::T, smem, s>>>(x, rows, y, twiddle_table());
    }
    ZKX_LAUNCHED("fft_rows_kernel");
    return ZKX_SUCCESS;
}

#define ZKX_DISPATCH_POW2(LOG, CALL)                                                    \
    switch (LOG) {                                                                      \
    case 0: return CALL(1);     case 1: return CALL(2);     case 2: return CALL(4);     \
    case 3: return CALL(8);     case 4: return CALL(16);    case 5: return CALL(32);    \
    case 6: return CALL(64);    case 7: return CALL(128);   case 8: return CALL(256);   \
    case 9: return CALL(512);   case 10: return CALL(1024); case 11: return CALL(2048); \
    case 12: return CALL(4096); case 13: return CALL(8192); case 14: return CALL(16384);\
    default: return fail(ZKX_UNSUPPORTED_OPERATION, "transform length above 16384");    \
    }

}  // namespace

int launch_replica_spectrum(const float2* replica, int length, int nfft, int normalize,
                            int window_kind, const float* explicit_window, float2* spectrum,
                            cudaStream_t stream)
{
    if (!is_pow2(nfft))
        return launch_replica_spectrum_any(replica, length, nfft, normalize, window_kind, explicit_window,
                                           spectrum, stream);
    if (nfft > (1 << kMaxSmemFftLog))
        return launch_long_replica_spectrum(replica, length, nfft, normalize, window_kind, explicit_window,
                                            spectrum, stream);
#define ZKX_CALL(NN) replica_impl<NN>(replica, length, normalize, window_kind, explicit_window, spectrum, stream)
    ZKX_DISPATCH_POW2(ilog2_host(nfft), ZKX_CALL)
#undef ZKX_CALL
}

int launch_pulse_compression(const float2* x, int pulses, int samples, int nfft,
                             const float2* spectrum, float2* y, cudaStream_t stream)
{
    return launch_pulse_compression_variant(x, pulses, samples, nfft, spectrum, y, ZKX_COMPRESSION_DEFAULT,
                                            stream);
}

int launch_pulse_compression_variant(const float2* x, int pulses, int samples, int nfft,
                                     const float2* spectrum, float2* y, int variant, cudaStream_t stream)
{
    const RowsContiguous src{x, samples};
    if (!is_pow2(nfft)) return launch_compression_any(src, pulses, samples, nfft, spectrum, y, stream);
    if (nfft > (1 << kMaxSmemFftLog))
        return launch_long_compression(src, pulses, samples, nfft, spectrum, y, variant, stream);
    const bool aligned16 = (samples & 1) == 0 && (reinterpret_cast<uintptr_t>(x) & 15) == 0;
#define ZKX_CALL(NN) compression_impl<NN>(src, aligned16, pulses, samples, spectrum, y, variant, stream)
    ZKX_DISPATCH_POW2(ilog2_host(nfft), ZKX_CALL)
#undef ZKX_CALL
}

int resolve_compression_variant(int pulses, int nfft, int variant, int* resolved)
{
    *resolved = variant;
    if (variant != ZKX_COMPRESSION_DEFAULT || !is_pow2(nfft)) return ZKX_SUCCESS;
    if (nfft == 2 * (1 << kMaxSmemFftLog) || nfft == 4 * (1 << kMaxSmemFftLog))
        return resolve_long_compression_variant(pulses, nfft, resolved);
    if (!local_fft_for(nfft)) return ZKX_SUCCESS;
    int slots = 0;
    switch (nfft) {
    case 4096: ZKX_TRY(local_compression_slots<4096>(&slots)); break;
    case 8192: ZKX_TRY(local_compression_slots<8192>(&slots)); break;
    default: ZKX_TRY(local_compression_slots<16384>(&slots)); break;
    }
    *resolved = default_variant_for(pulses, slots);
    return ZKX_SUCCESS;
}

int launch_pulse_compression_table(const float2* const* cpis, int count, int pulses_per_cpi,
                                   int samples, int nfft, const float2* spectrum, float2* y,
                                   int variant, cudaStream_t stream)
{
    if (count < 1 || count > kMaxRowTable)
        return fail(ZKX_INVALID_ARGUMENT, "pulse_compression: 1 to 64 CPIs per table launch");
    RowsTable src{};
    src.pulses = pulses_per_cpi;
    src.samples = samples;
    bool aligned16 = (samples & 1) == 0;
    for (int i = 0; i < count; ++i) {
        src.cpi[i] = cpis[i];
        aligned16 = aligned16 && (reinterpret_cast<uintptr_t>(cpis[i]) & 15) == 0;
    }
    const int pulses = count * pulses_per_cpi;
    if (!is_pow2(nfft)) return launch_compression_any(src, pulses, samples, nfft, spectrum, y, stream);
    if (nfft > (1 << kMaxSmemFftLog))
        return launch_long_compression(src, pulses, samples, nfft, spectrum, y, variant, stream);
#define ZKX_CALL(NN) compression_impl<NN>(src, aligned16, pulses, samples, spectrum, y, variant, stream)
    ZKX_DISPATCH_POW2(ilog2_host(nfft), ZKX_CALL)
#undef ZKX_CALL
}

int launch_pulse_doppler(const float2* x, int pulses, int samples, int nfft, const float* window,
                         float2* out, float* power, int batch, int columns, cudaStream_t stream)
{
    if (!is_pow2(nfft) || nfft > 4096)
        return launch_doppler_any(x, pulses, samples, nfft, window, out, power, batch, stream);
#define ZKX_CALL(NN) doppler_impl<NN>(x, pulses, samples, window, out, power, batch, columns, stream)
    ZKX_DISPATCH_POW2(ilog2_host(nfft), ZKX_CALL)
#undef ZKX_CALL
}

int launch_fft_rows(const float2* x, int rows, int n, int inverse, float2* y, cudaStream_t stream)
{
    if (!is_pow2(n)) return launch_dft_rows(x, rows, n, inverse, y, stream);
    if (n > (1 << kMaxSmemFftLog)) return launch_long_fft_rows(x, rows, n, inverse, y, stream);
#define ZKX_CALL(NN) fft_rows_impl<NN>(x, rows, inverse, y, stream)
    ZKX_DISPATCH_POW2(ilog2_host(n), ZKX_CALL)
#undef ZKX_CALL
}

int launch_doppler_window(int pulses, int window_kind, const float* explicit_window, float* out,
                          cudaStream_t stream)
{
    doppler_window_kernel<<<(pulses + 255) / 256, 256, 0, stream>>>(pulses, window_kind,
                                                                    explicit_window, out);
    ZKX_LAUNCHED("doppler_window_kernel");
    return ZKX_SUCCESS;
}

}  // namespace zkx
