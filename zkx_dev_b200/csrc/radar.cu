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
#include "worklist.h"

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
template <int N, int E = elems_for(N)>
constexpr bool compression_mid_table()
{
    return N >= 4096 && mid_table_elems<FftPlan<N, E>>() > 0;
}

// G transforms per CTA, thread group g = threadIdx.x / T: load row xr (zero-pad/truncate
// to N; null: an idle group), forward FFT, multiply by the replica spectrum, inverse FFT,
// store to yr (null: nothing stored).  Shared by the one-launch-per-pulse-group kernel and
// the work-list kernel, so both round identically.
template <int N, int E, int G>
__device__ __forceinline__ void compress_rows(const float2* __restrict__ xr, int samples,
                                              const float2* __restrict__ spectrum, float2* __restrict__ yr,
                                              const float2* __restrict__ tw, float2* sm)
{
    using PL = FftPlan<N, E>;
    const int g = threadIdx.x / PL::T;
    const int t = threadIdx.x - g * PL::T;
    float2* smg = sm + g * PL::smem_elems();
    // lengths that also have the persistent kernel take its second-pass twiddle table,
    // so both kernels round identically and the tuning choice never changes a result
    float2* mid = compression_mid_table<N, E>() ? sm + G * PL::smem_elems() : nullptr;
    if (mid) fill_mid_table<PL>(mid, threadIdx.x, G * PL::T, tw);
    float2 v[PL::E];
#pragma unroll
    for (int r = 0; r < PL::E; ++r) {
        const int e = t + PL::T * r;
        v[r] = (xr != nullptr && e < samples) ? __ldcs(&xr[e]) : make_float2(0.f, 0.f);
    }
    fft_block<PL, -1, 1>(v, smg, t, tw, mid);
#pragma unroll
    for (int r = 0; r < PL::E; ++r) v[r] = cmul(v[r], __ldg(&spectrum[t + PL::T * r]));
    if constexpr (PL::PASSES > 1) __syncthreads();
    fft_block<PL, 1, 1>(v, smg, t, tw, mid);
    if (yr != nullptr) {
#pragma unroll
        for (int r = 0; r < PL::E; ++r) yr[t + PL::T * r] = v[r];  // stays in L2 for the next stage
    }
}

// Shared memory of compress_rows<N, E, G>.
template <int N, int E, int G>
constexpr size_t compress_rows_smem()
{
    using PL = FftPlan<N, E>;
    return ((size_t)G * PL::smem_elems() + (compression_mid_table<N, E>() ? mid_table_elems<PL>() : 0)) *
           sizeof(float2);
}

// G pulses per CTA; each pulse: load (zero-pad/truncate to N), forward FFT, multiply
// by the replica spectrum, inverse FFT, store.  The cube crosses HBM once each way.
template <int N, int E, int G, class Src>
__global__ void __launch_bounds__(G * FftPlan<N, E>::T)
pulse_compression_kernel(const Src src, int pulses, int samples,
                         const float2* __restrict__ spectrum, float2* __restrict__ y,
                         const float2* __restrict__ tw)
{
    using PL = FftPlan<N, E>;
    extern __shared__ float2 sm[];
    const int pulse = blockIdx.x * G + (int)(threadIdx.x / PL::T);
    const bool active = pulse < pulses;
    compress_rows<N, E, G>(active ? src.row(pulse) : nullptr, samples, spectrum,
                        active ? y + (size_t)pulse * N : nullptr, tw, sm);
}

// Persistent variant for long pulses (one 512-thread CTA per SM holds a whole
// transform in shared memory, so CTAs cannot overlap each other's memory phases).
// Each CTA walks pulses blockIdx.x, +gridDim.x, ...; as soon as the inverse transform
// of one pulse has read the exchange buffer for the last time, one thread issues bulk
// copies of the CTA's next pulse into that buffer, so the load streams in while the
// current results are being stored.  Pulses are read from the staged copy
// (unpadded, element e at sm[e]), zero beyond `samples`.
template <int N, int E, class Src>
__global__ void __launch_bounds__(FftPlan<N, E>::T)
pulse_compression_persistent_kernel(const Src src, int pulses, int samples,
                                    const float2* __restrict__ spectrum, float2* __restrict__ y,
                                    const float2* __restrict__ tw, int* err)
{
    using PL = FftPlan<N, E>;
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

// TMA-fed Doppler tile: one thread issues the tile's 2-D bulk copies (boxes of C
// columns x up to 256 pulses, pulses beyond the input zero-filled by the copy engine)
// and the CTA waits on an mbarrier.  Row-strided tiles reach much higher bandwidth this
// way than with per-thread loads, whose throughput is bounded by the requests a thread
// can keep in flight.  The tile buffer doubles as the exchange buffer once every thread
// has read its values.  Tile = columns col0 .. col0+C-1 of CPI `cpi`, whose pulses are
// rows cpi*pulses .. of the map; out and power point at this CPI's planes.  Returns
// false (error word set) if the copy did not complete.  Shared by the per-shape kernel
// and the work-list kernel.
template <int N, int C>
constexpr int doppler_tile_span()
{
    using PL = FftPlan<N, elems_for(N)>;
    // the exchange of a narrower tile is padded and can outgrow the landed tile
    return C < 16 && C * PL::smem_elems(true) > N * C ? C * PL::smem_elems(true) : N * C;
}

template <int N, int C>
__device__ __forceinline__ bool doppler_tma_tile(const CUtensorMap* tmap, int pulses, int samples, int cpi,
                                                 int col0, const float* __restrict__ window,
                                                 float2* __restrict__ out, float* __restrict__ power,
                                                 const float2* __restrict__ tw, int* err, float2* sm)
{
    using PL = FftPlan<N, elems_for(N)>;
    constexpr int BOXH = N < 256 ? N : 256;
    constexpr int SPAN = doppler_tile_span<N, C>();
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + SPAN);
    const int c = threadIdx.x % C;
    const int t = threadIdx.x / C;
    if (threadIdx.x == 0) mbar_init(bar, 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        mbar_arrive_expect_tx(bar, (uint32_t)(N * C * sizeof(float2)));
#pragma unroll
        for (int b = 0; b < N / BOXH; ++b)
            tma_load_2d(sm + b * BOXH * C, tmap, 2 * col0, cpi * pulses + b * BOXH, bar);
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
        return false;
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
    return true;
}

// Per-shape Doppler: CTA (x, y) = column tile x of CPI y of a stacked batch.
template <int N, int C>
__global__ void __launch_bounds__(C * FftPlan<N, elems_for(N)>::T)
pulse_doppler_tma_kernel(const __grid_constant__ CUtensorMap tmap, int pulses, int samples,
                         const float* __restrict__ window, float2* __restrict__ out,
                         float* __restrict__ power, const float2* __restrict__ tw, int* err)
{
    extern __shared__ __align__(128) float2 sm[];
    const int cpi = blockIdx.y;
    doppler_tma_tile<N, C>(&tmap, pulses, samples, cpi, blockIdx.x * C, window,
                           out ? out + (size_t)cpi * N * samples : nullptr,
                           power ? power + (size_t)cpi * N * samples : nullptr, tw, err, sm);
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

// The Stockham-ordered compression with E values per thread: the persistent bulk-copy
// pipeline (variant ZKX_COMPRESSION_PERSISTENT, 16-byte aligned pulses, N >= 4096) or
// the one-launch-per-pulse-group kernel; both round identically.  ctas_per_sm > 0 caps the
// persistent kernel's CTAs per SM.
template <int N, int E, class Src>
int stockham_compression(const Src& x, bool aligned16, int pulses, int samples, const float2* spectrum,
                         float2* y, int variant, int ctas_per_sm, cudaStream_t s)
{
    using PL = FftPlan<N, E>;
    if constexpr (N >= 4096) {
        if (aligned16 && variant != ZKX_COMPRESSION_PLAIN) {
            int dev = 0, sms = 0;
            ZKX_CUDA(cudaGetDevice(&dev));
            ZKX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
            const size_t smem = ((size_t)PL::smem_elems() + 2 + mid_table_elems<PL>() +
                                 (size_t)PL::T * (ilog2(PL::E) | 1)) * sizeof(float2);
            auto k = pulse_compression_persistent_kernel<N, E, Src>;
            ZKX_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            int per_sm = 0;
            ZKX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, PL::T, smem));
            per_sm = std::max(per_sm, 1);
            if (ctas_per_sm > 0) per_sm = std::min(per_sm, ctas_per_sm);
            const int grid = std::max(1, std::min(pulses, sms * per_sm));
            k<<<grid, PL::T, smem, s>>>(x, pulses, samples, spectrum, y, twiddle_table(),
                                        kernel_error_word());
            ZKX_LAUNCHED("pulse_compression_persistent_kernel");
            return ZKX_SUCCESS;
        }
    }
    constexpr int G = PL::T >= 128 ? 1 : 128 / PL::T;   // >= 128 threads per CTA
    const size_t smem = compress_rows_smem<N, E, G>();
    auto k = pulse_compression_kernel<N, E, G, Src>;
    ZKX_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int blocks = (pulses + G - 1) / G;
    k<<<blocks, G * PL::T, smem, s>>>(x, pulses, samples, spectrum, y, twiddle_table());
    ZKX_LAUNCHED("pulse_compression_kernel");
    return ZKX_SUCCESS;
}

// Values per thread of the Stockham compression kernels besides the table's (the radix
// plan the autotuner may choose): 32 <-> 16 where the CTA stays within 32 .. 512 threads.
constexpr int alt_compression_radix(int n)
{
    return n < 1024 || n > 8192 ? 0 : (elems_for(n) == 32 ? 16 : 32);
}

template <int N, class Src>
int compression_impl(const Src& x, bool aligned16, int pulses, int samples, const float2* spectrum,
                     float2* y, int variant, int radix, int ctas_per_sm, cudaStream_t s)
{
    if (!twiddle_table()) return fail(ZKX_INTERNAL_ERROR, "twiddle table not initialised on this device");
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
            if (ctas_per_sm > 0) {
                int dev = 0, sms = 0;
                ZKX_CUDA(cudaGetDevice(&dev));
                ZKX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
                slots = std::min(slots, sms * ctas_per_sm);
            }
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
    constexpr int ALT = alt_compression_radix(N);
    if constexpr (ALT != 0) {
        if (radix == ALT)
            return stockham_compression<N, ALT, Src>(x, aligned16, pulses, samples, spectrum, y, variant,
                                                     ctas_per_sm, s);
    }
    return stockham_compression<N, elems_for(N), Src>(x, aligned16, pulses, samples, spectrum, y, variant,
                                                      ctas_per_sm, s);
}

template <int N, int CT>
int doppler_tma(const CUtensorMap& map, int pulses, int samples, const float* window, float2* out,
                float* power, int batch, cudaStream_t s)
{
    using PL = FftPlan<N, elems_for(N)>;
    const size_t smem = (size_t)doppler_tile_span<N, CT>() * sizeof(float2) + 16;
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
    } else if constexpr (N == 2048 || N == 4096) {
        // the longest slow-time transforms in one CTA: narrower bulk-copy tiles (C = 4 or 8
        // columns at 2048 pulses, 2 or 4 at 4096; 64-147 KB), the same tile code.  By shape:
        // 4 columns (chain 2048 x 16384: 474 us against 503 with 8; 4096 x 8192: 541 us
        // against 549 with 2 and 606 with per-thread loads, which the tuning value 1 keeps)
        if ((samples & 1) == 0 && (reinterpret_cast<uintptr_t>(x) & 15) == 0 && columns != 1) {
            constexpr int NARROW = N == 2048 ? 4 : 2;
            const int ct = columns == NARROW || columns == 2 * NARROW ? columns : 4;
            CUtensorMap map;
            if (encode_tensor_map_2d_f32(&map, x, 2ull * samples, (uint64_t)pulses * batch,
                                         (uint64_t)samples * sizeof(float2), 2 * ct, 256))
                return ct == NARROW ? doppler_tma<N, NARROW>(map, pulses, samples, window, out, power, batch, s)
                                    : doppler_tma<N, 2 * NARROW>(map, pulses, samples, window, out, power, batch, s);
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

// ------------------------------------------------------------------ work list

// Group of a work-list CTA: the last group whose first CTA is at or before blockIdx.x.
template <class Params>
__device__ __forceinline__ int wl_group(const Params& p)
{
    int g = 0;
    while (g + 1 < p.groups && (int)blockIdx.x >= p.g[g + 1].entry0) ++g;
    return g;
}

// Work-list resource classes: lengths with up to 16 values per thread (class 0) and with
// 32 (class 1) run in separate launches, so each kernel's registers and shared memory fit
// its own lengths instead of the largest.
constexpr int wl_class(int n) { return elems_for(n) == 32 ? 1 : 0; }

// CTA `local` of a compression group: 256 / T pulses of the group's flattened pulse list
// (CPI q / pulses, pulse q % pulses), the same transform code as pulse_compression_kernel.
template <int N>
__device__ __forceinline__ void wl_compress(const WlCompressionGroup& G, int local, const float2* tw, float2* sm)
{
    using PL = FftPlan<N, elems_for(N)>;
    constexpr int GR = kWlCompressionThreads / PL::T;
    const int q = local * GR + (int)(threadIdx.x / PL::T);
    const bool active = q < G.rows;
    const float2* xr = active ? G.xs[q / G.pulses] + (size_t)(q % G.pulses) * G.samples : nullptr;
    compress_rows<N, elems_for(N), GR>(xr, G.samples, G.spectrum, active ? G.y + (size_t)q * N : nullptr, tw, sm);
}

template <int N, int CLASS>
constexpr size_t wl_compress_smem()
{
    if constexpr (wl_class(N) != CLASS) return 0;
    else return compress_rows_smem<N, elems_for(N), kWlCompressionThreads / FftPlan<N, elems_for(N)>::T>();
}

template <int CLASS>
constexpr size_t wl_compression_smem()
{
    size_t m = 0;
    const size_t s[] = {wl_compress_smem<64, CLASS>(),   wl_compress_smem<128, CLASS>(),
                        wl_compress_smem<256, CLASS>(),  wl_compress_smem<512, CLASS>(),
                        wl_compress_smem<1024, CLASS>(), wl_compress_smem<2048, CLASS>(),
                        wl_compress_smem<4096, CLASS>(), wl_compress_smem<8192, CLASS>()};
    for (size_t v : s) m = v > m ? v : m;
    return m;
}

#define ZKX_WL_CASE(NN, CALL)                               \
    case NN:                                                \
        if constexpr (wl_class(NN) == CLASS) CALL;          \
        break;

// Range compression of every CPI of the work list with a length of this class: one CTA
// per (group, 256 / T pulses) entry, the code path chosen by the group's length.
template <int CLASS>
__global__ void __launch_bounds__(kWlCompressionThreads)
compression_worklist_kernel(const __grid_constant__ WlCompressionParams p, const float2* __restrict__ tw)
{
    extern __shared__ __align__(16) float2 sm[];
    const WlCompressionGroup& G = p.g[wl_group(p)];
    const int local = (int)blockIdx.x - G.entry0;
    switch (G.nfft) {
    ZKX_WL_CASE(64, (wl_compress<64>(G, local, tw, sm)))
    ZKX_WL_CASE(128, (wl_compress<128>(G, local, tw, sm)))
    ZKX_WL_CASE(256, (wl_compress<256>(G, local, tw, sm)))
    ZKX_WL_CASE(512, (wl_compress<512>(G, local, tw, sm)))
    ZKX_WL_CASE(1024, (wl_compress<1024>(G, local, tw, sm)))
    ZKX_WL_CASE(2048, (wl_compress<2048>(G, local, tw, sm)))
    ZKX_WL_CASE(4096, (wl_compress<4096>(G, local, tw, sm)))
    ZKX_WL_CASE(8192, (wl_compress<8192>(G, local, tw, sm)))
    default: break;
    }
}

// CTA `local` of a Doppler group: column tile local % tiles_x of CPI local / tiles_x,
// 256 / T columns, the same tile code as pulse_doppler_tma_kernel; power only.
template <int N>
__device__ __forceinline__ void wl_doppler(const WlDopplerGroup& G, int local, const float2* tw, int* err,
                                           float2* sm)
{
    constexpr int C = kWlDopplerThreads / FftPlan<N, elems_for(N)>::T;
    const int b = local / G.tiles_x;
    const int tile = local - b * G.tiles_x;
    doppler_tma_tile<N, C>(&G.map, G.pulses, G.nr, b, tile * C, G.window, nullptr,
                           G.power + (size_t)b * N * G.nr, tw, err, sm);
}

template <int N, int CLASS>
constexpr size_t wl_doppler_smem_for()
{
    if constexpr (wl_class(N) != CLASS) return 0;
    else return (size_t)doppler_tile_span<N, kWlDopplerThreads / FftPlan<N, elems_for(N)>::T>() * sizeof(float2) + 16;
}

template <int CLASS>
constexpr size_t wl_doppler_smem()
{
    size_t m = 0;
    const size_t s[] = {wl_doppler_smem_for<64, CLASS>(), wl_doppler_smem_for<128, CLASS>(),
                        wl_doppler_smem_for<256, CLASS>(), wl_doppler_smem_for<512, CLASS>(),
                        wl_doppler_smem_for<1024, CLASS>()};
    for (size_t v : s) m = v > m ? v : m;
    return m;
}

// Slow-time transform + window + |.|^2 of every CPI of the work list with a Doppler length
// of this class: one CTA per (group, CPI, column tile) entry.
template <int CLASS>
__global__ void __launch_bounds__(kWlDopplerThreads)
doppler_worklist_kernel(const __grid_constant__ WlDopplerParams p, const float2* __restrict__ tw, int* err)
{
    extern __shared__ __align__(128) float2 sm[];
    const WlDopplerGroup& G = p.g[wl_group(p)];
    const int local = (int)blockIdx.x - G.entry0;
    switch (G.nd) {
    ZKX_WL_CASE(64, (wl_doppler<64>(G, local, tw, err, sm)))
    ZKX_WL_CASE(128, (wl_doppler<128>(G, local, tw, err, sm)))
    ZKX_WL_CASE(256, (wl_doppler<256>(G, local, tw, err, sm)))
    ZKX_WL_CASE(512, (wl_doppler<512>(G, local, tw, err, sm)))
    ZKX_WL_CASE(1024, (wl_doppler<1024>(G, local, tw, err, sm)))
    default: break;
    }
}
#undef ZKX_WL_CASE

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
                                     const float2* spectrum, float2* y, int variant, cudaStream_t stream,
                                     int radix, int ctas_per_sm)
{
    const RowsContiguous src{x, samples};
    if (!is_pow2(nfft)) return launch_compression_any(src, pulses, samples, nfft, spectrum, y, stream);
    if (nfft > (1 << kMaxSmemFftLog))
        return launch_long_compression(src, pulses, samples, nfft, spectrum, y, variant, stream);
    const bool aligned16 = (samples & 1) == 0 && (reinterpret_cast<uintptr_t>(x) & 15) == 0;
#define ZKX_CALL(NN) compression_impl<NN>(src, aligned16, pulses, samples, spectrum, y, variant, radix, ctas_per_sm, stream)
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
                                   int variant, cudaStream_t stream, int radix, int ctas_per_sm)
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
#define ZKX_CALL(NN) compression_impl<NN>(src, aligned16, pulses, samples, spectrum, y, variant, radix, ctas_per_sm, stream)
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

bool wl_compression_length(int n)
{
    return is_pow2(n) && n >= 64 && n <= 8192;
}

int wl_length_class(int n)
{
    return wl_class(n);
}

int wl_compression_ctas(int n, int rows)
{
    const int per = kWlCompressionThreads / (n / elems_for(n));
    return (int)(((long long)rows + per - 1) / per);
}

template <int CLASS>
int compression_worklist_launch(const WlCompressionParams& p, int ctas, cudaStream_t stream)
{
    constexpr size_t smem = wl_compression_smem<CLASS>();
    auto k = compression_worklist_kernel<CLASS>;
    ZKX_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k<<<ctas, kWlCompressionThreads, smem, stream>>>(p, twiddle_table());
    ZKX_LAUNCHED("compression_worklist_kernel");
    return ZKX_SUCCESS;
}

int launch_compression_worklist(const WlCompressionParams& p, int ctas, int cls, cudaStream_t stream)
{
    if (!twiddle_table()) return fail(ZKX_INTERNAL_ERROR, "twiddle table not initialised on this device");
    return cls == 0 ? compression_worklist_launch<0>(p, ctas, stream) : compression_worklist_launch<1>(p, ctas, stream);
}

bool wl_doppler_length(int n)
{
    return is_pow2(n) && n >= 64 && n <= 1024;
}

int wl_doppler_columns(int n)
{
    return kWlDopplerThreads / (n / elems_for(n));
}

int wl_doppler_box_rows(int n)
{
    return n < 256 ? n : 256;
}

template <int CLASS>
int doppler_worklist_launch(const WlDopplerParams& p, int ctas, cudaStream_t stream)
{
    constexpr size_t smem = wl_doppler_smem<CLASS>();
    auto k = doppler_worklist_kernel<CLASS>;
    ZKX_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k<<<ctas, kWlDopplerThreads, smem, stream>>>(p, twiddle_table(), kernel_error_word());
    ZKX_LAUNCHED("doppler_worklist_kernel");
    return ZKX_SUCCESS;
}

int launch_doppler_worklist(const WlDopplerParams& p, int ctas, int cls, cudaStream_t stream)
{
    if (!twiddle_table()) return fail(ZKX_INTERNAL_ERROR, "twiddle table not initialised on this device");
    return cls == 0 ? doppler_worklist_launch<0>(p, ctas, stream) : doppler_worklist_launch<1>(p, ctas, stream);
}

int compression_alt_radix(int nfft)
{
    return is_pow2(nfft) ? alt_compression_radix(nfft) : 0;
}

}  // namespace zkx
