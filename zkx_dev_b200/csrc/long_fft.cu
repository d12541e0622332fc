// Range transforms longer than one CTA's shared memory (N = 32768 and 65536) for
// sm_100a.  N = R * M with M = 16384: the R CTAs of a thread-block cluster (R = 2 or
// 4) each hold one M-point sub-transform in shared memory and registers (512 threads x
// 32 values, the same plan as the single-CTA 16384-point transform), and the radix-R
// butterflies between the sub-transforms are exchanged through distributed shared
// memory:
//
//   forward (decimation in frequency):
//     b_k1[n2]       = W_N^(n2 k1) sum_n1 x[n1 M + n2] W_R^(n1 k1)      (cross-CTA pass)
//     X[k1 + R k2]   = sum_n2 b_k1[n2] W_M^(n2 k2)          in CTA k1   (local transform)
//   inverse (decimation in time), CTA k1 holds Y[k1 + R k2]:
//     z_k1[m]        = W_N^(-m k1) sum_k2 Y[k1 + R k2] W_M^(-m k2)     (local transform)
//     y[c M + m]     = sum_k1 W_R^(-c k1) z_k1[m]                       (cross-CTA pass)
//
// Each cross-CTA pass splits the M positions into R slices of S = M / R: the CTA that
// owns a slice computes the whole R-point butterfly for it and pushes every result
// straight into the shared memory of the CTA that needs it (remote stores, which do
// not stall the sender), so each value crosses the SM-to-SM network at most once per
// pass and the input and output cross HBM exactly once.  Range compression keeps the
// spectrum in "cluster order" (bin k1 + R k2 at k1 M + k2) and never reorders.
#include <algorithm>

#include <cooperative_groups.h>

#include "fft_core.cuh"
#include "fft_local.cuh"
#include "tma.cuh"
#include "window.cuh"
#include "zkx_internal.h"

namespace cg = cooperative_groups;

namespace zkx {
namespace {

using SubPlan = FftPlan<1 << kMaxSmemFftLog, 32>;
constexpr int kM = SubPlan::N;
constexpr int kT = SubPlan::T;
constexpr int kE = SubPlan::E;

// 32-bit shared::cluster address of `p` (this CTA's shared memory) in cluster CTA `rank`.
__device__ __forceinline__ uint32_t cluster_address(const void* p, int rank)
{
    const uint32_t local = (uint32_t)__cvta_generic_to_shared(p);
    uint32_t remote;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(remote) : "r"(local), "r"(rank));
    return remote;
}

__device__ __forceinline__ void store_cluster(uint32_t address, float2 v)
{
    asm volatile("st.shared::cluster.v2.f32 [%0], {%1, %2};" ::"r"(address), "f"(v.x), "f"(v.y)
                 : "memory");
}

// exp(DIR * 2 pi i j / N) for N = R * M, from the FP64-generated 65536-entry table.
template <int R, int DIR>
__device__ __forceinline__ float2 long_twiddle(const float2* __restrict__ tw, int j)
{
    constexpr int LOGN = kMaxSmemFftLog + ilog2(R);
    const float2 w = __ldg(&tw[((unsigned)j << (kTwiddleLog - LOGN)) & (kTwiddleSize - 1)]);
    return DIR > 0 ? cconj(w) : w;
}

// Cross-CTA decimation-in-frequency pass.  CTA c owns n2 in [c S, c S + S): it reads
// x[n1 M + n2] for every n1 through `load(index)` and stores b_k1[n2] into sm[n2] of
// cluster CTA k1.  On return (after a cluster barrier) sm[n2] of this CTA holds its
// own b[n2] for all n2.
template <int R, int DIR, class Load>
__device__ __forceinline__ void cross_dif_scatter(const cg::cluster_group& cl, float2* sm, int c,
                                                  int t, const float2* __restrict__ tw, Load load)
{
    constexpr int S = kM / R, PER = S / kT;
    uint32_t dst[R];
#pragma unroll
    for (int k = 0; k < R; ++k) dst[k] = cluster_address(sm, k);
    cl.sync();  // every CTA of the cluster is running before its shared memory is written
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        const int n2 = c * S + t + kT * j;
        float2 a[R];
#pragma unroll
        for (int n1 = 0; n1 < R; ++n1) a[n1] = load(n1 * kM + n2);
        dft<R, DIR>(a);
#pragma unroll
        for (int k1 = 0; k1 < R; ++k1)
            store_cluster(dst[k1] + 8u * n2, k1 ? cmul(a[k1], long_twiddle<R, DIR>(tw, n2 * k1)) : a[k1]);
    }
    cl.sync();  // all of this CTA's b values have arrived
}

// Cross-CTA decimation-in-time pass after the local inverse sub-transforms: v[r] of
// CTA k1 holds z_k1[m] (before its twiddle), m = t + T r.  Slice s of every z_k1 goes
// to CTA s, which writes y[c M + m] = scale * sum_k1 W_R^(DIR c k1) W_N^(DIR m k1) z_k1[m]
// for its m and every c.
template <int R, int DIR>
__device__ __forceinline__ void cross_dit_gather(const cg::cluster_group& cl, const float2 (&v)[kE],
                                                 float2* sm, int k1, int t,
                                                 const float2* __restrict__ tw, float2* yr,
                                                 float scale)
{
    constexpr int S = kM / R, PER = S / kT;
    uint32_t dst[R];
#pragma unroll
    for (int k = 0; k < R; ++k) dst[k] = cluster_address(sm, k);
    cl.sync();  // every CTA has finished its local transform: exchange buffers are free
#pragma unroll
    for (int r = 0; r < kE; ++r) {
        const int m = t + kT * r;
        const float2 zv = k1 ? cmul(v[r], long_twiddle<R, DIR>(tw, m * k1)) : v[r];
        store_cluster(dst[r / PER] + 8u * (k1 * S + t + kT * (r % PER)), zv);
    }
    cl.sync();
#pragma unroll
    for (int j = 0; j < PER; ++j) {
        const int mm = t + kT * j;
        float2 a[R];
#pragma unroll
        for (int k = 0; k < R; ++k) a[k] = sm[k * S + mm];
        dft<R, DIR>(a);
#pragma unroll
        for (int c = 0; c < R; ++c) {
            float2 o = a[c];
            if (scale != 1.0f) o = make_float2(o.x * scale, o.y * scale);
            yr[(size_t)c * kM + k1 * S + mm] = o;
        }
    }
}

// After a forward-ordered local transform CTA k1 holds X[k1 + R k2] in v[r]
// (k2 = t + T r); bin k belongs to output chunk k / M, which receives it through its
// shared memory and writes the chunk in natural order.
template <int R>
__device__ __forceinline__ void cross_natural_scatter(const cg::cluster_group& cl,
                                                      const float2 (&v)[kE], float2* sm, int k1,
                                                      int t, float2* yr, float scale)
{
    constexpr int S = kM / R, PER = S / kT;
    uint32_t dst[R];
#pragma unroll
    for (int k = 0; k < R; ++k) dst[k] = cluster_address(sm, k);
    cl.sync();
#pragma unroll
    for (int r = 0; r < kE; ++r)
        store_cluster(dst[r / PER] + 8u * (k1 + R * (t + kT * (r % PER))), v[r]);
    cl.sync();
    float2* out = yr + (size_t)k1 * kM;
#pragma unroll
    for (int r = 0; r < kE; ++r) {
        float2 o = sm[t + kT * r];
        if (scale != 1.0f) o = make_float2(o.x * scale, o.y * scale);
        out[t + kT * r] = o;
    }
}

// Twiddles of the cross-CTA passes of one CTA of the persistent kernel, the same for every
// pulse it transforms.  Clusters of two take the forward pass on position pairs (PAIRED:
// 128-bit loads and remote stores; measured 1.7-2% faster at 32768 points, 4-5% slower at
// 65536 with clusters of four, which keep single positions).  Forward pass, position
// n2 = c S + P (t + T j) (+1 for the pair's second, P = 2 when PAIRED, else 1):
// W_N^(n2 k1) = base[k1 - 1] (base1 for the second) * step[j (R - 1) + k1 - 1] with
// base = W_N^((c S + P t) k1), base1 = W_N^((c S + P t + 1) k1) per thread and
// step = W_N^(P T j k1) shared.  Inverse pass of CTA k1: W_N^(-m k1) for m = t + T r is
// ibase * istep[r] with ibase = W_N^(-t k1), istep = W_N^(-T r k1).  One complex product
// replaces a table load per value (the product differs from the table value by about one
// unit in the last place).
template <int R>
struct CrossTwiddles {
    static constexpr bool PAIRED = R == 2;
    static constexpr int P = PAIRED ? 2 : 1;
    static constexpr int PER = kM / R / kT;
    static constexpr int STEP = PER / P * (R - 1);   // forward steps
    static constexpr int WORDS = STEP + kE;           // shared words (forward + inverse steps)
    float2 base[R - 1];
    float2 base1[R - 1];
    float2 ibase;
};

// Fill the shared steps (all threads) and this thread's bases.
template <int R>
__device__ __forceinline__ void cross_twiddles_init(CrossTwiddles<R>& c, float2* steps, int k1, int t,
                                                    const float2* __restrict__ tw)
{
    using CT = CrossTwiddles<R>;
    for (int i = t; i < CT::STEP; i += kT) {
        const int j = i / (R - 1), k = i - j * (R - 1) + 1;
        steps[i] = long_twiddle<R, -1>(tw, CT::P * kT * j * k);
    }
    for (int r = t; r < kE; r += kT) steps[CT::STEP + r] = long_twiddle<R, 1>(tw, kT * r * k1);
#pragma unroll
    for (int k = 1; k < R; ++k) {
        c.base[k - 1] = long_twiddle<R, -1>(tw, (k1 * (kM / R) + CT::P * t) * k);
        c.base1[k - 1] = long_twiddle<R, -1>(tw, (k1 * (kM / R) + CT::P * t + 1) * k);
    }
    c.ibase = long_twiddle<R, 1>(tw, t * k1);
}

__device__ __forceinline__ void store_cluster2(uint32_t address, float2 a, float2 b)
{
    asm volatile("st.shared::cluster.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(address), "f"(a.x), "f"(a.y),
                 "f"(b.x), "f"(b.y)
                 : "memory");
}

// cross_dif_scatter (forward, DIR -1) with the twiddles of cross_twiddles_init.  load2(e)
// returns elements e and e + 1 as one float4 (only .x, .y used for single positions).
template <int R, class Load2>
__device__ __forceinline__ void cross_dif_scatter_tw(const cg::cluster_group& cl, float2* sm, int c, int t,
                                                     const CrossTwiddles<R>& ct, const float2* steps, Load2 load2)
{
    using CT = CrossTwiddles<R>;
    constexpr int S = kM / R, PER = S / kT;
    static_assert(PER % CT::P == 0, "position pairs");
    uint32_t dst[R];
#pragma unroll
    for (int k = 0; k < R; ++k) dst[k] = cluster_address(sm, k);
    cl.sync();  // every CTA of the cluster is running before its shared memory is written
#pragma unroll
    for (int j = 0; j < PER / CT::P; ++j) {
        const int n2 = c * S + CT::P * (t + kT * j);
        float2 a[R], b[R];
#pragma unroll
        for (int n1 = 0; n1 < R; ++n1) {
            const float4 q = load2(n1 * kM + n2);
            a[n1] = make_float2(q.x, q.y);
            b[n1] = make_float2(q.z, q.w);
        }
        dft<R, -1>(a);
        if constexpr (CT::PAIRED) {
            dft<R, -1>(b);
            store_cluster2(dst[0] + 8u * n2, a[0], b[0]);
#pragma unroll
            for (int k1 = 1; k1 < R; ++k1) {
                const float2 st = steps[j * (R - 1) + k1 - 1];
                store_cluster2(dst[k1] + 8u * n2, cmul(a[k1], cmul(ct.base[k1 - 1], st)),
                               cmul(b[k1], cmul(ct.base1[k1 - 1], st)));
            }
        } else {
            store_cluster(dst[0] + 8u * n2, a[0]);
#pragma unroll
            for (int k1 = 1; k1 < R; ++k1)
                store_cluster(dst[k1] + 8u * n2, cmul(a[k1], cmul(ct.base[k1 - 1], steps[j * (R - 1) + k1 - 1])));
        }
    }
    cl.sync();  // all of this CTA's b values have arrived
}

// cross_dit_gather (inverse, DIR +1, unscaled) with the twiddles of cross_twiddles_init; with
// PAIRED the final butterflies take position pairs (128-bit shared loads, and 128-bit stores
// when yr is 16-byte aligned).
template <int R>
__device__ __forceinline__ void cross_dit_gather_tw(const cg::cluster_group& cl, const float2 (&v)[kE], float2* sm,
                                                    int k1, int t, const CrossTwiddles<R>& ct, const float2* steps,
                                                    float2* yr)
{
    using CT = CrossTwiddles<R>;
    constexpr int S = kM / R, PER = S / kT;
    const float2* istep = steps + CT::STEP;
    uint32_t dst[R];
#pragma unroll
    for (int k = 0; k < R; ++k) dst[k] = cluster_address(sm, k);
    cl.sync();  // every CTA has finished its local transform: exchange buffers are free
#pragma unroll
    for (int r = 0; r < kE; ++r) {
        const float2 zv = k1 ? cmul(v[r], cmul(ct.ibase, istep[r])) : v[r];
        store_cluster(dst[r / PER] + 8u * (k1 * S + t + kT * (r % PER)), zv);
    }
    cl.sync();
    if constexpr (CT::PAIRED) {
        const bool pairs = (reinterpret_cast<uintptr_t>(yr) & 15) == 0;
#pragma unroll
        for (int j = 0; j < PER / 2; ++j) {
            const int mm = 2 * (t + kT * j);
            float2 a[R], b[R];
#pragma unroll
            for (int k = 0; k < R; ++k) {
                const float4 q = *reinterpret_cast<const float4*>(&sm[k * S + mm]);
                a[k] = make_float2(q.x, q.y);
                b[k] = make_float2(q.z, q.w);
            }
            dft<R, 1>(a);
            dft<R, 1>(b);
#pragma unroll
            for (int c = 0; c < R; ++c) {
                float2* o = yr + (size_t)c * kM + k1 * S + mm;
                if (pairs) {
                    *reinterpret_cast<float4*>(o) = make_float4(a[c].x, a[c].y, b[c].x, b[c].y);
                } else {
                    o[0] = a[c];
                    o[1] = b[c];
                }
            }
        }
    } else {
#pragma unroll
        for (int j = 0; j < PER; ++j) {
            const int mm = t + kT * j;
            float2 a[R];
#pragma unroll
            for (int k = 0; k < R; ++k) a[k] = sm[k * S + mm];
            dft<R, 1>(a);
#pragma unroll
            for (int c = 0; c < R; ++c) yr[(size_t)c * kM + k1 * S + mm] = a[c];
        }
    }
}

// v[r] = sm[t + T r], then a block barrier so the local transform may reuse sm.
__device__ __forceinline__ void take_own(float2 (&v)[kE], const float2* sm, int t)
{
#pragma unroll
    for (int r = 0; r < kE; ++r) v[r] = sm[t + kT * r];
    __syncthreads();
}

// Replica spectrum in cluster order: spectrum[k1 M + k2] = conj(H[k1 + R k2]) / N with
// H = FFT(w h / ||w h||, N); the FP64 norm runs over all `length` samples
// (radartools_typed.cpp:639-648) and is recomputed by each CTA of the cluster.
template <int R>
__global__ void __cluster_dims__(R, 1, 1) __launch_bounds__(kT, 1)
long_replica_kernel(const float2* __restrict__ h, int length, int normalize, int window_kind,
                    const float* __restrict__ explicit_window, float2* __restrict__ spectrum,
                    const float2* __restrict__ tw)
{
    extern __shared__ __align__(16) float2 sm[];
    __shared__ double partial[kT];
    const cg::cluster_group cl = cg::this_cluster();
    const int k1 = (int)cl.block_rank();
    const int t = threadIdx.x;
    constexpr int N = R * kM;
    double acc = 0.0;
    for (int i = t; i < length; i += kT) {
        const double w = window_value(window_kind, explicit_window, i, length);
        const float2 hv = h[i];
        const double re = (double)hv.x * w, im = (double)hv.y * w;
        acc += re * re + im * im;
    }
    partial[t] = acc;
    __syncthreads();
    if (t == 0) {
        double total = 0.0;
        for (int i = 0; i < kT; ++i) total += partial[i];
        partial[0] = total;
    }
    __syncthreads();
    const double norm = normalize ? sqrt(partial[0]) : 1.0;
    const float scale = (float)(1.0 / (norm * (double)N));
    cross_dif_scatter<R, -1>(cl, sm, k1, t, tw, [&](int e) {
        float2 val = make_float2(0.f, 0.f);
        if (e < length) {
            const float w = window_value(window_kind, explicit_window, e, length);
            const float2 hv = h[e];
            val = make_float2(hv.x * w, hv.y * w);
        }
        return val;
    });
    float2 v[kE];
    take_own(v, sm, t);
    fft_block<SubPlan, -1, 1>(v, sm, t, tw);
    float2* out = spectrum + (size_t)k1 * kM;
#pragma unroll
    for (int r = 0; r < kE; ++r) out[t + kT * r] = make_float2(v[r].x * scale, -v[r].y * scale);
}

// One pulse per cluster: cross-CTA pass on the pulse (zero-padded/truncated to N),
// local forward transform, product with the cluster-order spectrum, local inverse
// transform, cross-CTA pass and store.
//
// One CTA per SM and no pulse loop, so nothing hides a CTA's loads behind another's
// work.  Each CTA therefore starts by pulling its slice of pulse `pulse + ahead` (the
// pulse this SM's next cluster is due to take, ahead = resident clusters) into L2, so
// that cluster's loads hit L2 instead of HBM (512 x 32768: 215.5 -> 205.3 us, 2048 x
// 65536: 1764 -> 1702 us; two or three generations ahead were slower than none).
template <int R, class Src>
__global__ void __cluster_dims__(R, 1, 1) __launch_bounds__(kT, 1)
long_compression_kernel(const Src src, int pulses, int samples,
                        const float2* __restrict__ spectrum, float2* __restrict__ y,
                        const float2* __restrict__ tw, int ahead)
{
    extern __shared__ __align__(16) float2 sm[];
    const cg::cluster_group cl = cg::this_cluster();
    const int k1 = (int)cl.block_rank();
    const int t = threadIdx.x;
    const size_t pulse = blockIdx.x / R;
    constexpr int N = R * kM;
    const int avail = samples < N ? samples : N;
    if (t < R && ahead > 0 && pulse + ahead < (size_t)pulses) {
        // chunk n1 = t of the slice this CTA reads: [t M + k1 S, t M + k1 S + S) within the
        // row's `avail` samples, whole 16-byte words of a 16-byte aligned row only
        constexpr int S = kM / R;
        const float2* nx = src.row((int)(pulse + ahead));
        const int lo = t * kM + k1 * S;
        const int hi = (lo + S < avail ? lo + S : avail) & ~1;
        if (hi > lo && (reinterpret_cast<uintptr_t>(nx) & 15) == 0)
            bulk_prefetch_l2(nx + lo, (uint32_t)(hi - lo) * (uint32_t)sizeof(float2));
    }
    const float2* xr = src.row((int)pulse);
    cross_dif_scatter<R, -1>(cl, sm, k1, t, tw,
                             [&](int e) { return e < avail ? __ldcs(&xr[e]) : make_float2(0.f, 0.f); });
    float2 v[kE];
    take_own(v, sm, t);
    fft_block<SubPlan, -1, 1>(v, sm, t, tw);
    const float2* sp = spectrum + (size_t)k1 * kM;
#pragma unroll
    for (int r = 0; r < kE; ++r) v[r] = cmul(v[r], __ldg(&sp[t + kT * r]));
    __syncthreads();
    fft_block<SubPlan, 1, 1>(v, sm, t, tw);
    cross_dit_gather<R, 1>(cl, v, sm, k1, t, tw, y + pulse * (size_t)N, 1.0f);
}

// Persistent form of the kernel above: each cluster walks pulses cluster, +clusters, ...
// (clusters = the clusters resident on the GPU), so the per-CTA set-up happens once: the
// local sub-transform uses the four-step ordering of fft_local.cuh (one block-wide exchange
// per direction), and the CTA's slice of the cluster-order spectrum sits in tensor memory
// in the digit-reversed order that ordering leaves in registers (tcgen05.st once,
// tcgen05.ld per pulse: 256 columns, one CTA per SM).  At the start of each pulse every
// CTA pulls its slice of the cluster's next pulse into L2, so that pulse's cross-CTA pass
// reads L2.  The cross-CTA passes are those above with their twiddles formed from
// per-thread bases and shared steps set up once (CrossTwiddles) instead of table loads per
// value; their cluster barriers also order one pulse's last reads of shared memory before
// the next pulse's remote writes.
template <int R, class Src>
__global__ void __cluster_dims__(R, 1, 1) __launch_bounds__(kT, 1)
long_compression_local_kernel(const Src src, int pulses, int samples, const float2* __restrict__ spectrum,
                              float2* __restrict__ y, const float2* __restrict__ tw)
{
    using LP = LocalPlan<kM>;
    static_assert(LP::T == kT && LP::E == kE, "the local plan of the 16384-point sub-transform");
    constexpr int LOGE = ilog2(kE);
    constexpr uint32_t kCols = (kT / 128) * 2 * kE;
    constexpr int N = R * kM;
    constexpr int S = kM / R;
    extern __shared__ __align__(128) float2 sm[];
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + LP::EXCHANGE);
    float2* tab = sm + LP::EXCHANGE + 2;
    const cg::cluster_group cl = cg::this_cluster();
    const int k1 = (int)cl.block_rank();
    const int t = threadIdx.x;
    const int warp = t >> 5;
    const int cluster = (int)(blockIdx.x / R), clusters = (int)(gridDim.x / R);
    const int avail = samples < N ? samples : N;
    if (warp == 0) {
        tmem_alloc(tmem_slot, kCols);
        tmem_relinquish();
    }
    float2* first = tab + LP::TABLE + t * (LOGE | 1);
    float2* steps = tab + LP::TABLE + kT * (LOGE | 1);   // CrossTwiddles<R>::WORDS
    CrossTwiddles<R> ct;
    cross_twiddles_init<R>(ct, steps, k1, t, tw);
    fill_local_table<LP>(tab, t, kT, tw);
    {
        float2 wb[LOGE];
        load_twiddle_bases<kE, LP::LOGN>(wb, t, tw);
#pragma unroll
        for (int b = 0; b < LOGE; ++b) first[b] = wb[b];
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;
    const uint32_t spec_cols = tmem_base + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(warp >> 2) * (2 * kE);
    spectrum_to_tmem<LP>(spectrum + (size_t)k1 * kM, t, spec_cols);
    auto twiddle = [&](float2(&x)[kE]) { apply_twiddles_from<kE, -1>(x, first); };
    auto twiddle_conj = [&](float2(&x)[kE]) { apply_twiddles_from<kE, 1>(x, first); };
    for (int pulse = cluster; pulse < pulses; pulse += clusters) {
        if (t < R && pulse + clusters < pulses) {
            // chunk n1 = t of the slice this CTA reads next: [t M + k1 S, t M + k1 S + S) within
            // the row's `avail` samples, whole 16-byte words of a 16-byte aligned row only
            const float2* nx = src.row(pulse + clusters);
            const int lo = t * kM + k1 * S;
            const int hi = (lo + S < avail ? lo + S : avail) & ~1;
            if (hi > lo && (reinterpret_cast<uintptr_t>(nx) & 15) == 0)
                bulk_prefetch_l2(nx + lo, (uint32_t)(hi - lo) * (uint32_t)sizeof(float2));
        }
        const float2* xr = src.row(pulse);
        const bool aligned = (reinterpret_cast<uintptr_t>(xr) & 15) == 0;
        cross_dif_scatter_tw<R>(cl, sm, k1, t, ct, steps, [&](int e) {
            if constexpr (CrossTwiddles<R>::PAIRED) {
                if (aligned && e + 1 < avail) return __ldcs(reinterpret_cast<const float4*>(xr + e));
                const float2 u = e < avail ? __ldcs(&xr[e]) : make_float2(0.f, 0.f);
                const float2 w = e + 1 < avail ? __ldcs(&xr[e + 1]) : make_float2(0.f, 0.f);
                return make_float4(u.x, u.y, w.x, w.y);
            } else {
                const float2 u = e < avail ? __ldcs(&xr[e]) : make_float2(0.f, 0.f);
                return make_float4(u.x, u.y, 0.f, 0.f);
            }
        });
        float2 v[kE];
        take_own(v, sm, t);
        local_fft_forward<LP>(v, sm, t, twiddle, tab);
        tmem_multiply<kE, false>(v, spec_cols);
        local_fft_inverse<LP>(v, sm, t, twiddle_conj, tab);
        cross_dit_gather_tw<R>(cl, v, sm, k1, t, ct, steps, y + (size_t)pulse * N);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem_base, kCols);
    }
}

// Batched C2C rows of length N, natural order in and out; forward unnormalised,
// inverse scaled by 1/N.  Every CTA reads its input slice before the second cluster
// barrier and writes only after later ones, so x == y is safe.
template <int R, int DIR>
__global__ void __cluster_dims__(R, 1, 1) __launch_bounds__(kT, 1)
long_fft_rows_kernel(const float2* x, float2* y, const float2* __restrict__ tw)
{
    extern __shared__ __align__(16) float2 sm[];
    const cg::cluster_group cl = cg::this_cluster();
    const int k1 = (int)cl.block_rank();
    const int t = threadIdx.x;
    const size_t row = blockIdx.x / R;
    constexpr int N = R * kM;
    const float2* xr = x + row * (size_t)N;
    cross_dif_scatter<R, DIR>(cl, sm, k1, t, tw, [&](int e) { return xr[e]; });
    float2 v[kE];
    take_own(v, sm, t);
    fft_block<SubPlan, DIR, 1>(v, sm, t, tw);
    cross_natural_scatter<R>(cl, v, sm, k1, t, y + row * (size_t)N, DIR > 0 ? 1.0f / (float)N : 1.0f);
}

constexpr size_t kSmemBytes = (size_t)SubPlan::smem_elems() * sizeof(float2);

template <class K>
int prepare(K kernel)
{
    if (!twiddle_table()) return fail(ZKX_INTERNAL_ERROR, "twiddle table not initialised on this device");
    ZKX_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes));
    return ZKX_SUCCESS;
}

template <int R>
int replica_long(const float2* h, int length, int normalize, int kind, const float* w,
                 float2* spectrum, cudaStream_t s)
{
    auto k = long_replica_kernel<R>;
    ZKX_TRY(prepare(k));
    k<<<R, kT, kSmemBytes, s>>>(h, length, normalize, kind, w, spectrum, twiddle_table());
    ZKX_LAUNCHED("long_replica_kernel");
    return ZKX_SUCCESS;
}

constexpr size_t kLocalSmemBytes =
    ((size_t)LocalPlan<kM>::EXCHANGE + 2 + LocalPlan<kM>::TABLE + (size_t)kT * (ilog2(kE) | 1) +
     (size_t)std::max(CrossTwiddles<2>::WORDS, CrossTwiddles<4>::WORDS)) * sizeof(float2);

// Clusters of the persistent kernel resident on the GPU at once.
template <int R>
int local_long_clusters(int* clusters)
{
    auto k = long_compression_local_kernel<R, RowsContiguous>;
    ZKX_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kLocalSmemBytes));
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(R);
    cfg.blockDim = dim3(kT);
    cfg.dynamicSmemBytes = kLocalSmemBytes;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = R;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    ZKX_CUDA(cudaOccupancyMaxActiveClusters(clusters, k, &cfg));
    *clusters = std::max(1, *clusters);
    return ZKX_SUCCESS;
}

// The default: the persistent kernel once every resident cluster gets at least four pulses,
// one cluster per pulse below that (measured chain times: 2048 x 65536 2940 vs 3120 us,
// 512 x 32768 324 vs 329 us; 64 x 65536 114 vs 106 us, 256 x 32768 192 vs 189 us).
int long_default_variant(int pulses, int clusters)
{
    return pulses >= 4 * clusters ? ZKX_COMPRESSION_LOCAL : ZKX_COMPRESSION_PERSISTENT;
}

template <int R, class Src>
int compression_long(const Src& x, int pulses, int samples, const float2* spectrum, float2* y,
                     int variant, cudaStream_t s)
{
    if (!twiddle_table()) return fail(ZKX_INTERNAL_ERROR, "twiddle table not initialised on this device");
    int clusters = 1;
    if (variant == ZKX_COMPRESSION_DEFAULT || variant == ZKX_COMPRESSION_LOCAL) {
        ZKX_TRY(local_long_clusters<R>(&clusters));
        if (variant == ZKX_COMPRESSION_DEFAULT) variant = long_default_variant(pulses, clusters);
    }
    if (variant == ZKX_COMPRESSION_LOCAL) {
        auto k = long_compression_local_kernel<R, Src>;
        ZKX_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kLocalSmemBytes));
        clusters = std::max(1, std::min(pulses, clusters));
        k<<<(unsigned)clusters * R, kT, kLocalSmemBytes, s>>>(x, pulses, samples, spectrum, y, twiddle_table());
        ZKX_LAUNCHED("long_compression_local_kernel");
        return ZKX_SUCCESS;
    }
    auto k = long_compression_kernel<R, Src>;
    ZKX_TRY(prepare(k));
    int dev = 0, sms = 0;
    ZKX_CUDA(cudaGetDevice(&dev));
    ZKX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    k<<<(unsigned)pulses * R, kT, kSmemBytes, s>>>(x, pulses, samples, spectrum, y, twiddle_table(),
                                                   sms / R);
    ZKX_LAUNCHED("long_compression_kernel");
    return ZKX_SUCCESS;
}

template <int R, int DIR>
int fft_rows_long(const float2* x, int rows, float2* y, cudaStream_t s)
{
    auto k = long_fft_rows_kernel<R, DIR>;
    ZKX_TRY(prepare(k));
    k<<<(unsigned)rows * R, kT, kSmemBytes, s>>>(x, y, twiddle_table());
    ZKX_LAUNCHED("long_fft_rows_kernel");
    return ZKX_SUCCESS;
}

int unsupported() { return fail(ZKX_UNSUPPORTED_OPERATION, "transform length above 65536"); }

}  // namespace

int launch_long_replica_spectrum(const float2* replica, int length, int nfft, int normalize,
                                 int window_kind, const float* explicit_window, float2* spectrum,
                                 cudaStream_t stream)
{
    if (nfft == 2 * kM) return replica_long<2>(replica, length, normalize, window_kind, explicit_window, spectrum, stream);
    if (nfft == 4 * kM) return replica_long<4>(replica, length, normalize, window_kind, explicit_window, spectrum, stream);
    return unsupported();
}

template <class Src>
int long_compression(const Src& x, int pulses, int samples, int nfft, const float2* spectrum,
                     float2* y, int variant, cudaStream_t stream)
{
    if (nfft == 2 * kM) return compression_long<2>(x, pulses, samples, spectrum, y, variant, stream);
    if (nfft == 4 * kM) return compression_long<4>(x, pulses, samples, spectrum, y, variant, stream);
    return unsupported();
}

int resolve_long_compression_variant(int pulses, int nfft, int* resolved)
{
    int clusters = 1;
    if (nfft == 2 * kM) ZKX_TRY(local_long_clusters<2>(&clusters));
    else if (nfft == 4 * kM) ZKX_TRY(local_long_clusters<4>(&clusters));
    else return unsupported();
    *resolved = long_default_variant(pulses, clusters);
    return ZKX_SUCCESS;
}

int launch_long_compression(const RowsContiguous& x, int pulses, int samples, int nfft,
                            const float2* spectrum, float2* y, int variant, cudaStream_t stream)
{
    return long_compression(x, pulses, samples, nfft, spectrum, y, variant, stream);
}

int launch_long_compression(const RowsTable& x, int pulses, int samples, int nfft,
                            const float2* spectrum, float2* y, int variant, cudaStream_t stream)
{
    return long_compression(x, pulses, samples, nfft, spectrum, y, variant, stream);
}

int launch_long_fft_rows(const float2* x, int rows, int n, int inverse, float2* y,
                         cudaStream_t stream)
{
    if (n == 2 * kM) return inverse ? fft_rows_long<2, 1>(x, rows, y, stream) : fft_rows_long<2, -1>(x, rows, y, stream);
    if (n == 4 * kM) return inverse ? fft_rows_long<4, 1>(x, rows, y, stream) : fft_rows_long<4, -1>(x, rows, y, stream);
    return unsupported();
}

}  // namespace zkx
