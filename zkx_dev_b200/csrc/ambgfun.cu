// ambgfun: the normalised ambiguity function of x against y (y = x by default) and its
// delay and Doppler cuts, with the semantics of the reference's ambgfun_typed_cpu /
// ambgfun_device (radartools_typed.cpp:330-463; device path radartools_typed.cu:30-126):
//
//   2-D    out[r][s]   = | sum_c ŷ[c] conj(x̂[c - (nx-1) + r]) exp(+2 pi i f c / F) |,
//                        f = (s - F/2) mod F, r < nx + ny - 1, F = next pow2(nx + ny - 1)
//   delay  out[i]      = F |IDFT_F( ŷ conj(x_shift) )[(i + F/2) mod F]|, x_shift =
//                        IDFT_F( DFT_F(x̂) exp(2 pi i (-fs/2 + fs k/F) cut_value) )
//   Doppler out[i]     = | c[(i - rows/2) mod rows] |, c the circular cross-correlation of
//                        ŷ with x̂ exp(2 pi i cut_value n / fs) over rows = nx + ny - 1
//
// where x̂ = x / ||x||, ŷ = y / ||y|| with the norms over the whole arrays (only the first
// nx / ny samples enter the sums).  The 2-D cut runs one shared-memory FFT per delay row,
// fused with building the delayed product and the shifted magnitude (one HBM write per
// output value).  Because rows >= nx + ny - 1 leaves no circular wrap, the Doppler cut's
// rows-point correlation equals the linear correlation, which a zero-padded power-of-two
// transform of length F gives exactly; its lags are mapped back to the reference's indices.
// Phases are evaluated in FP64 and rounded once.
#include <cmath>
#include <limits>

#include "fft_core.cuh"
#include "zkx_internal.h"

namespace zkx {
namespace {

constexpr int kMaxFusedLog = kMaxSmemFftLog;  // 2-D rows transformed in one CTA up to 16384

// inv[b] = 1 / ||v_b|| over all elements (block 0: x, block 1: y), summed in FP64; a zero
// norm gives NaN, the value the reference's division produces.
__global__ void __launch_bounds__(256) ambgfun_norm_kernel(const float2* __restrict__ x, int x_count,
                                                           const float2* __restrict__ y, int y_count,
                                                           float* __restrict__ inv)
{
    const float2* v = blockIdx.x == 0 ? x : y;
    const int n = blockIdx.x == 0 ? x_count : y_count;
    __shared__ double part[256];
    double acc = 0.0;
    for (int i = threadIdx.x; i < n; i += 256) {
        const float2 a = v[i];
        acc += (double)a.x * a.x + (double)a.y * a.y;
    }
    part[threadIdx.x] = acc;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) part[threadIdx.x] += part[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double nrm = sqrt(part[0]);
        inv[blockIdx.x] = nrm == 0.0 ? __int_as_float(0x7fc00000) : (float)(1.0 / nrm);
    }
}

__device__ __forceinline__ float2 delay_product(const float2* __restrict__ x, int nx,
                                                const float2* __restrict__ y, int ny, int row,
                                                int c, float scale)
{
    float2 val = make_float2(0.f, 0.f);
    const int xc = c - (nx - 1) + row;
    if (c < ny && xc >= 0 && xc < nx) {
        const float2 p = cmulc(y[c], x[xc]);
        val = make_float2(p.x * scale, p.y * scale);
    }
    return val;
}

// 2-D cut, G delay rows per CTA: product row -> unnormalised inverse DFT -> |.| at the
// shifted frequency index.
template <int NF, int G>
__global__ void __launch_bounds__(G * FftPlan<NF, elems_for(NF)>::T)
ambgfun_2d_kernel(const float2* __restrict__ x, int nx, const float2* __restrict__ y, int ny,
                  int rows, const float* __restrict__ inv, float* __restrict__ out,
                  const float2* __restrict__ tw)
{
    using PL = FftPlan<NF, elems_for(NF)>;
    extern __shared__ float2 sm[];
    constexpr int S = PL::smem_elems() % 16 == 0 && PL::T < 16 ? PL::smem_elems() + 8 : PL::smem_elems();
    const int g = threadIdx.x / PL::T;
    const int t = threadIdx.x - g * PL::T;
    const int row = blockIdx.x * G + g;
    const bool active = row < rows;
    const float scale = inv[0] * inv[1];
    float2 v[PL::E];
#pragma unroll
    for (int r = 0; r < PL::E; ++r)
        v[r] = active ? delay_product(x, nx, y, ny, row, t + PL::T * r, scale) : make_float2(0.f, 0.f);
    fft_block<PL, 1, 1>(v, sm + g * S, t, tw);
    if (active) {
        float* o = out + (size_t)row * NF;
#pragma unroll
        for (int r = 0; r < PL::E; ++r) {
            const int c = t + PL::T * r;
            __stcs(&o[(c + NF / 2) & (NF - 1)], hypotf(v[r].x, v[r].y));
        }
    }
}

// ---- general path (any power-of-two F up to 65536): elementwise kernels around the
// batched row transforms

__global__ void ambgfun_build_kernel(const float2* __restrict__ x, int nx, const float2* __restrict__ y,
                                     int ny, int rows, int nf, const float* __restrict__ inv,
                                     float2* __restrict__ prod)
{
    const size_t total = (size_t)rows * nf;
    const float scale = inv[0] * inv[1];
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
         i += (size_t)gridDim.x * blockDim.x) {
        const int row = (int)(i / nf), c = (int)(i - (size_t)row * nf);
        prod[i] = delay_product(x, nx, y, ny, row, c, scale);
    }
}

// out[row][(c + F/2) mod F] = factor * |v[row][c]|
__global__ void ambgfun_magnitude_kernel(const float2* __restrict__ v, int rows, int nf, float factor,
                                         float* __restrict__ out)
{
    const size_t total = (size_t)rows * nf;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
         i += (size_t)gridDim.x * blockDim.x) {
        const int row = (int)(i / nf), c = (int)(i - (size_t)row * nf);
        const float2 a = v[i];
        __stcs(&out[(size_t)row * nf + ((c + nf / 2) & (nf - 1))], factor * hypotf(a.x, a.y));
    }
}

// a[e] = e < n ? v[e] * inv * exp(2 pi i cycles_per_sample e) : 0   (FP64 phase)
__global__ void ambgfun_pack_kernel(const float2* __restrict__ v, int n, const float* __restrict__ inv,
                                    int which, double cycles_per_sample, int nf, float2* __restrict__ a)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nf) return;
    float2 r = make_float2(0.f, 0.f);
    if (e < n) {
        const float s = inv[which];
        r = make_float2(v[e].x * s, v[e].y * s);
        if (cycles_per_sample != 0.0) {
            double sn, cs;
            sincospi(2.0 * cycles_per_sample * (double)e, &sn, &cs);
            r = cmul(r, make_float2((float)cs, (float)sn));
        }
    }
    a[e] = r;
}

// a[k] *= exp(2 pi i (-fs/2 + fs k / F) cut_value)   (the delay cut's phase, FP64)
__global__ void ambgfun_delay_phase_kernel(float2* __restrict__ a, int nf, double fs, double cut_value)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nf) return;
    const double f = -0.5 * fs + fs * (double)k / (double)nf;
    double sn, cs;
    sincospi(2.0 * f * cut_value, &sn, &cs);
    a[k] = cmul(a[k], make_float2((float)cs, (float)sn));
}

// dst[e] = (e < n ? v[e] * inv[which] : 0) * conj(b[e])
__global__ void ambgfun_conj_product_kernel(const float2* __restrict__ v, int n,
                                            const float* __restrict__ inv, int which,
                                            const float2* __restrict__ b, int nf,
                                            float2* __restrict__ dst)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nf) return;
    float2 r = make_float2(0.f, 0.f);
    if (e < n) {
        const float s = inv[which];
        r = cmulc(make_float2(v[e].x * s, v[e].y * s), b[e]);
    }
    dst[e] = r;
}

// dst[e] = a[e] * conj(b[e])  (dst may be a or b)
__global__ void ambgfun_spectrum_product_kernel(const float2* a, const float2* b, int nf, float2* dst)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < nf) dst[e] = cmulc(a[e], b[e]);
}

// Doppler cut: correlation lag of bin e (0 .. ny-1 positive, F-nx+1 .. F-1 negative) to the
// reference's rows-point index, then |.| at (j + rows/2) mod rows.
__global__ void ambgfun_doppler_out_kernel(const float2* __restrict__ c, int nx, int ny, int nf,
                                           float* __restrict__ out)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nf) return;
    const int rows = nx + ny - 1;
    int j;
    if (e < ny) j = e;
    else if (e >= nf - nx + 1) j = e - nf + rows;
    else return;
    const float2 a = c[e];
    out[(j + rows / 2) % rows] = hypotf(a.x, a.y);
}

template <int NF>
int ambgfun_2d_fused(const float2* x, int nx, const float2* y, int ny, int rows, const float* inv,
                     float* out, cudaStream_t s)
{
    using PL = FftPlan<NF, elems_for(NF)>;
    constexpr int G = rows_per_cta(NF);
    constexpr int S = PL::smem_elems() % 16 == 0 && PL::T < 16 ? PL::smem_elems() + 8 : PL::smem_elems();
    const size_t smem = (size_t)G * S * sizeof(float2);
    auto k = ambgfun_2d_kernel<NF, G>;
    ZKX_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k<<<(rows + G - 1) / G, G * PL::T, smem, s>>>(x, nx, y, ny, rows, inv, out, twiddle_table());
    ZKX_LAUNCHED("ambgfun_2d_kernel");
    return ZKX_SUCCESS;
}

int dispatch_2d_fused(int log_nf, const float2* x, int nx, const float2* y, int ny, int rows,
                      const float* inv, float* out, cudaStream_t s)
{
    switch (log_nf) {
    case 0: return ambgfun_2d_fused<1>(x, nx, y, ny, rows, inv, out, s);
    case 1: return ambgfun_2d_fused<2>(x, nx, y, ny, rows, inv, out, s);
    case 2: return ambgfun_2d_fused<4>(x, nx, y, ny, rows, inv, out, s);
    case 3: return ambgfun_2d_fused<8>(x, nx, y, ny, rows, inv, out, s);
    case 4: return ambgfun_2d_fused<16>(x, nx, y, ny, rows, inv, out, s);
    case 5: return ambgfun_2d_fused<32>(x, nx, y, ny, rows, inv, out, s);
    case 6: return ambgfun_2d_fused<64>(x, nx, y, ny, rows, inv, out, s);
    case 7: return ambgfun_2d_fused<128>(x, nx, y, ny, rows, inv, out, s);
    case 8: return ambgfun_2d_fused<256>(x, nx, y, ny, rows, inv, out, s);
    case 9: return ambgfun_2d_fused<512>(x, nx, y, ny, rows, inv, out, s);
    case 10: return ambgfun_2d_fused<1024>(x, nx, y, ny, rows, inv, out, s);
    case 11: return ambgfun_2d_fused<2048>(x, nx, y, ny, rows, inv, out, s);
    case 12: return ambgfun_2d_fused<4096>(x, nx, y, ny, rows, inv, out, s);
    case 13: return ambgfun_2d_fused<8192>(x, nx, y, ny, rows, inv, out, s);
    case 14: return ambgfun_2d_fused<16384>(x, nx, y, ny, rows, inv, out, s);
    default: return fail(ZKX_INTERNAL_ERROR, "ambgfun: fused 2-D length out of range");
    }
}

unsigned grid_for(size_t n, int threads)
{
    const size_t blocks = (n + threads - 1) / threads;
    return (unsigned)(blocks < 65536u * 16u ? blocks : 65536u * 16u);
}

}  // namespace
}  // namespace zkx

using namespace zkx;

extern "C" int zkx_ambgfun_shape(int nx, int ny, int cut, long long* count, int* rows, int* nfreq)
{
    if (!count || !rows || !nfreq) return fail(ZKX_INVALID_ARGUMENT, "ambgfun: null pointer");
    if (nx < 1 || ny < 1) return fail(ZKX_INVALID_ARGUMENT, "ambgfun inputs must be nonempty");
    if (cut < 0 || cut > 2) return fail(ZKX_INVALID_ARGUMENT, "ambgfun cut is invalid");
    if (nx > std::numeric_limits<int>::max() - ny + 1)
        return fail(ZKX_INVALID_ARGUMENT, "ambgfun input length exceeds int capacity");
    const int r = nx + ny - 1;
    long long f = 1;
    while (f < r) f <<= 1;
    if (f > (1 << 16))
        return fail(ZKX_UNSUPPORTED_OPERATION, "ambgfun: nx + ny - 1 above 65536 is not supported");
    *rows = r;
    *nfreq = (int)f;
    *count = cut == 0 ? (long long)r * f : cut == 1 ? f : r;
    return ZKX_SUCCESS;
}

extern "C" int zkx_ambgfun_c64(const void* xv, int x_count, int nx, const void* yv, int y_count,
                               int ny, int cut, double fs, double cut_value, float* out,
                               zkx_stream_t stream)
{
    if (!yv) {
        yv = xv;
        y_count = x_count;
        ny = nx;
    }
    if (!xv || !out) return fail(ZKX_INVALID_ARGUMENT, "ambgfun: null pointer");
    if (x_count < 1 || y_count < 1 || nx < 1 || ny < 1 || nx > x_count || ny > y_count)
        return fail(ZKX_INVALID_ARGUMENT, "ambgfun inputs must be nonempty");
    if ((cut == 1 || cut == 2) && fs == 0.0)
        return fail(ZKX_INVALID_ARGUMENT, "ambgfun fs must be nonzero for one-dimensional cuts");
    long long count = 0;
    int rows = 0, nf = 0;
    ZKX_TRY(zkx_ambgfun_shape(nx, ny, cut, &count, &rows, &nf));
    ZKX_TRY(ensure_device_ready());
    const auto* x = static_cast<const float2*>(xv);
    const auto* y = static_cast<const float2*>(yv);
    // scratch: two inverse norms, then the transform buffers of the general path
    const bool fused = cut == 0 && nf <= (1 << kMaxFusedLog);
    const size_t buffers = cut == 0 ? (fused ? 0 : (size_t)rows * nf) : 2 * (size_t)nf;
    void* ws = nullptr;
    ZKX_TRY(scratch(kScratchAmbgfun, 256 + buffers * sizeof(float2), &ws));
    float* inv = static_cast<float*>(ws);
    float2* a = reinterpret_cast<float2*>(static_cast<char*>(ws) + 256);
    float2* b = a + nf;
    ambgfun_norm_kernel<<<2, 256, 0, stream>>>(x, x_count, y, y_count, inv);
    ZKX_LAUNCHED("ambgfun_norm_kernel");
    const int T = 256;
    const unsigned g1 = (unsigned)((nf + T - 1) / T);
    if (cut == 0) {
        if (fused) return dispatch_2d_fused(ilog2_host(nf), x, nx, y, ny, rows, inv, out, stream);
        ambgfun_build_kernel<<<grid_for((size_t)rows * nf, T), T, 0, stream>>>(x, nx, y, ny, rows, nf, inv, a);
        ZKX_LAUNCHED("ambgfun_build_kernel");
        ZKX_TRY(launch_fft_rows(a, rows, nf, 1, a, stream));  // inverse, scaled 1/F
        ambgfun_magnitude_kernel<<<grid_for((size_t)rows * nf, T), T, 0, stream>>>(a, rows, nf, (float)nf, out);
        ZKX_LAUNCHED("ambgfun_magnitude_kernel");
        return ZKX_SUCCESS;
    }
    if (cut == 1) {
        ambgfun_pack_kernel<<<g1, T, 0, stream>>>(x, nx, inv, 0, 0.0, nf, a);
        ZKX_LAUNCHED("ambgfun_pack_kernel");
        ZKX_TRY(launch_fft_rows(a, 1, nf, 0, a, stream));
        ambgfun_delay_phase_kernel<<<g1, T, 0, stream>>>(a, nf, fs, cut_value);
        ZKX_LAUNCHED("ambgfun_delay_phase_kernel");
        ZKX_TRY(launch_fft_rows(a, 1, nf, 1, a, stream));  // x shifted in delay
        ambgfun_conj_product_kernel<<<g1, T, 0, stream>>>(y, ny, inv, 1, a, nf, b);
        ZKX_LAUNCHED("ambgfun_conj_product_kernel");
        ZKX_TRY(launch_fft_rows(b, 1, nf, 1, b, stream));
        ambgfun_magnitude_kernel<<<g1, T, 0, stream>>>(b, 1, nf, (float)nf, out);
        ZKX_LAUNCHED("ambgfun_magnitude_kernel");
        return ZKX_SUCCESS;
    }
    // Doppler cut: a = x̂ modulated, b = ŷ; both transformed in one two-row launch
    ambgfun_pack_kernel<<<g1, T, 0, stream>>>(x, nx, inv, 0, cut_value / fs, nf, a);
    ZKX_LAUNCHED("ambgfun_pack_kernel");
    ambgfun_pack_kernel<<<g1, T, 0, stream>>>(y, ny, inv, 1, 0.0, nf, b);
    ZKX_LAUNCHED("ambgfun_pack_kernel");
    ZKX_TRY(launch_fft_rows(a, 2, nf, 0, a, stream));
    ambgfun_spectrum_product_kernel<<<g1, T, 0, stream>>>(b, a, nf, a);
    ZKX_LAUNCHED("ambgfun_spectrum_product_kernel");
    ZKX_TRY(launch_fft_rows(a, 1, nf, 1, a, stream));  // correlation, scaled 1/F
    ambgfun_doppler_out_kernel<<<g1, T, 0, stream>>>(a, nx, ny, nf, out);
    ZKX_LAUNCHED("ambgfun_doppler_out_kernel");
    return ZKX_SUCCESS;
}
