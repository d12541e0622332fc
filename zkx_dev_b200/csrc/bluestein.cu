// Transforms of any length: the reference's FFT backend switches to Bluestein's chirp-z
// transform for lengths that are not powers of two (backends/fft/fft_thrust.cu:702-765), and its
// CPU operators take any nfft (radartools_typed.cpp:625-800).  Here a length-n DFT is
//
//   X[k] = conj(w[k]) * sum_j (x[j] conj(w[j])) w[k - j],   w[m] = exp(i pi m^2 / n),
//
// a circular convolution of length M = next pow2(2n - 1) (so n <= 32768) on the library's
// power-of-two transforms: pre-multiplication, then one pass of the range-compression kernel
// (forward FFT, product with the FFT of the chirp, inverse FFT), post-multiplication.  The inverse DFT runs the same steps on conjugated data.
// Chirp phases are reduced exactly in integers (m^2 mod 2n) and evaluated in FP64.
//
// The same row pipeline with n a power of two and no chirp (M = n, plain FFT) serves Doppler
// transforms longer than the single-CTA kernel holds.  Rows are processed in passes whose
// workspace (stream-ordered, so concurrent streams never share it) stays under 256 MB.
#include <algorithm>
#include <cstdint>

#include "fft_core.cuh"
#include "rows.cuh"
#include "window.cuh"
#include "zkx_internal.h"

namespace zkx {
namespace {

constexpr size_t kPassBytes = size_t(1) << 28;  // row workspace per pass

__device__ __forceinline__ float2 chirp(long long m, int n)
{
    const long long r = (m * m) % (2LL * n);  // exp(i pi m^2 / n) has period 2n in m^2
    double s, c;
    sincospi((double)r / (double)n, &s, &c);
    return make_float2((float)c, (float)s);
}

// W[j] = w[j] for j < n; h[m] = conj(w[m]) for m < n, h[M - m] = conj(w[m]) for 0 < m < n,
// zero between.  h is the conjugate of the even convolution kernel b, so the compression
// spectrum conj(FFT(h)) / M equals FFT(b) / M.
__global__ void chirp_tables_kernel(int n, int M, float2* __restrict__ h, float2* __restrict__ W)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= M) return;
    float2 v = make_float2(0.f, 0.f);
    if (i < n) {
        v = chirp(i, n);
        W[i] = v;
    } else if (M - i < n) {
        v = chirp(M - i, n);
    }
    h[i] = make_float2(v.x, -v.y);
}

// a[r][j] = x_r[j] (conjugated when conj_in) * conj(W[j]) for j < n_in, zero up to M.
template <class Src>
__global__ void rows_pre_kernel(const Src src, int row0, int rows, int n_in, int log_m, int conj_in,
                                const float2* __restrict__ W, float2* __restrict__ a)
{
    const long long total = (long long)rows << log_m;
    const int mask = (1 << log_m) - 1;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(e >> log_m), j = (int)(e & mask);
        float2 v = make_float2(0.f, 0.f);
        if (j < n_in) {
            v = src.row(row0 + r)[j];
            if (conj_in) v.y = -v.y;
            if (W) v = cmulc(v, W[j]);
        }
        a[e] = v;
    }
}

// y[row0 + r][k] = scale * (a[r][k] * conj(W[k])) (conjugated when conj_out), k < n.
__global__ void rows_post_kernel(const float2* __restrict__ a, int rows, int n, int log_m, int conj_out,
                                 float scale, const float2* __restrict__ W, float2* __restrict__ y, int row0)
{
    const long long total = (long long)rows * n;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(e / n), k = (int)(e - (long long)r * n);
        float2 v = a[((long long)r << log_m) + k];
        if (W) v = cmulc(v, W[k]);
        if (conj_out) v.y = -v.y;
        y[(size_t)(row0 + r) * n + k] = make_float2(v.x * scale, v.y * scale);
    }
}

// Between the forward and the inverse transform of range compression: finish the forward
// DFT (k < n), multiply by the replica spectrum S, and start the inverse on conj(.) in place.
__global__ void compression_bridge_kernel(float2* __restrict__ a, int rows, int n, int log_m,
                                          const float2* __restrict__ W, const float2* __restrict__ S)
{
    const long long total = (long long)rows << log_m;
    const int mask = (1 << log_m) - 1;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(e & mask);
        float2 v = make_float2(0.f, 0.f);
        if (k < n) {
            v = a[e];
            if (W) v = cmulc(v, W[k]);
            v = cmul(v, S[k]);
            v.y = -v.y;
            if (W) v = cmulc(v, W[k]);
        }
        a[e] = v;
    }
}

// Doppler input, transposed through shared memory: a[b * ncol + c][j] =
// window[j] * x[cpi0 + b][j][col0 + c] * conj(W[j]) for pulses j < n_in, zero up to M.
// Block 32 x 8 over a 32-column x 32-pulse tile; grid (columns, pulses of M, CPIs).
__global__ void __launch_bounds__(256)
doppler_pre_kernel(const float2* __restrict__ x, int pulses, int samples, int cpi0, int col0, int ncol,
                   int n_in, int M, const float* __restrict__ window, const float2* __restrict__ W,
                   float2* __restrict__ a)
{
    __shared__ float2 tile[32][33];
    const int c0 = blockIdx.x * 32, j0 = blockIdx.y * 32, b = blockIdx.z;
    const size_t cpi = (size_t)cpi0 + b;
    for (int jj = threadIdx.y; jj < 32; jj += 8) {
        const int j = j0 + jj, c = c0 + threadIdx.x;
        float2 v = make_float2(0.f, 0.f);
        if (j < n_in && c < ncol) {
            v = x[(cpi * pulses + j) * samples + col0 + c];
            if (window) {
                const float w = window[j];
                v = make_float2(v.x * w, v.y * w);
            }
            if (W) v = cmulc(v, W[j]);
        }
        tile[jj][threadIdx.x] = v;
    }
    __syncthreads();
    for (int cc = threadIdx.y; cc < 32; cc += 8) {
        const int c = c0 + cc, j = j0 + threadIdx.x;
        if (c < ncol && j < M) a[((size_t)b * ncol + c) * M + j] = tile[threadIdx.x][cc];
    }
}

// Doppler output, transposed back: out[cpi0 + b][k][col0 + c] = a[b * ncol + c][k] * conj(W[k])
// for k < n, and its power |.|^2.  Grid (columns, bins of n, CPIs).
__global__ void __launch_bounds__(256)
doppler_post_kernel(const float2* __restrict__ a, int samples, int cpi0, int col0, int ncol, int n, int M,
                    const float2* __restrict__ W, float2* __restrict__ out, float* __restrict__ power)
{
    __shared__ float2 tile[32][33];
    const int c0 = blockIdx.x * 32, k0 = blockIdx.y * 32, b = blockIdx.z;
    for (int cc = threadIdx.y; cc < 32; cc += 8) {
        const int c = c0 + cc, k = k0 + threadIdx.x;
        float2 v = make_float2(0.f, 0.f);
        if (c < ncol && k < n) {
            v = a[((size_t)b * ncol + c) * M + k];
            if (W) v = cmulc(v, W[k]);
        }
        tile[cc][threadIdx.x] = v;
    }
    __syncthreads();
    const size_t base = ((size_t)cpi0 + b) * n * samples + col0;
    for (int kk = threadIdx.y; kk < 32; kk += 8) {
        const int k = k0 + kk, c = c0 + threadIdx.x;
        if (k < n && c < ncol) {
            const float2 v = tile[threadIdx.x][kk];
            const size_t o = base + (size_t)k * samples + c;
            if (out) out[o] = v;
            if (power) power[o] = fmaf(v.x, v.x, v.y * v.y);
        }
    }
}

// Windowed replica of a transform of any length, scaled so that its conjugated DFT is the
// spectrum the compression kernels multiply by: row[e] = w[e] h[e] / (||w h|| * nfft) for
// e < min(length, nfft), zero up to nfft (the norm runs over all `length` samples).  One CTA.
__global__ void __launch_bounds__(1024)
replica_row_kernel(const float2* __restrict__ h, int length, int nfft, int normalize, int kind,
                   const float* __restrict__ explicit_window, float2* __restrict__ row)
{
    __shared__ double partial[1024];
    const int t = threadIdx.x;
    double acc = 0.0;
    for (int i = t; i < length; i += 1024) {
        const double w = window_value(kind, explicit_window, i, length);
        const float2 v = h[i];
        const double re = (double)v.x * w, im = (double)v.y * w;
        acc += re * re + im * im;
    }
    partial[t] = acc;
    __syncthreads();
    for (int s = 512; s > 0; s >>= 1) {
        if (t < s) partial[t] += partial[t + s];
        __syncthreads();
    }
    const double norm = normalize ? sqrt(partial[0]) : 1.0;
    const float scale = (float)(1.0 / (norm * (double)nfft));
    for (int e = t; e < nfft; e += 1024) {
        float2 v = make_float2(0.f, 0.f);
        if (e < length) {
            const float w = window_value(kind, explicit_window, e, length);
            const float2 hv = h[e];
            v = make_float2(hv.x * w * scale, hv.y * w * scale);
        }
        row[e] = v;
    }
}

unsigned grid_for(long long elems)
{
    const long long b = (elems + 255) / 256;
    return (unsigned)std::max(1LL, std::min(b, 148LL * 16));
}

// Geometry, chirp tables and workspace of one transform length.
struct Dft {
    int n = 0, M = 0, log_m = 0;
    bool direct = false;    // n a power of two: plain FFT of length n, no chirp
    float2* S = nullptr;    // FFT(b) / M in the layout of the compression kernels, M entries
    float2* W = nullptr;    // chirp, n entries (nullptr when direct)
    float2* a = nullptr;    // pass workspace, chunk x M
    int chunk = 0;          // rows per pass
};

int prepare(int n, long long rows, cudaStream_t s, StreamWorkspace* ws, Dft* d)
{
    d->n = n;
    d->direct = is_pow2(n);
    int M = n;
    if (!d->direct)
        for (M = 1; M < 2 * n - 1; M <<= 1) {}
    d->M = M;
    d->log_m = ilog2_host(M);
    // S (M) | h (M) | W (n, rounded up to keep a 16-byte aligned) | a
    const size_t table = d->direct ? 0 : 2 * (size_t)M + (((size_t)n + 1) & ~size_t(1));
    const long long fit = std::max(1LL, (long long)(kPassBytes / ((size_t)M * sizeof(float2))));
    d->chunk = (int)std::max(1LL, std::min(rows, fit));
    ws->stream = s;
    ZKX_TRY(stream_workspace((table + (size_t)d->chunk * M) * sizeof(float2), s, &ws->ptr));
    float2* base = static_cast<float2*>(ws->ptr);
    d->a = base + table;
    if (d->direct) return ZKX_SUCCESS;
    d->S = base;
    float2* h = base + M;
    d->W = base + 2 * M;
    chirp_tables_kernel<<<(M + 255) / 256, 256, 0, s>>>(n, M, h, d->W);
    ZKX_LAUNCHED("chirp_tables_kernel");
    return launch_replica_spectrum(h, M, M, 0, ZKX_WINDOW_NONE, nullptr, d->S, s);
}

// The circular convolution with the chirp in place -- one pass of the range-compression
// kernels (forward FFT, product with S, inverse FFT per row) -- or the plain forward FFT
// when direct.
int convolve(const Dft& d, int rows, cudaStream_t s)
{
    if (d.direct) return launch_fft_rows(d.a, rows, d.M, 0, d.a, s);
    return launch_pulse_compression_variant(d.a, rows, d.M, d.M, d.S, d.a, ZKX_COMPRESSION_DEFAULT, s);
}

// Row DFTs of length n over `rows` rows of src (first n_in samples, zero beyond), written
// as [rows, n] to y.
template <class Src>
int dft_rows(const Src& src, int rows, int n_in, int n, int inverse, float scale, float2* y, cudaStream_t s)
{
    Dft d;
    StreamWorkspace ws;
    ZKX_TRY(prepare(n, rows, s, &ws, &d));
    for (int r0 = 0; r0 < rows; r0 += d.chunk) {
        const int r = std::min(d.chunk, rows - r0);
        rows_pre_kernel<Src><<<grid_for((long long)r << d.log_m), 256, 0, s>>>(src, r0, r, n_in, d.log_m,
                                                                                 inverse, d.W, d.a);
        ZKX_LAUNCHED("rows_pre_kernel");
        ZKX_TRY(convolve(d, r, s));
        rows_post_kernel<<<grid_for((long long)r * n), 256, 0, s>>>(d.a, r, n, d.log_m, inverse, scale, d.W, y, r0);
        ZKX_LAUNCHED("rows_post_kernel");
    }
    return ZKX_SUCCESS;
}

template <class Src>
int compression_any(const Src& src, int pulses, int samples, int nfft, const float2* spectrum, float2* y,
                    cudaStream_t s)
{
    Dft d;
    StreamWorkspace ws;
    ZKX_TRY(prepare(nfft, pulses, s, &ws, &d));
    const int n_in = std::min(samples, nfft);
    for (int r0 = 0; r0 < pulses; r0 += d.chunk) {
        const int r = std::min(d.chunk, pulses - r0);
        const unsigned g = grid_for((long long)r << d.log_m);
        rows_pre_kernel<Src><<<g, 256, 0, s>>>(src, r0, r, n_in, d.log_m, 0, d.W, d.a);
        ZKX_LAUNCHED("rows_pre_kernel");
        ZKX_TRY(convolve(d, r, s));
        compression_bridge_kernel<<<g, 256, 0, s>>>(d.a, r, nfft, d.log_m, d.W, spectrum);
        ZKX_LAUNCHED("compression_bridge_kernel");
        ZKX_TRY(convolve(d, r, s));
        rows_post_kernel<<<grid_for((long long)r * nfft), 256, 0, s>>>(d.a, r, nfft, d.log_m, 1, 1.0f, d.W, y, r0);
        ZKX_LAUNCHED("rows_post_kernel");
    }
    return ZKX_SUCCESS;
}

}  // namespace

int launch_dft_rows(const float2* x, int rows, int n, int inverse, float2* y, cudaStream_t stream)
{
    if (n < 1 || n > kMaxBluesteinLength)
        return fail(ZKX_UNSUPPORTED_OPERATION, "transform lengths that are not powers of two stop at 32768");
    return dft_rows(RowsContiguous{x, n}, rows, n, n, inverse ? 1 : 0, inverse ? (float)(1.0 / n) : 1.0f, y,
                    stream);
}

int launch_replica_spectrum_any(const float2* replica, int length, int nfft, int normalize, int window_kind,
                                const float* explicit_window, float2* spectrum, cudaStream_t stream)
{
    if (nfft < 1 || nfft > kMaxBluesteinLength)
        return fail(ZKX_UNSUPPORTED_OPERATION, "transform lengths that are not powers of two stop at 32768");
    replica_row_kernel<<<1, 1024, 0, stream>>>(replica, length, nfft, normalize, window_kind, explicit_window,
                                               spectrum);
    ZKX_LAUNCHED("replica_row_kernel");
    // spectrum = conj(DFT(row)): the inverse-direction steps conjugate the output
    Dft d;
    StreamWorkspace ws;
    ZKX_TRY(prepare(nfft, 1, stream, &ws, &d));
    rows_pre_kernel<RowsContiguous><<<grid_for(d.M), 256, 0, stream>>>(RowsContiguous{spectrum, nfft}, 0, 1,
                                                                        nfft, d.log_m, 0, d.W, d.a);
    ZKX_LAUNCHED("rows_pre_kernel");
    ZKX_TRY(convolve(d, 1, stream));
    rows_post_kernel<<<grid_for(nfft), 256, 0, stream>>>(d.a, 1, nfft, d.log_m, 1, 1.0f, d.W, spectrum, 0);
    ZKX_LAUNCHED("rows_post_kernel");
    return ZKX_SUCCESS;
}

int launch_compression_any(const RowsContiguous& x, int pulses, int samples, int nfft, const float2* spectrum,
                           float2* y, cudaStream_t stream)
{
    if (nfft < 1 || nfft > kMaxBluesteinLength)
        return fail(ZKX_UNSUPPORTED_OPERATION, "transform lengths that are not powers of two stop at 32768");
    return compression_any(x, pulses, samples, nfft, spectrum, y, stream);
}

int launch_compression_any(const RowsTable& x, int pulses, int samples, int nfft, const float2* spectrum,
                           float2* y, cudaStream_t stream)
{
    if (nfft < 1 || nfft > kMaxBluesteinLength)
        return fail(ZKX_UNSUPPORTED_OPERATION, "transform lengths that are not powers of two stop at 32768");
    return compression_any(x, pulses, samples, nfft, spectrum, y, stream);
}

int launch_doppler_any(const float2* x, int pulses, int samples, int nfft, const float* window, float2* out,
                       float* power, int batch, cudaStream_t stream)
{
    if (nfft < 1 || (!is_pow2(nfft) && nfft > kMaxBluesteinLength) || nfft > (1 << 16))
        return fail(ZKX_UNSUPPORTED_OPERATION,
                    "pulse_doppler: nfft above 65536, or above 32768 and not a power of two");
    Dft d;
    StreamWorkspace ws;
    ZKX_TRY(prepare(nfft, (long long)batch * samples, stream, &ws, &d));
    const int n_in = std::min(pulses, nfft);
    // a pass covers whole CPIs when one CPI's columns fit, else column ranges of one CPI
    const int ncol = std::min(samples, d.chunk);
    const int ncpi = samples <= d.chunk ? std::min(std::min(batch, d.chunk / samples), 65535) : 1;
    const unsigned mt = (unsigned)((d.M + 31) / 32), nt = (unsigned)((nfft + 31) / 32);
    for (int c0 = 0; c0 < batch; c0 += ncpi) {
        const int nc = std::min(ncpi, batch - c0);
        for (int col0 = 0; col0 < samples; col0 += ncol) {
            const int w = std::min(ncol, samples - col0);
            const unsigned ct = (unsigned)((w + 31) / 32);
            doppler_pre_kernel<<<dim3(ct, mt, nc), dim3(32, 8), 0, stream>>>(x, pulses, samples, c0, col0, w, n_in,
                                                                              d.M, window, d.W, d.a);
            ZKX_LAUNCHED("doppler_pre_kernel");
            ZKX_TRY(convolve(d, nc * w, stream));
            doppler_post_kernel<<<dim3(ct, nt, nc), dim3(32, 8), 0, stream>>>(d.a, samples, c0, col0, w, nfft, d.M,
                                                                               d.W, out, power);
            ZKX_LAUNCHED("doppler_post_kernel");
        }
    }
    return ZKX_SUCCESS;
}

}  // namespace zkx
