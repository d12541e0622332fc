// extern "C" entry points of libzkx_rd.so: argument validation with the reference's
// rules and error codes, then asynchronous kernel launches on the caller's stream.
#include "fft_core.cuh"
#include "zkx_internal.h"

#include <algorithm>
#include <climits>
#include <map>
#include <vector>
#include <mutex>
#include <tuple>
#include <cmath>
#include <numeric>
#include <string>

using namespace zkx;

namespace {

constexpr int kMaxNfft = 1 << 16;  // 65536 (two or four clustered CTAs above 16384)

bool valid_window(int kind, const void* explicit_window)
{
    if (kind < ZKX_WINDOW_NONE || kind > ZKX_WINDOW_EXPLICIT_FP64) return false;
    const bool is_explicit = kind == ZKX_WINDOW_EXPLICIT_FP32 || kind == ZKX_WINDOW_EXPLICIT_FP64;
    return is_explicit == (explicit_window != nullptr);
}

// Powers of two up to 65536; any other length up to 32768 (chirp-z on power-of-two FFTs).
int check_transform_length(int nfft, const char* fn)
{
    if (nfft < 1) return fail(ZKX_INVALID_ARGUMENT, std::string(fn) + ": nfft must be positive");
    if (nfft > kMaxNfft || (!is_pow2(nfft) && nfft > kMaxBluesteinLength))
        return fail(ZKX_UNSUPPORTED_OPERATION,
                    std::string(fn) + ": nfft must be at most 32768, or a power of two up to 65536");
    return ZKX_SUCCESS;
}

// radartools_typed.cpp:280-286: both extents >= 1 and the product fits an int.
int check_radar_shape(int first, int second, const char* fn)
{
    const long long count = (long long)first * second;
    if (first < 1 || second < 1 || count > INT_MAX)
        return fail(ZKX_INVALID_SHAPE, std::string(fn) + " shape exceeds kernel capacity");
    return ZKX_SUCCESS;
}

int compression_checks(const void* x, int P, int N, const void* replica, int L, int nfft,
                       int kind, const float* w, const void* y)
{
    ZKX_TRY(check_radar_shape(P, N, "pulse_compression"));
    ZKX_TRY(check_radar_shape(P, nfft, "pulse_compression"));
    if (L < 1) return fail(ZKX_INVALID_SHAPE, "pulse_compression shape is invalid");
    if (!valid_window(kind, w)) return fail(ZKX_INVALID_ARGUMENT, "pulse_compression window is invalid");
    if (!x || !replica || !y) return fail(ZKX_INVALID_ARGUMENT, "pulse_compression: null pointer");
    return check_transform_length(nfft, "pulse_compression");
}

struct CfarGeometry {
    int nref = 0;
    double alpha = 0.0;
};

// radartools_typed.cpp:161-220
int cfar_checks(int rank, int rows, int cols, int gr, int gc, int rr, int rc, double pfa,
                CfarGeometry* g)
{
    if (rank != 1 && rank != 2) return fail(ZKX_INVALID_SHAPE, "ca_cfar supports only 1D or 2D input here");
    if (rows < 0 || (rank == 2 && cols < 0)) return fail(ZKX_INVALID_SHAPE, "ca_cfar shape dimensions must be nonnegative");
    if (gr < 0 || rr < 1 || (rank == 2 && (gc < 0 || rc < 1)))
        return fail(ZKX_INVALID_ARGUMENT, "ca_cfar guard/reference cells are invalid");
    if ((long long)rows <= 2LL * ((long long)gr + rr) ||
        (rank == 2 && (long long)cols <= 2LL * ((long long)gc + rc)))
        return fail(ZKX_INVALID_SHAPE, "ca_cfar input dimension is too small");
    if (!std::isfinite(pfa) || pfa <= 0.0 || pfa > 1.0) return fail(ZKX_INVALID_ARGUMENT, "ca_cfar pfa must be in (0,1]");
    if ((long long)rows * (rank == 2 ? cols : 1) > INT_MAX)
        return fail(ZKX_INVALID_SHAPE, "ca_cfar input size or capacity is invalid");
    long long nref = rank == 2 ? 2LL * rr * (2LL * rc + 2LL * gc + 1) + 2LL * (2LL * gr + 1) * rc : 2LL * rr;
    if (nref > INT_MAX) return fail(ZKX_INVALID_ARGUMENT, "ca_cfar reference count exceeds int capacity");
    g->nref = (int)nref;
    g->alpha = (double)nref * (std::pow(pfa, -1.0 / (double)nref) - 1.0);
    return ZKX_SUCCESS;
}

}  // namespace

// ------------------------------------------------------------------ radar ops

extern "C" int zkx_replica_spectrum_c64(const void* replica, int L, int nfft, int normalize,
                                        int kind, const float* w, void* spectrum,
                                        zkx_stream_t stream)
{
    if (L < 1) return fail(ZKX_INVALID_SHAPE, "replica length must be positive");
    if (!valid_window(kind, w)) return fail(ZKX_INVALID_ARGUMENT, "replica window is invalid");
    if (!replica || !spectrum) return fail(ZKX_INVALID_ARGUMENT, "replica_spectrum: null pointer");
    ZKX_TRY(check_transform_length(nfft, "replica_spectrum"));
    ZKX_TRY(ensure_device_ready());
    return launch_replica_spectrum(static_cast<const float2*>(replica), L, nfft, normalize, kind, w,
                                   static_cast<float2*>(spectrum), stream);
}

extern "C" int zkx_pulse_compression_spectrum_c64(const void* x, int P, int N, int nfft,
                                                  const void* spectrum, void* y,
                                                  zkx_stream_t stream)
{
    if (nfft == -1) nfft = N;
    ZKX_TRY(check_radar_shape(P, N, "pulse_compression"));
    ZKX_TRY(check_radar_shape(P, nfft, "pulse_compression"));
    if (!x || !spectrum || !y) return fail(ZKX_INVALID_ARGUMENT, "pulse_compression: null pointer");
    ZKX_TRY(check_transform_length(nfft, "pulse_compression"));
    ZKX_TRY(ensure_device_ready());
    return launch_pulse_compression(static_cast<const float2*>(x), P, N, nfft,
                                    static_cast<const float2*>(spectrum), static_cast<float2*>(y),
                                    stream);
}

extern "C" int zkx_pulse_compression_spectrum_ex_c64(const void* x, int P, int N, int nfft,
                                                     const void* spectrum, int precision, void* y,
                                                     zkx_stream_t stream)
{
    if (precision == ZKX_PRECISION_FP32)
        return zkx_pulse_compression_spectrum_c64(x, P, N, nfft, spectrum, y, stream);
    if (nfft == -1) nfft = N;
    if (precision != ZKX_PRECISION_TC_F16 && precision != ZKX_PRECISION_TC_BF16)
        return fail(ZKX_INVALID_ARGUMENT, "pulse_compression: unknown precision");
    ZKX_TRY(check_radar_shape(P, N, "pulse_compression"));
    ZKX_TRY(check_radar_shape(P, nfft, "pulse_compression"));
    if (!x || !spectrum || !y) return fail(ZKX_INVALID_ARGUMENT, "pulse_compression: null pointer");
    if (nfft != 4096 && nfft != 8192 && nfft != 16384)
        return fail(ZKX_UNSUPPORTED_OPERATION,
                    "pulse_compression: tensor-core precision needs nfft 4096, 8192 or 16384");
    ZKX_TRY(ensure_device_ready());
    return launch_pulse_compression_tc(static_cast<const float2*>(x), P, N, nfft,
                                       static_cast<const float2*>(spectrum), static_cast<float2*>(y),
                                       precision, stream);
}

extern "C" int zkx_pulse_compression_c64(const void* x, int P, int N, const void* replica, int L,
                                         int nfft, int normalize, int kind, const float* w,
                                         void* y, zkx_stream_t stream)
{
    if (nfft == -1) nfft = N;
    ZKX_TRY(compression_checks(x, P, N, replica, L, nfft, kind, w, y));
    ZKX_TRY(ensure_device_ready());
    void* spec = nullptr;
    ZKX_TRY(scratch(kScratchReplica, (size_t)nfft * sizeof(float2), &spec));
    ZKX_TRY(launch_replica_spectrum(static_cast<const float2*>(replica), L, nfft, normalize, kind, w,
                                    static_cast<float2*>(spec), stream));
    return launch_pulse_compression(static_cast<const float2*>(x), P, N, nfft,
                                    static_cast<const float2*>(spec), static_cast<float2*>(y), stream);
}

extern "C" int zkx_pulse_doppler_c64(const void* x, int P, int N, int nfft, int kind,
                                     const float* w, void* out, float* power, zkx_stream_t stream)
{
    if (nfft == -1) nfft = P;
    ZKX_TRY(check_radar_shape(P, N, "pulse_doppler"));
    ZKX_TRY(check_radar_shape(nfft, N, "pulse_doppler"));
    if (!valid_window(kind, w)) return fail(ZKX_INVALID_ARGUMENT, "pulse_doppler window is invalid");
    if (!x || (!out && !power)) return fail(ZKX_INVALID_ARGUMENT, "pulse_doppler: null pointer");
    ZKX_TRY(check_transform_length(nfft, "pulse_doppler"));
    ZKX_TRY(ensure_device_ready());
    float* win = nullptr;
    if (kind != ZKX_WINDOW_NONE) {
        void* p = nullptr;
        ZKX_TRY(scratch(kScratchDopplerWindow, (size_t)P * sizeof(float), &p));
        win = static_cast<float*>(p);
        ZKX_TRY(launch_doppler_window(P, kind, w, win, stream));
    }
    return launch_pulse_doppler(static_cast<const float2*>(x), P, N, nfft, win,
                                static_cast<float2*>(out), power, 1, 0, stream);
}

extern "C" int zkx_fft_c2c_c64(const void* x, int batch, int n, int inverse, void* y,
                               zkx_stream_t stream)
{
    ZKX_TRY(check_radar_shape(batch, n, "fft"));
    if (!x || !y) return fail(ZKX_INVALID_ARGUMENT, "fft: null pointer");
    ZKX_TRY(check_transform_length(n, "fft"));
    ZKX_TRY(ensure_device_ready());
    return launch_fft_rows(static_cast<const float2*>(x), batch, n, inverse ? 1 : 0,
                           static_cast<float2*>(y), stream);
}

// ------------------------------------------------------------------------ CFAR

extern "C" int zkx_cfar_alpha(double pfa, int reference_count, double* alpha)
{
    // radartools_typed.cpp:592-603
    if (!alpha) return fail(ZKX_INVALID_ARGUMENT, "cfar_alpha: null pointer");
    if (reference_count < 1 || !std::isfinite(pfa) || pfa <= 0.0 || pfa > 1.0)
        return fail(ZKX_INVALID_ARGUMENT, "cfar_alpha requires reference >= 1 and pfa in (0,1]");
    *alpha = (double)reference_count * (std::pow(pfa, -1.0 / (double)reference_count) - 1.0);
    return ZKX_SUCCESS;
}

extern "C" int zkx_cfar_reference_count(int rank, int gr, int gc, int rr, int rc)
{
    if (rank == 1) return 2 * rr;
    return 2 * rr * (2 * rc + 2 * gc + 1) + 2 * (2 * gr + 1) * rc;
}

extern "C" int zkx_ca_cfar_f32(const float* x, int rank, int rows, int cols, int gr, int gc,
                               int rr, int rc, double pfa, int mode, float* threshold,
                               uint8_t* detections, zkx_stream_t stream)
{
    CfarGeometry g;
    ZKX_TRY(cfar_checks(rank, rows, cols, gr, gc, rr, rc, pfa, &g));
    if (mode != ZKX_CFAR_ACCURATE && mode != ZKX_CFAR_COMPAT)
        return fail(ZKX_INVALID_ARGUMENT, "ca_cfar: unknown mode");
    if (!x || !threshold || !detections) return fail(ZKX_INVALID_ARGUMENT, "ca_cfar: null pointer");
    ZKX_TRY(ensure_device_ready());
    if (rank == 1 || mode == ZKX_CFAR_COMPAT) {
        const long long count = (long long)rows * (rank == 2 ? cols : 1);
        void* cum = nullptr;
        ZKX_TRY(scratch(kScratchCfarIntegral, (size_t)count * sizeof(float), &cum));
        return launch_ca_cfar_compat(x, rank, rows, rank == 2 ? cols : 1, gr, gc, rr, rc,
                                     (float)g.alpha, g.nref, static_cast<float*>(cum), threshold,
                                     detections, stream);
    }
    return launch_ca_cfar_accurate(x, rows, cols, gr, gc, rr, rc, g.alpha, g.nref, threshold,
                                   detections, 1, ZKX_CFAR_TILE_DEFAULT, stream);
}

// --------------------------------------------------------------------- filters

extern "C" int zkx_fir_f32(const float* b, int nb, const float* x, int lines, int n,
                           const float* zi, float* y, float* zf, zkx_stream_t stream)
{
    // filtering_typed.cpp:1125-1146 (coefficients, shape) ...
    if (nb < 1) return fail(ZKX_INVALID_ARGUMENT, "firfilter coefficients");
    if (lines < 1 || n < 1 || (long long)lines * n > INT_MAX)
        return fail(ZKX_INVALID_SHAPE, "firfilter input shape");
    if (!b || !x || !y || (zi && nb > 1 && !zf)) return fail(ZKX_INVALID_ARGUMENT, "firfilter: null pointer");
    ZKX_TRY(ensure_device_ready());
    return launch_fir(b, nb, x, lines, n, zi, y, zi ? zf : nullptr, stream);
}

extern "C" int zkx_fir_ex_f32(const float* b, int nb, const float* x, int lines, int n, const float* zi,
                              float* y, float* zf, int method, zkx_stream_t stream)
{
    if (method < ZKX_FIR_AUTO || method > ZKX_FIR_FFT) return fail(ZKX_INVALID_ARGUMENT, "firfilter: unknown method");
    if (nb < 1) return fail(ZKX_INVALID_ARGUMENT, "firfilter coefficients");
    if (lines < 1 || n < 1 || (long long)lines * n > INT_MAX)
        return fail(ZKX_INVALID_SHAPE, "firfilter input shape");
    if (!b || !x || !y || (zi && nb > 1 && !zf)) return fail(ZKX_INVALID_ARGUMENT, "firfilter: null pointer");
    if (method == ZKX_FIR_FFT && nb > 4096) return fail(ZKX_UNSUPPORTED_OPERATION, "firfilter: FFT method takes at most 4096 taps");
    ZKX_TRY(ensure_device_ready());
    return launch_fir(b, nb, x, lines, n, zi, y, zi ? zf : nullptr, stream, method);
}

extern "C" long long zkx_upfirdn_length(int n, int nh, int up, int down)
{
    if (nh < 1 || up < 1 || down < 1 || n < 0) return -1;
    const long long num = ((long long)n - 1) * up + nh - 1;
    long long q = num / down;
    if (num % down != 0 && num < 0) --q;
    return q + 1;
}

extern "C" int zkx_upfirdn_f32(const float* h, int nh, const float* x, int lines, int n, int up,
                               int down, float* y, zkx_stream_t stream)
{
    // filtering_typed.cpp:1046-1117
    if (nh < 1) return fail(ZKX_INVALID_ARGUMENT, "upfirdn coefficients");
    if (up < 1 || down < 1) return fail(ZKX_INVALID_ARGUMENT, "upfirdn factors");
    if (lines < 1 || n < 0) return fail(ZKX_INVALID_SHAPE, "upfirdn input shape");
    const long long nout = zkx_upfirdn_length(n, nh, up, down);
    if (nout < 0 || nout > INT_MAX || (long long)lines * nout > INT_MAX)
        return fail(ZKX_INVALID_SHAPE, "upfirdn output sample count");
    if (!h || (!x && n > 0) || (!y && nout > 0)) return fail(ZKX_INVALID_ARGUMENT, "upfirdn: null pointer");
    ZKX_TRY(ensure_device_ready());
    return launch_polyphase(h, nh, up, down, 0, x, lines, n, y, (int)nout, stream);
}

extern "C" int zkx_resample_poly_layout(int n, int up, int down, int custom, int ncoeffs,
                                        zkx_resample_layout* L)
{
    // filtering_typed.cpp:933-1044
    if (!L) return fail(ZKX_INVALID_ARGUMENT, "resample_poly: null layout");
    if (up < 1 || down < 1) return fail(ZKX_INVALID_ARGUMENT, "resample_poly factors");
    if (n < 0) return fail(ZKX_INVALID_SHAPE, "resample_poly input shape");
    *L = zkx_resample_layout{};
    const int g = std::gcd(up, down);
    L->up = up / g;
    L->down = down / g;
    L->identity = L->up == 1 && L->down == 1;
    if (L->identity) {
        L->output_samples = n;
        return ZKX_SUCCESS;
    }
    const long long out = ((long long)n * L->up + L->down - 1) / L->down;
    if (out > INT_MAX) return fail(ZKX_INVALID_SHAPE, "resample_poly output sample count");
    L->output_samples = (int)out;
    if (custom) {
        if (ncoeffs < 0) return fail(ZKX_INVALID_ARGUMENT, "resample_poly coefficients");
        L->coefficient_count = ncoeffs;
        L->half_length = ncoeffs == 0 ? -1 : (ncoeffs - 1) / 2;
    } else {
        const int mr = L->up > L->down ? L->up : L->down;
        if (mr > (INT_MAX - 1) / 20) return fail(ZKX_INVALID_ARGUMENT, "resample_poly designed filter length");
        L->half_length = 10 * mr;
        L->coefficient_count = 2 * L->half_length + 1;
    }
    const int rem = ((L->half_length % L->down) + L->down) % L->down;
    L->prefix_zeros = L->down - rem;
    L->output_start = (L->half_length + L->prefix_zeros) / L->down;
    return ZKX_SUCCESS;
}

namespace {
// Abramowitz-Stegun polynomial I0 used by the reference's design
// (filtering_typed.cpp:159-174); kept so designed taps match the reference exactly.
double bessel_i0_as(double v)
{
    const double a = std::fabs(v);
    if (a < 3.75) {
        const double r = v / 3.75, y = r * r;
        return 1.0 + y * (3.5156229 + y * (3.0899424 + y * (1.2067492 + y * (0.2659732 +
               y * (0.0360768 + y * 0.0045813)))));
    }
    const double y = 3.75 / a;
    return std::exp(a) / std::sqrt(a) * (0.39894228 + y * (0.01328592 + y * (0.00225319 + y *
           (-0.00157565 + y * (0.00916281 + y * (-0.02057706 + y * (0.02635537 + y *
           (-0.01647633 + y * 0.00392377))))))));
}
}  // namespace

extern "C" int zkx_resample_poly_design(const zkx_resample_layout* L, double beta, double* taps)
{
    // filtering_typed.cpp:176-222 (Kaiser window, windowed sinc, sum scaled to up)
    if (!L || !taps) return fail(ZKX_INVALID_ARGUMENT, "resample_poly_design: null pointer");
    const int count = L->coefficient_count, half = L->half_length;
    if (count < 1 || half < 1) return fail(ZKX_INVALID_ARGUMENT, "resample_poly_design: empty design");
    const double denom = bessel_i0_as(beta);
    const double cutoff = 1.0 / (L->up > L->down ? L->up : L->down);
    const double pi = 3.1415926535897932384626433832795;
    double scale = 0.0;
    for (int i = 0; i < count; ++i) {
        const double ratio = (double)(i - half) / half;
        const double bounded = std::max(0.0, 1.0 - ratio * ratio);
        const double w = bessel_i0_as(beta * std::sqrt(bounded)) / denom;
        const int off = i - half;
        const double sinc = off == 0 ? cutoff : std::sin(pi * cutoff * off) / (pi * off);
        taps[i] = sinc * w;
        scale += taps[i];
    }
    for (int i = 0; i < count; ++i) taps[i] = taps[i] / scale * L->up;
    return ZKX_SUCCESS;
}

extern "C" int zkx_resample_poly_design_window(const zkx_resample_layout* L, const double* window,
                                               double* taps)
{
    // filtering_typed.cpp:208-222 with the window supplied by the caller
    if (!L || !window || !taps) return fail(ZKX_INVALID_ARGUMENT, "resample_poly_design_window: null pointer");
    const int count = L->coefficient_count, half = L->half_length;
    if (count < 1) return fail(ZKX_INVALID_ARGUMENT, "resample_poly_design_window: empty design");
    const double cutoff = 1.0 / (L->up > L->down ? L->up : L->down);
    const double pi = 3.1415926535897932384626433832795;
    double scale = 0.0;
    for (int i = 0; i < count; ++i) {
        const int off = i - half;
        const double sinc = off == 0 ? cutoff : std::sin(pi * cutoff * off) / (pi * off);
        taps[i] = sinc * window[i];
        scale += taps[i];
    }
    for (int i = 0; i < count; ++i) taps[i] = taps[i] / scale * L->up;
    return ZKX_SUCCESS;
}

extern "C" int zkx_resample_poly_f32(const float* x, int lines, int n, const zkx_resample_layout* L,
                                     const float* taps, float* y, zkx_stream_t stream)
{
    if (!L) return fail(ZKX_INVALID_ARGUMENT, "resample_poly: null layout");
    if (lines < 1 || n < 0 || (long long)lines * L->output_samples > INT_MAX)
        return fail(ZKX_INVALID_SHAPE, "resample_poly workspace shape");
    if (L->identity) {
        if (n > 0) ZKX_CUDA(cudaMemcpyAsync(y, x, (size_t)lines * n * sizeof(float),
                                            cudaMemcpyDeviceToDevice, stream));
        return ZKX_SUCCESS;
    }
    if (L->coefficient_count < 1) return fail(ZKX_INVALID_ARGUMENT, "resample_poly coefficients");
    if (!x || !taps || !y) return fail(ZKX_INVALID_ARGUMENT, "resample_poly: null pointer");
    ZKX_TRY(ensure_device_ready());
    const long long offset = (long long)L->output_start * L->down - L->prefix_zeros;
    return launch_polyphase(taps, L->coefficient_count, L->up, L->down, offset, x, lines, n, y,
                            L->output_samples, stream);
}

// ------------------------------------------------------------------ the chain

struct zkx_rd_plan_s {
    zkx_rd_desc d{};
    int range_nfft = 0;
    int doppler_nfft = 0;
    int device = 0;
    float2* spectrum = nullptr;
    float* doppler_window = nullptr;
    float2* compressed = nullptr;  // used when the caller passes no compressed buffer
    size_t compressed_elems = 0;
    float* power = nullptr;        // used when the caller passes no power buffer
    size_t power_elems = 0;
    float* cumulative = nullptr;   // compat CFAR integral image
    size_t cumulative_elems = 0;
    CfarGeometry cfar;
    zkx_rd_tuning tuning{};        // per-shape kernel choices (0 = heuristic)
};

namespace {
// Autotuned kernel choices per plan shape, shared by every plan of the process.
struct TuneKey {
    int pulses, samples, range_nfft, doppler_nfft;
    bool operator<(const TuneKey& o) const
    {
        return std::tie(pulses, samples, range_nfft, doppler_nfft) <
               std::tie(o.pulses, o.samples, o.range_nfft, o.doppler_nfft);
    }
};
std::mutex g_tune_mutex;
std::map<TuneKey, zkx_rd_tuning> g_tune_table;
}  // namespace

namespace {
void release_plan(zkx_rd_plan p)
{
    if (!p) return;
    cudaFree(p->spectrum);
    cudaFree(p->doppler_window);
    cudaFree(p->compressed);
    cudaFree(p->power);
    cudaFree(p->cumulative);
    delete p;
}
}  // namespace

extern "C" int zkx_rd_plan_create(const zkx_rd_desc* d, const void* replica,
                                  const float* range_window, const float* doppler_window,
                                  zkx_stream_t stream, zkx_rd_plan* out)
{
    if (!d || !out || !replica) return fail(ZKX_INVALID_ARGUMENT, "rd_plan_create: null pointer");
    *out = nullptr;
    const int P = d->num_pulses, N = d->samples_per_pulse;
    const int nr = d->range_nfft == -1 ? N : d->range_nfft;
    const int nd = d->doppler_nfft == -1 ? P : d->doppler_nfft;
    ZKX_TRY(compression_checks(replica, P, N, replica, d->replica_length, nr, d->range_window,
                               range_window, replica));
    ZKX_TRY(check_radar_shape(nd, nr, "pulse_doppler"));
    if (!valid_window(d->doppler_window, doppler_window))
        return fail(ZKX_INVALID_ARGUMENT, "pulse_doppler window is invalid");
    ZKX_TRY(check_transform_length(nd, "pulse_doppler"));
    if (d->precision != ZKX_PRECISION_FP32 && d->precision != ZKX_PRECISION_TC_F16 &&
        d->precision != ZKX_PRECISION_TC_BF16)
        return fail(ZKX_INVALID_ARGUMENT, "rd_plan: unknown precision");
    if (d->precision != ZKX_PRECISION_FP32 && nr != 4096 && nr != 8192 && nr != 16384)
        return fail(ZKX_UNSUPPORTED_OPERATION,
                    "rd_plan: tensor-core precision needs a range nfft of 4096, 8192 or 16384");
    if (d->cfar_mode != ZKX_CFAR_ACCURATE && d->cfar_mode != ZKX_CFAR_COMPAT)
        return fail(ZKX_INVALID_ARGUMENT, "rd_plan: unknown CFAR mode");
    CfarGeometry g;
    ZKX_TRY(cfar_checks(2, nd, nr, d->guard_cells[0], d->guard_cells[1], d->reference_cells[0],
                        d->reference_cells[1], d->pfa, &g));
    ZKX_TRY(ensure_device_ready());
    auto* p = new zkx_rd_plan_s;
    p->d = *d;
    p->range_nfft = nr;
    p->doppler_nfft = nd;
    p->cfar = g;
    cudaGetDevice(&p->device);
    cudaError_t e = cudaMalloc(&p->spectrum, (size_t)nr * sizeof(float2));
    if (e == cudaSuccess && d->doppler_window != ZKX_WINDOW_NONE)
        e = cudaMalloc(&p->doppler_window, (size_t)P * sizeof(float));
    if (e == cudaSuccess && d->cfar_mode == ZKX_CFAR_COMPAT) {
        e = cudaMalloc(&p->cumulative, (size_t)nd * nr * sizeof(float));
        if (e == cudaSuccess) p->cumulative_elems = (size_t)nd * nr;
    }
    if (e != cudaSuccess) {
        release_plan(p);
        return cuda_status(e, "rd_plan_create allocation");
    }
    int rc = launch_replica_spectrum(static_cast<const float2*>(replica), d->replica_length, nr,
                                     d->normalize, d->range_window, range_window, p->spectrum, stream);
    if (rc == ZKX_SUCCESS && p->doppler_window)
        rc = launch_doppler_window(P, d->doppler_window, doppler_window, p->doppler_window, stream);
    if (rc != ZKX_SUCCESS) {
        release_plan(p);
        return rc;
    }
    {
        std::lock_guard<std::mutex> lk(g_tune_mutex);
        auto it = g_tune_table.find(TuneKey{P, N, nr, nd});
        if (it != g_tune_table.end()) p->tuning = it->second;
    }
    *out = p;
    return ZKX_SUCCESS;
}

extern "C" int zkx_rd_plan_destroy(zkx_rd_plan plan)
{
    if (!plan) return ZKX_SUCCESS;
    release_plan(plan);
    return ZKX_SUCCESS;
}

extern "C" int zkx_rd_plan_shape(zkx_rd_plan plan, int* range_bins, int* doppler_bins)
{
    if (!plan) return fail(ZKX_INVALID_ARGUMENT, "rd_plan_shape: null plan");
    if (range_bins) *range_bins = plan->range_nfft;
    if (doppler_bins) *doppler_bins = plan->doppler_nfft;
    return ZKX_SUCCESS;
}

namespace zkx {
int rd_execute_batch_ws(zkx_rd_plan p, const void* x, int batch, void* compressed, void* rd,
                        float* power, float* threshold, uint8_t* detections, float* cumulative,
                        cudaStream_t stream, const void* const* table)
{
    if (!p || !(x || table) || !threshold || !detections)
        return fail(ZKX_INVALID_ARGUMENT, "rd_execute: null pointer");
    if (batch < 1) return fail(ZKX_INVALID_SHAPE, "rd_execute: batch must be positive");
    const int P = p->d.num_pulses, N = p->d.samples_per_pulse;
    const int nr = p->range_nfft, nd = p->doppler_nfft;
    if ((long long)batch * P * (nr > N ? nr : N) > INT_MAX || (long long)batch * nd * nr > INT_MAX)
        return fail(ZKX_INVALID_SHAPE, "rd_execute: batch exceeds kernel capacity");
    const size_t cube = (size_t)batch * P * nr, map = (size_t)batch * nd * nr;
    if (!compressed) {
        if (p->compressed_elems < cube) {
            cudaFree(p->compressed);
            p->compressed = nullptr;
            p->compressed_elems = 0;
            ZKX_CUDA(cudaMalloc(&p->compressed, cube * sizeof(float2)));
            p->compressed_elems = cube;
        }
        compressed = p->compressed;
    }
    if (!power) {
        if (p->power_elems < map) {
            cudaFree(p->power);
            p->power = nullptr;
            p->power_elems = 0;
            ZKX_CUDA(cudaMalloc(&p->power, map * sizeof(float)));
            p->power_elems = map;
        }
        power = p->power;
    }
    if (!cumulative) cumulative = p->cumulative;
    if (p->d.cfar_mode == ZKX_CFAR_COMPAT && !cumulative)
        return fail(ZKX_INTERNAL_ERROR, "rd_execute: compat workspace missing");
    // the CPIs of a batch are contiguous, so range compression sees batch*P pulses; the
    // default kernel is chosen from one CPI's shape, so a CPI gets the same bits alone and in
    // any batch
    int variant = p->tuning.compression_variant;
    ZKX_TRY(resolve_compression_variant(P, nr, variant, &variant));
    if (p->d.precision != ZKX_PRECISION_FP32) {
        if (table) return fail(ZKX_UNSUPPORTED_OPERATION, "rd_execute: tensor-core plans take contiguous batches");
        ZKX_TRY(launch_pulse_compression_tc(static_cast<const float2*>(x), batch * P, N, nr, p->spectrum,
                                            static_cast<float2*>(compressed), p->d.precision, stream));
    } else if (table)
        ZKX_TRY(launch_pulse_compression_table(reinterpret_cast<const float2* const*>(table), batch, P,
                                               N, nr, p->spectrum, static_cast<float2*>(compressed),
                                               variant, stream, p->tuning.compression_radix,
                                               p->tuning.compression_ctas_per_sm));
    else
        ZKX_TRY(launch_pulse_compression_variant(static_cast<const float2*>(x), batch * P, N, nr, p->spectrum,
                                                 static_cast<float2*>(compressed), variant, stream,
                                                 p->tuning.compression_radix, p->tuning.compression_ctas_per_sm));
    ZKX_TRY(launch_pulse_doppler(static_cast<const float2*>(compressed), P, nr, nd, p->doppler_window,
                                 static_cast<float2*>(rd), power, batch, p->tuning.doppler_columns, stream));
    const int* gd = p->d.guard_cells;
    const int* rf = p->d.reference_cells;
    if (p->d.cfar_mode == ZKX_CFAR_COMPAT) {
        for (int b = 0; b < batch; ++b)
            ZKX_TRY(launch_ca_cfar_compat(power + (size_t)b * nd * nr, 2, nd, nr, gd[0], gd[1], rf[0], rf[1],
                                          (float)p->cfar.alpha, p->cfar.nref, cumulative,
                                          threshold + (size_t)b * nd * nr, detections + (size_t)b * nd * nr,
                                          stream));
        return ZKX_SUCCESS;
    }
    return launch_ca_cfar_accurate(power, nd, nr, gd[0], gd[1], rf[0], rf[1], p->cfar.alpha,
                                   p->cfar.nref, threshold, detections, batch, p->tuning.cfar_tile, stream,
                                   p->tuning.cfar_ctas_per_sm);
}
}  // namespace zkx

namespace zkx {
int rd_plan_view(zkx_rd_plan p, RdPlanView* v)
{
    if (!p || !v) return fail(ZKX_INVALID_ARGUMENT, "null plan");
    v->d = p->d;
    v->range_nfft = p->range_nfft;
    v->doppler_nfft = p->doppler_nfft;
    v->spectrum = p->spectrum;
    v->doppler_window = p->doppler_window;
    v->cumulative = p->cumulative;
    v->alpha = p->cfar.alpha;
    v->nref = p->cfar.nref;
    v->tuning = p->tuning;
    return ZKX_SUCCESS;
}
}  // namespace zkx

extern "C" int zkx_rd_execute_batch(zkx_rd_plan p, const void* x, int batch, void* compressed,
                                    void* rd, float* power, float* threshold, uint8_t* detections,
                                    zkx_stream_t stream)
{
    return rd_execute_batch_ws(p, x, batch, compressed, rd, power, threshold, detections, nullptr,
                               stream, nullptr);
}

extern "C" int zkx_rd_execute(zkx_rd_plan p, const void* x, void* compressed, void* rd,
                              float* power, float* threshold, uint8_t* detections,
                              zkx_stream_t stream)
{
    return zkx_rd_execute_batch(p, x, 1, compressed, rd, power, threshold, detections, stream);
}

// ------------------------------------------------------------ autotuning

namespace {
// Median time in ms of `reps` launches of f on stream s after two warm-ups.
template <class F>
int time_median(F&& f, cudaStream_t s, float* ms)
{
    constexpr int kReps = 5;
    cudaEvent_t a, b;
    ZKX_CUDA(cudaEventCreate(&a));
    cudaError_t e = cudaEventCreate(&b);
    if (e != cudaSuccess) {
        cudaEventDestroy(a);
        return cuda_status(e, "autotune event");
    }
    float t[kReps];
    int rc = ZKX_SUCCESS;
    for (int i = 0; i < 2 && rc == ZKX_SUCCESS; ++i) rc = f();
    for (int i = 0; i < kReps && rc == ZKX_SUCCESS; ++i) {
        cudaEventRecord(a, s);
        rc = f();
        cudaEventRecord(b, s);
        e = cudaEventSynchronize(b);
        if (rc == ZKX_SUCCESS && e != cudaSuccess) rc = cuda_status(e, "autotune timing");
        if (rc == ZKX_SUCCESS) cudaEventElapsedTime(&t[i], a, b);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (rc != ZKX_SUCCESS) return rc;
    std::sort(t, t + kReps);
    *ms = t[kReps / 2];
    return ZKX_SUCCESS;
}
}  // namespace

extern "C" int zkx_rd_plan_autotune(zkx_rd_plan p, const void* x, int batch, zkx_stream_t stream,
                                    zkx_rd_tuning* chosen)
{
    if (!p || !x) return fail(ZKX_INVALID_ARGUMENT, "rd_plan_autotune: null pointer");
    if (batch < 1) return fail(ZKX_INVALID_SHAPE, "rd_plan_autotune: batch must be positive");
    const int P = p->d.num_pulses, N = p->d.samples_per_pulse, nr = p->range_nfft, nd = p->doppler_nfft;
    const size_t cube = (size_t)batch * P * nr, map = (size_t)batch * nd * nr;
    float2* comp = nullptr;
    float* power = nullptr;
    ZKX_CUDA(cudaMalloc(&comp, cube * sizeof(float2)));
    cudaError_t e = cudaMalloc(&power, map * sizeof(float));
    if (e != cudaSuccess) {
        cudaFree(comp);
        return cuda_status(e, "rd_plan_autotune allocation");
    }
    zkx_rd_tuning best = p->tuning;
    int rc = ZKX_SUCCESS;
    if (p->d.precision == ZKX_PRECISION_FP32) {
        auto time_compression = [&](int v, int radix, int ctas, float* ms) {
            return time_median([&] {
                return launch_pulse_compression_variant(static_cast<const float2*>(x), batch * P, N, nr,
                                                        p->spectrum, comp, v, stream, radix, ctas);
            }, stream, ms);
        };
        // the kernel, then the radix plan of the Stockham kernels, then the CTAs per SM of
        // the persistent ones
        float tbest = 0.f;
        best.compression_radix = 0;
        best.compression_ctas_per_sm = 0;
        for (int v : {ZKX_COMPRESSION_PLAIN, ZKX_COMPRESSION_PERSISTENT, ZKX_COMPRESSION_LOCAL}) {
            float ms = 0.f;
            rc = time_compression(v, 0, 0, &ms);
            if (rc != ZKX_SUCCESS) break;
            if (v == ZKX_COMPRESSION_PLAIN || ms < tbest) {
                tbest = ms;
                best.compression_variant = v;
            }
        }
        const int alt = compression_alt_radix(nr);
        if (rc == ZKX_SUCCESS && alt != 0 && best.compression_variant != ZKX_COMPRESSION_LOCAL) {
            float ms = 0.f;
            rc = time_compression(best.compression_variant, alt, 0, &ms);
            if (rc == ZKX_SUCCESS && ms < tbest) {
                tbest = ms;
                best.compression_radix = alt;
            }
        }
        if (is_pow2(nr) && nr <= 16384 && best.compression_variant != ZKX_COMPRESSION_PLAIN) {
            for (int k : {1, 2}) {
                if (rc != ZKX_SUCCESS) break;
                float ms = 0.f;
                rc = time_compression(best.compression_variant, best.compression_radix, k, &ms);
                if (rc == ZKX_SUCCESS && ms < tbest) {
                    tbest = ms;
                    best.compression_ctas_per_sm = k;
                }
            }
        }
    }
    if (rc == ZKX_SUCCESS) {
        float tbest = 0.f;
        // bulk-copy tile widths: 16 or 8 columns; 8 or 4 at 2048 pulses; 4 or 2 at 4096,
        // or its per-thread-load kernel (1)
        std::vector<int> widths = nd == 2048 ? std::vector<int>{8, 4}
                                  : nd == 4096 ? std::vector<int>{4, 2, 1} : std::vector<int>{16, 8};
        for (int c : widths) {
            float ms = 0.f;
            rc = time_median([&] {
                return launch_pulse_doppler(comp, P, nr, nd, p->doppler_window, nullptr, power, batch, c, stream);
            }, stream, &ms);
            if (rc != ZKX_SUCCESS) break;
            if (c == widths[0] || ms < tbest) {
                tbest = ms;
                best.doppler_columns = c;
            }
        }
    }
    if (rc == ZKX_SUCCESS && p->d.cfar_mode == ZKX_CFAR_ACCURATE) {
        // both CA-CFAR kernels on the power map the Doppler candidates left behind
        float* thr = nullptr;
        uint8_t* det = nullptr;
        cudaError_t ea = cudaMalloc(&thr, map * sizeof(float));
        if (ea == cudaSuccess) ea = cudaMalloc(&det, map);
        if (ea != cudaSuccess) {
            rc = cuda_status(ea, "rd_plan_autotune allocation");
        } else {
            const int* gd = p->d.guard_cells;
            const int* rf = p->d.reference_cells;
            float tbest = 0.f;
            for (int tile : {ZKX_CFAR_TILE_FULL, ZKX_CFAR_TILE_HALVES, ZKX_CFAR_TILE_STREAM}) {
                float ms = 0.f;
                rc = time_median([&] {
                    return launch_ca_cfar_accurate(power, nd, nr, gd[0], gd[1], rf[0], rf[1], p->cfar.alpha,
                                                   p->cfar.nref, thr, det, batch, tile, stream);
                }, stream, &ms);
                if (rc != ZKX_SUCCESS) break;
                if (tile == ZKX_CFAR_TILE_FULL || ms < tbest) {
                    tbest = ms;
                    best.cfar_tile = tile;
                }
            }
            best.cfar_ctas_per_sm = 0;
            if (rc == ZKX_SUCCESS && best.cfar_tile == ZKX_CFAR_TILE_STREAM) {
                float ms = 0.f;
                rc = time_median([&] {
                    return launch_ca_cfar_accurate(power, nd, nr, gd[0], gd[1], rf[0], rf[1], p->cfar.alpha,
                                                   p->cfar.nref, thr, det, batch, ZKX_CFAR_TILE_STREAM, stream, 1);
                }, stream, &ms);
                if (rc == ZKX_SUCCESS && ms < tbest) best.cfar_ctas_per_sm = 1;
            }
        }
        cudaFree(thr);
        cudaFree(det);
    }
    cudaFree(comp);
    cudaFree(power);
    if (rc != ZKX_SUCCESS) return rc;
    p->tuning = best;
    {
        std::lock_guard<std::mutex> lk(g_tune_mutex);
        g_tune_table[TuneKey{P, N, nr, nd}] = best;
    }
    if (chosen) *chosen = best;
    return ZKX_SUCCESS;
}

extern "C" int zkx_rd_plan_get_tuning(zkx_rd_plan p, zkx_rd_tuning* t)
{
    if (!p || !t) return fail(ZKX_INVALID_ARGUMENT, "rd_plan_get_tuning: null pointer");
    *t = p->tuning;
    return ZKX_SUCCESS;
}

extern "C" int zkx_rd_plan_set_tuning(zkx_rd_plan p, const zkx_rd_tuning* t)
{
    if (!p || !t) return fail(ZKX_INVALID_ARGUMENT, "rd_plan_set_tuning: null pointer");
    if (t->compression_variant < 0 || t->compression_variant > ZKX_COMPRESSION_LOCAL ||
        (t->doppler_columns != 0 && t->doppler_columns != 1 && t->doppler_columns != 2 &&
         t->doppler_columns != 4 && t->doppler_columns != 8 && t->doppler_columns != 16) ||
        t->cfar_tile < 0 || t->cfar_tile > ZKX_CFAR_TILE_STREAM ||
        (t->compression_radix != 0 && t->compression_radix != 16 && t->compression_radix != 32) ||
        t->compression_ctas_per_sm < 0 || t->compression_ctas_per_sm > 32 || t->cfar_ctas_per_sm < 0 ||
        t->cfar_ctas_per_sm > 32)
        return fail(ZKX_INVALID_ARGUMENT, "rd_plan_set_tuning: unknown kernel choice");
    p->tuning = *t;
    return ZKX_SUCCESS;
}

// ------------------------------------------------------------ graph capture

struct zkx_rd_graph_s {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

extern "C" int zkx_rd_graph_create(zkx_rd_plan p, const void* x, int batch, void* compressed, void* rd,
                                   float* power, float* threshold, uint8_t* detections,
                                   zkx_rd_graph* out)
{
    if (!out) return fail(ZKX_INVALID_ARGUMENT, "rd_graph_create: null pointer");
    *out = nullptr;
    // one eager run first: allocates plan-owned buffers and sets kernel attributes, so
    // the captured launches neither allocate nor change state
    cudaStream_t s;
    ZKX_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    int rc = zkx_rd_execute_batch(p, x, batch, compressed, rd, power, threshold, detections, s);
    if (rc == ZKX_SUCCESS) {
        const cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) rc = cuda_status(e, "rd_graph_create warm-up");
    }
    cudaGraph_t graph = nullptr;
    if (rc == ZKX_SUCCESS) {
        cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) rc = cuda_status(e, "cudaStreamBeginCapture");
        else {
            rc = zkx_rd_execute_batch(p, x, batch, compressed, rd, power, threshold, detections, s);
            e = cudaStreamEndCapture(s, &graph);
            if (rc == ZKX_SUCCESS && e != cudaSuccess) rc = cuda_status(e, "cudaStreamEndCapture");
        }
    }
    cudaGraphExec_t exec = nullptr;
    if (rc == ZKX_SUCCESS) {
        const cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
        if (e != cudaSuccess) rc = cuda_status(e, "cudaGraphInstantiate");
    }
    cudaStreamDestroy(s);
    if (rc != ZKX_SUCCESS) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    auto* g = new zkx_rd_graph_s;
    g->graph = graph;
    g->exec = exec;
    *out = g;
    return ZKX_SUCCESS;
}

extern "C" int zkx_rd_graph_launch(zkx_rd_graph g, zkx_stream_t stream)
{
    if (!g) return fail(ZKX_INVALID_ARGUMENT, "rd_graph_launch: null graph");
    ZKX_CUDA(cudaGraphLaunch(g->exec, stream));
    return ZKX_SUCCESS;
}

extern "C" int zkx_rd_graph_destroy(zkx_rd_graph g)
{
    if (!g) return ZKX_SUCCESS;
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
    return ZKX_SUCCESS;
}
