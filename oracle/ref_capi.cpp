// Test infrastructure only: a C-ABI shim over the reference library's own CPU
// implementations (the `*_typed_cpu` functions of ZKX/cusignal_cpp), so that the
// Python tests, the golden-fixture script and bench.py's CPU baseline can call the
// unmodified reference algorithms through ctypes.  This file is compiled together
// with the reference sources by oracle/Makefile into oracle/_ref/libzkx_ref.so; it is
// never linked into the product library.
//
// Every entry point returns 0 on success and a nonzero code on failure; the text
// of the last failure is available from zkx_ref_last_error().
//
// Reference interfaces wrapped (paths within ZKX/cusignal_cpp):
//   pulse_compression_typed_cpu  src/operators/radartools/radartools_typed.cpp:618-675
//   pulse_doppler_typed_cpu      src/operators/radartools/radartools_typed.cpp:714-759
//   ca_cfar_typed_cpu            src/operators/radartools/radartools_typed.cpp:465-555
//   cfar_alpha_typed_cpu         src/operators/radartools/radartools_typed.cpp:592-603
//   firfilter_typed_cpu          src/operators/filtering/filtering_typed.cpp:1536-1590
//   upfirdn_typed_cpu            src/operators/filtering/filtering_typed.cpp:2548-2616
//   resample_poly_typed_cpu      src/operators/filtering/filtering_typed.cpp:2617-2716
//   firwin_typed_cpu             include/cusignal/operators/filter_design/filter_design_typed.h:132
//   kaiser_typed_cpu             include/cusignal/operators/windows/windows_typed.h:169
//   ambgfun_typed_cpu            src/operators/radartools/radartools_typed.cpp:330-463
//   firfilter2_typed_cpu         src/operators/filtering/filtering_typed.cpp:1631-1730
//   hilbert_typed_cpu            src/operators/filtering/filtering_typed.cpp:1819-1872
#include <cusignal/operators/radartools/radartools_typed.h>
#include <cusignal/operators/filtering/filtering_typed.h>
#include <cusignal/operators/filter_design/filter_design_typed.h>
#include <cusignal/operators/windows/windows_typed.h>

#include <cstdint>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

namespace {
thread_local std::string g_last_error;

template <class F>
int guarded(F&& body)
{
    try {
        body();
        return 0;
    } catch (const std::invalid_argument& e) {
        g_last_error = e.what();
        return 1001;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return 2099;
    } catch (...) {
        g_last_error = "unknown exception";
        return 2099;
    }
}

std::vector<cusignal::TypedComplex<float>> complex_vector(const float* interleaved, std::size_t count)
{
    std::vector<cusignal::TypedComplex<float>> v(count);
    for (std::size_t i = 0; i < count; ++i) v[i] = {interleaved[2 * i], interleaved[2 * i + 1]};
    return v;
}

void store_complex_result(const cusignal::RadarComplexCpuResult& r, double* out, int* is_fp64)
{
    if (r.is_fp64) {
        for (std::size_t i = 0; i < r.fp64.size(); ++i) {
            out[2 * i] = r.fp64[i].re;
            out[2 * i + 1] = r.fp64[i].im;
        }
    } else {
        for (std::size_t i = 0; i < r.fp32.size(); ++i) {
            out[2 * i] = static_cast<double>(r.fp32[i].re);
            out[2 * i + 1] = static_cast<double>(r.fp32[i].im);
        }
    }
    if (is_fp64) *is_fp64 = r.is_fp64 ? 1 : 0;
}
}  // namespace

extern "C" {

const char* zkx_ref_last_error(void) { return g_last_error.c_str(); }

// x: [P, N] interleaved complex64; tmpl: [L] interleaved complex64;
// out: [P, nfft] interleaved complex as double (FP32 results are widened exactly).
int zkx_ref_pulse_compression_f32(
    const float* x, int num_pulses, int samples_per_pulse,
    const float* tmpl, int template_length, int nfft, int normalize,
    int window_kind, const float* explicit_window, double* out, int* is_fp64)
{
    return guarded([&] {
        cusignal::PulseCompressionOptions o;
        o.num_pulses = num_pulses;
        o.samples_per_pulse = samples_per_pulse;
        o.normalize = normalize != 0;
        o.nfft = nfft;
        o.window = static_cast<cusignal::RadarWindowKind>(window_kind);
        const auto xv = complex_vector(x, static_cast<std::size_t>(num_pulses) * samples_per_pulse);
        const auto tv = complex_vector(tmpl, static_cast<std::size_t>(template_length));
        std::vector<float> w;
        if (explicit_window) w.assign(explicit_window, explicit_window + template_length);
        const auto r = cusignal::pulse_compression_typed_cpu<float>(
            xv, tv, o, explicit_window ? &w : nullptr);
        store_complex_result(r, out, is_fp64);
    });
}

// x: [P, N] interleaved complex64; out: [nfft, N] interleaved complex as double.
int zkx_ref_pulse_doppler_f32(
    const float* x, int num_pulses, int samples_per_pulse, int nfft,
    int window_kind, const float* explicit_window, double* out, int* is_fp64)
{
    return guarded([&] {
        cusignal::PulseDopplerOptions o;
        o.num_pulses = num_pulses;
        o.samples_per_pulse = samples_per_pulse;
        o.nfft = nfft;
        o.window = static_cast<cusignal::RadarWindowKind>(window_kind);
        const auto xv = complex_vector(x, static_cast<std::size_t>(num_pulses) * samples_per_pulse);
        std::vector<float> w;
        if (explicit_window) w.assign(explicit_window, explicit_window + num_pulses);
        const auto r = cusignal::pulse_doppler_typed_cpu<float>(
            xv, o, explicit_window ? &w : nullptr);
        store_complex_result(r, out, is_fp64);
    });
}

// rank 1: shape {rows}; rank 2: shape {rows, columns}.
int zkx_ref_ca_cfar_f32(
    const float* x, int rank, int rows, int columns,
    int guard_rows, int guard_columns, int reference_rows, int reference_columns,
    double pfa, float* threshold, std::uint8_t* detections)
{
    return guarded([&] {
        std::vector<int> shape;
        cusignal::CaCfarOptions o;
        o.pfa = pfa;
        if (rank >= 1) {
            shape.push_back(rows);
            o.guard_cells.push_back(guard_rows);
            o.reference_cells.push_back(reference_rows);
        }
        if (rank == 2) {
            shape.push_back(columns);
            o.guard_cells.push_back(guard_columns);
            o.reference_cells.push_back(reference_columns);
        }
        std::size_t count = 1;
        for (int s : shape) count *= static_cast<std::size_t>(s);
        std::vector<float> xv(x, x + count);
        const auto r = cusignal::ca_cfar_typed_cpu<float>(xv, shape, o);
        std::memcpy(threshold, r.threshold.data(), r.threshold.size() * sizeof(float));
        for (std::size_t i = 0; i < r.detections.size(); ++i)
            detections[i] = static_cast<std::uint8_t>(r.detections[i]);
    });
}

int zkx_ref_cfar_alpha_f32(float pfa, int reference, double* out)
{
    return guarded([&] { *out = cusignal::cfar_alpha_typed_cpu<float>(pfa, reference); });
}

// x: row-major [rows, n] filtered along the last axis; y: [rows, n].
// zi (optional): [rows, nb-1]; zf (written when zi is given): [rows, nb-1].
int zkx_ref_firfilter_f32(
    const float* b, int nb, const float* x, int rows, int n,
    const float* zi, float* y, float* zf)
{
    return guarded([&] {
        cusignal::FirfilterOptions o;
        o.shape = {rows, n};
        o.axis = -1;
        std::vector<float> bv(b, b + nb);
        std::vector<float> xv(x, x + static_cast<std::size_t>(rows) * n);
        std::vector<float> ziv;
        if (zi) {
            ziv.assign(zi, zi + static_cast<std::size_t>(rows) * (nb - 1));
            o.zi_shape = {rows, nb - 1};
        }
        const auto r = cusignal::firfilter_typed_cpu<float>(bv, xv, o, zi ? &ziv : nullptr);
        std::memcpy(y, r.y.data(), r.y.size() * sizeof(float));
        if (zi && zf) std::memcpy(zf, r.zf.data(), r.zf.size() * sizeof(float));
    });
}

// x: row-major [rows, n] resampled along the last axis; out sized by the caller
// from zkx_ref_upfirdn_length.
int zkx_ref_upfirdn_f32(
    const float* h, int nh, const float* x, int rows, int n,
    int up, int down, float* out, int* out_samples)
{
    return guarded([&] {
        cusignal::UpfirdnOptions o;
        o.shape = {rows, n};
        o.axis = -1;
        std::vector<float> hv(h, h + nh);
        std::vector<float> xv(x, x + static_cast<std::size_t>(rows) * n);
        const auto r = cusignal::upfirdn_typed_cpu<float>(hv, xv, up, down, o);
        std::memcpy(out, r.fp32.data(), r.fp32.size() * sizeof(float));
        *out_samples = r.shape.back();
    });
}

// Default Kaiser(beta) design when coeffs == nullptr, otherwise custom taps.
// out receives doubles (FP32 results are widened exactly); *is_fp64 tells which.
int zkx_ref_resample_poly_f32(
    const float* x, int rows, int n, int up, int down, double kaiser_beta,
    const float* coeffs, int ncoeffs, double* out, int* out_samples, int* is_fp64)
{
    return guarded([&] {
        cusignal::ResamplePolyOptions o;
        o.shape = {rows, n};
        o.axis = 1;
        o.kaiser_beta = kaiser_beta;
        std::vector<float> xv(x, x + static_cast<std::size_t>(rows) * n);
        std::vector<float> cv;
        if (coeffs) cv.assign(coeffs, coeffs + ncoeffs);
        const auto r = cusignal::resample_poly_typed_cpu<float>(
            xv, up, down, o, coeffs ? &cv : nullptr);
        *out_samples = r.shape.back();
        if (r.dtype == cusignal::ResamplePolyOutputDtype::fp64) {
            std::memcpy(out, r.fp64.data(), r.fp64.size() * sizeof(double));
            *is_fp64 = 1;
        } else {
            for (std::size_t i = 0; i < r.fp32.size(); ++i) out[i] = r.fp32[i];
            *is_fp64 = 0;
        }
    });
}

// Lowpass design used by the front end: firwin(numtaps, cutoff) with an explicit
// Kaiser(beta) window, fs = 2 convention, scale = true.
int zkx_ref_firwin_kaiser(int numtaps, double cutoff, double beta, double* out)
{
    return guarded([&] {
        cusignal::FirwinOptions o;
        o.window_mode = cusignal::FirwinWindowMode::explicit_values;
        o.window = cusignal::kaiser_typed_cpu<float>(numtaps, static_cast<float>(beta));
        const auto taps = cusignal::firwin_typed_cpu<float>(
            numtaps, std::vector<float>{static_cast<float>(cutoff)}, o);
        std::memcpy(out, taps.data(), taps.size() * sizeof(double));
    });
}

}  // extern "C"

// ambgfun_typed_cpu<float>.  x [x_count] with logical shape {nx, x_count / nx} when
// x_count != nx (only the 2-D cut accepts that); y = NULL means y = x.  out receives the
// values as double (FP32 results widened); *shape0 / *shape1 the result shape.
extern "C" int zkx_ref_ambgfun_f32(const float* x, int x_count, int nx, const float* y,
                                   int y_count, int ny, int cut, double fs, double cut_value,
                                   double* out, int* is_fp64)
{
    return guarded([&] {
        cusignal::AmbgfunOptions o;
        o.fs = fs;
        o.cut = static_cast<cusignal::AmbgfunCut>(cut);
        o.cut_value = cut_value;
        if (x_count != nx) o.input_shape = {nx, x_count / nx};
        const auto xv = complex_vector(x, static_cast<std::size_t>(x_count));
        std::vector<cusignal::TypedComplex<float>> yv;
        if (y) {
            yv = complex_vector(y, static_cast<std::size_t>(y_count));
            if (y_count != ny) o.reference_shape = {ny, y_count / ny};
        }
        const auto r = cusignal::ambgfun_typed_cpu<float>(xv, o, y ? &yv : nullptr);
        *is_fp64 = r.dtype == cusignal::AmbgfunOutputDtype::fp64 ? 1 : 0;
        if (*is_fp64) {
            std::memcpy(out, r.fp64.data(), r.fp64.size() * sizeof(double));
        } else {
            for (std::size_t i = 0; i < r.fp32.size(); ++i) out[i] = r.fp32[i];
        }
    });
}

// firfilter2_typed_cpu<T> and hilbert_typed_cpu<T> for the element types the reference
// instantiates (dtype 0 float, 1 __half, 2 int32, 3 int16, 4 int8; b and x hold raw
// elements of that type).  x has row-major `shape` (rank entries) and is filtered along
// `axis`; results are widened to double (complex results interleaved), *is_fp64 tells
// whether the reference produced FP64 storage.
//   firfilter2_typed_cpu   src/operators/filtering/filtering_typed.cpp:1631-1730
//   hilbert_typed_cpu      src/operators/filtering/filtering_typed.cpp:1819-1872
namespace {
template <class T>
std::vector<T> typed_vector(const void* p, std::size_t n)
{
    const T* t = static_cast<const T*>(p);
    return std::vector<T>(t, t + n);
}

template <class T>
void run_firfilter2(const void* b, int nb, const void* x, const int* shape, int rank, int axis,
                    int padtype, int has_padlen, int padlen, double* out, int* is_fp64)
{
    cusignal::Firfilter2Options o;
    std::size_t count = 1;
    for (int i = 0; i < rank; ++i) {
        o.shape.push_back(shape[i]);
        count *= static_cast<std::size_t>(shape[i]);
    }
    o.axis = axis;
    o.padtype = static_cast<cusignal::Firfilter2PadType>(padtype);
    if (has_padlen) o.padlen = padlen;
    const auto r = cusignal::firfilter2_typed_cpu<T>(typed_vector<T>(b, nb), typed_vector<T>(x, count), o);
    *is_fp64 = r.dtype == cusignal::Firfilter2OutputDtype::fp64 ? 1 : 0;
    if (*is_fp64) std::memcpy(out, r.fp64.data(), r.fp64.size() * sizeof(double));
    else for (std::size_t i = 0; i < r.fp32.size(); ++i) out[i] = r.fp32[i];
}

template <class T>
void run_hilbert(const void* x, const int* shape, int rank, int axis, int has_n, int n, double* out,
                 int* is_fp64)
{
    cusignal::HilbertOptions o;
    std::size_t count = 1;
    for (int i = 0; i < rank; ++i) {
        o.shape.push_back(shape[i]);
        count *= static_cast<std::size_t>(shape[i]);
    }
    o.axis = axis;
    if (has_n) o.fft_length = n;
    const auto r = cusignal::hilbert_typed_cpu<T>(typed_vector<T>(x, count), o);
    *is_fp64 = r.dtype == cusignal::HilbertOutputDtype::complex_fp64 ? 1 : 0;
    if (*is_fp64) {
        for (std::size_t i = 0; i < r.complex_fp64.size(); ++i) {
            out[2 * i] = r.complex_fp64[i].re;
            out[2 * i + 1] = r.complex_fp64[i].im;
        }
    } else {
        for (std::size_t i = 0; i < r.complex_fp32.size(); ++i) {
            out[2 * i] = r.complex_fp32[i].re;
            out[2 * i + 1] = r.complex_fp32[i].im;
        }
    }
}

template <class F>
void by_dtype(int dtype, F&& f)
{
    switch (dtype) {
    case 0: f(float{}); break;
    case 1: f(__half{}); break;
    case 2: f(std::int32_t{}); break;
    case 3: f(std::int16_t{}); break;
    case 4: f(std::int8_t{}); break;
    default: throw std::invalid_argument("dtype");
    }
}
}  // namespace

extern "C" int zkx_ref_firfilter2(int dtype, const void* b, int nb, const void* x, const int* shape, int rank,
                                  int axis, int padtype, int has_padlen, int padlen, double* out,
                                  int* is_fp64)
{
    return guarded([&] {
        by_dtype(dtype, [&](auto tag) {
            run_firfilter2<decltype(tag)>(b, nb, x, shape, rank, axis, padtype, has_padlen, padlen, out, is_fp64);
        });
    });
}

extern "C" int zkx_ref_hilbert(int dtype, const void* x, const int* shape, int rank, int axis, int has_n, int n,
                               double* out, int* is_fp64)
{
    return guarded([&] {
        by_dtype(dtype, [&](auto tag) {
            run_hilbert<decltype(tag)>(x, shape, rank, axis, has_n, n, out, is_fp64);
        });
    });
}
