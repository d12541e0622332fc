// cusignal_cpp filtering operators on the radar front end -- firfilter, upfirdn,
// resample_poly, and the adjacent firfilter2 and hilbert -- with the signatures of
// ZKX/cusignal_cpp/include/cusignal/operators/filtering/filtering_typed.h (552-567,
// 745-770), implemented over libzkx_rd.so.  T is one of float, __half, int32_t,
// int16_t, int8_t; non-float inputs are converted to FP32 on the device first, as the
// reference does.  Arrays are row-major; inputs of rank 1 or 2 are supported (any axis),
// higher ranks when the filtered axis is the last one.  Work runs on the legacy default
// stream.  The *_typed_cpu CPU references keep their declarations for callers that link
// the reference's own CPU implementation.
#pragma once

#include <cuda_fp16.h>

#include <cusignal/backends/fft/fft_interface.h>
#include <cusignal/detail/zkx_call.h>
#include <cusignal/runtime/cuda_utils.h>
#include <cusignal/runtime/device_array.h>

#include <cmath>
#include <cstdint>
#include <numeric>
#include <optional>
#include <stdexcept>
#include <type_traits>
#include <vector>

namespace cusignal {

template <typename T>
struct TypedComplex {
    T real;
    T imag;
};

enum class ResamplePolyWindowMode { kaiser, hamming, explicit_values };
enum class ResamplePolyOutputDtype { fp16, fp32, fp64, int32, int16, int8 };
enum class UpfirdnOutputDtype { fp32, fp64 };

struct UpfirdnOptions {
    std::vector<int> shape;
    int axis = -1;
};

struct UpfirdnCpuResult {
    UpfirdnOutputDtype dtype{UpfirdnOutputDtype::fp32};
    std::vector<float> fp32;
    std::vector<double> fp64;
    std::vector<int> shape;
};

struct UpfirdnDeviceResult {
    UpfirdnOutputDtype dtype{UpfirdnOutputDtype::fp32};
    DeviceArray<float> fp32;
    DeviceArray<double> fp64;
    std::vector<int> shape;
};

struct ResamplePolyOptions {
    std::vector<int> shape;
    int axis = 0;
    ResamplePolyWindowMode window_mode = ResamplePolyWindowMode::kaiser;
    double kaiser_beta = 5.0;
    std::vector<double> design_window;
    bool gpupath = true;
};

struct ResamplePolyCpuResult {
    ResamplePolyOutputDtype dtype{ResamplePolyOutputDtype::fp64};
    std::vector<__half> fp16;
    std::vector<float> fp32;
    std::vector<double> fp64;
    std::vector<std::int32_t> int32;
    std::vector<std::int16_t> int16;
    std::vector<std::int8_t> int8;
    std::vector<int> shape;
};

struct ResamplePolyDeviceResult {
    ResamplePolyOutputDtype dtype{ResamplePolyOutputDtype::fp64};
    DeviceArray<__half> fp16;
    DeviceArray<float> fp32;
    DeviceArray<double> fp64;
    DeviceArray<std::int32_t> int32;
    DeviceArray<std::int16_t> int16;
    DeviceArray<std::int8_t> int8;
    std::vector<int> shape;
};

struct FirfilterOptions {
    std::vector<int> shape;
    int axis = -1;
    std::vector<int> zi_shape;
};

struct FirfilterCpuResult {
    std::vector<float> y;
    std::vector<float> zf;
    std::vector<int> y_shape;
    std::vector<int> zf_shape;
    bool has_zf = false;
};

struct FirfilterDeviceResult {
    DeviceArray<float> y;
    DeviceArray<float> zf;
    std::vector<int> y_shape;
    std::vector<int> zf_shape;
    bool has_zf = false;
};

enum class Firfilter2PadType { odd, even, constant, none };
enum class Firfilter2Method { pad, gust };
enum class Firfilter2OutputDtype { fp32, fp64 };

struct Firfilter2Options {
    std::vector<int> shape;
    int axis = -1;
    Firfilter2PadType padtype = Firfilter2PadType::odd;
    std::optional<int> padlen;
    Firfilter2Method method = Firfilter2Method::pad;
    std::optional<int> irlen;  // ignored by the pad method, as in the reference
};

struct Firfilter2CpuResult {
    Firfilter2OutputDtype dtype{Firfilter2OutputDtype::fp32};
    std::vector<float> fp32;
    std::vector<double> fp64;
    std::vector<int> shape;
};

struct Firfilter2DeviceResult {
    Firfilter2OutputDtype dtype{Firfilter2OutputDtype::fp32};
    DeviceArray<float> fp32;
    DeviceArray<double> fp64;
    std::vector<int> shape;
};

enum class HilbertOutputDtype { complex_fp32, complex_fp64 };

struct HilbertOptions {
    std::vector<int> shape;
    std::optional<int> fft_length;
    int axis = -1;
};

struct HilbertCpuResult {
    HilbertOutputDtype dtype{HilbertOutputDtype::complex_fp32};
    std::vector<ComplexFloat> complex_fp32;
    std::vector<ComplexDouble> complex_fp64;
    std::vector<int> shape;
};

struct HilbertDeviceResult {
    HilbertOutputDtype dtype{HilbertOutputDtype::complex_fp32};
    DeviceArray<ComplexFloat> complex_fp32;
    DeviceArray<ComplexDouble> complex_fp64;
    std::vector<int> shape;
};

namespace detail {

template <typename T>
constexpr int zkx_dtype()
{
    if constexpr (std::is_same_v<T, float>) return ZKX_DTYPE_F32;
    else if constexpr (std::is_same_v<T, __half>) return ZKX_DTYPE_F16;
    else if constexpr (std::is_same_v<T, std::int32_t>) return ZKX_DTYPE_I32;
    else if constexpr (std::is_same_v<T, std::int16_t>) return ZKX_DTYPE_I16;
    else if constexpr (std::is_same_v<T, std::int8_t>) return ZKX_DTYPE_I8;
    else static_assert(!sizeof(T), "unsupported business dtype: float, __half, int32, int16 or int8");
}

// FP32 staging copy of `count` scalars of device data of type T.
template <typename T>
DeviceArray<float> staged_f32(const void* data, std::size_t count)
{
    DeviceArray<float> out(count);
    if (count) zkx_check(zkx_convert_to_f32(data, zkx_dtype<T>(), (long long)count, out.data(), nullptr));
    return out;
}

inline DeviceArray<double> widened(const DeviceArray<float>& a)
{
    DeviceArray<double> out(a.size());
    if (a.size()) zkx_check(zkx_widen_f32_to_f64(a.data(), (long long)a.size(), out.data(), nullptr));
    return out;
}

// Row-major shape -> (outer lines, samples along axis, inner stride); only layouts the
// last-axis kernels can run directly or after one 2-D transpose are accepted.
struct AxisLayout {
    std::vector<int> shape;
    int axis = 0;
    long long lines = 1;
    int samples = 0;
    bool transpose = false;  // rank-2 input filtered along axis 0
};

inline AxisLayout axis_layout(std::size_t size, const std::vector<int>& shape_in, int axis, const char* fn)
{
    AxisLayout a;
    a.shape = shape_in.empty() ? std::vector<int>{static_cast<int>(size)} : shape_in;
    long long prod = 1;
    for (int e : a.shape) {
        if (e < 0) throw std::invalid_argument(std::string(fn) + " input shape");
        prod *= e;
    }
    if (prod != (long long)size) throw std::invalid_argument(std::string(fn) + " input shape product");
    const int rank = static_cast<int>(a.shape.size());
    a.axis = axis < 0 ? axis + rank : axis;
    if (a.axis < 0 || a.axis >= rank) throw std::invalid_argument(std::string(fn) + " axis");
    a.samples = a.shape[a.axis];
    if (a.axis != rank - 1) {
        if (rank != 2) throw std::invalid_argument(std::string(fn) + ": only the last axis of inputs above rank 2");
        a.transpose = true;
    }
    a.lines = a.samples ? prod / a.samples : 0;
    return a;
}

// Moves the filtered axis last (rank-2 axis-0 inputs) or returns the staged input.
inline DeviceArray<float> axis_last(DeviceArray<float>&& x, const AxisLayout& a)
{
    if (!a.transpose) return std::move(x);
    DeviceArray<float> t(x.size());
    zkx_check(zkx_transpose_f32(x.data(), a.shape[0], a.shape[1], t.data(), nullptr));
    return t;
}

// Inverse of axis_last for a result with `out_samples` along the filtered axis.
inline DeviceArray<float> axis_back(DeviceArray<float>&& y, const AxisLayout& a, int out_samples)
{
    if (!a.transpose) return std::move(y);
    DeviceArray<float> t(y.size());
    zkx_check(zkx_transpose_f32(y.data(), a.shape[1], out_samples, t.data(), nullptr));
    return t;
}

}  // namespace detail

/// Causal FIR along options.axis (same length as x); with zi also the final state zf.
template <typename T>
void firfilter_device(const DeviceArray<T>& b, const DeviceArray<T>& x, FirfilterDeviceResult& out,
                      const FirfilterOptions& options = {}, const DeviceArray<T>* zi = nullptr)
{
    if (b.empty()) throw std::invalid_argument("firfilter coefficients");
    const auto a = detail::axis_layout(x.size(), options.shape, options.axis, "firfilter");
    for (int e : a.shape)
        if (e <= 0) throw std::invalid_argument("firfilter input shape");
    const int nb = static_cast<int>(b.size());
    auto bf = detail::staged_f32<T>(b.data(), b.size());
    auto xf = detail::axis_last(detail::staged_f32<T>(x.data(), x.size()), a);
    out = FirfilterDeviceResult{};
    out.y_shape = a.shape;
    DeviceArray<float> y(x.size());
    DeviceArray<float> zif, zf;
    if (zi) {
        std::vector<int> state = a.shape;
        state[a.axis] = nb - 1;
        std::vector<int> zshape = options.zi_shape.empty() ? state : options.zi_shape;
        if (zshape.size() != state.size()) throw std::invalid_argument("firfilter zi rank");
        long long zprod = 1;
        for (std::size_t d = 0; d < state.size(); ++d) {
            const bool ok = (int)d == a.axis ? zshape[d] == state[d] : (zshape[d] == state[d] || zshape[d] == 1);
            if (!ok) throw std::invalid_argument("firfilter zi broadcast shape");
            zprod *= zshape[d];
        }
        if (zprod != (long long)zi->size()) throw std::invalid_argument("firfilter zi shape product");
        // expand a broadcast state to one row per line, in the axis-last layout
        auto zstage = detail::staged_f32<T>(zi->data(), zi->size());
        zif = DeviceArray<float>((std::size_t)a.lines * (nb - 1));
        if (nb > 1) {
            if (zprod == a.lines * (long long)(nb - 1) && !a.transpose) {
                cuda_utils::copy_device_to_device(zif.data(), zstage.data(), zif.size());
            } else {
                auto host = zstage.to_host();
                std::vector<float> rows((std::size_t)a.lines * (nb - 1));
                const bool axis0 = a.transpose;
                for (long long l = 0; l < a.lines; ++l)
                    for (int j = 0; j < nb - 1; ++j) {
                        std::size_t src;
                        if (axis0) src = (std::size_t)j * zshape[1] + (zshape[1] == 1 ? 0 : l);
                        else src = (zprod == nb - 1 ? 0 : (std::size_t)l * (nb - 1)) + j;
                        rows[(std::size_t)l * (nb - 1) + j] = host[src];
                    }
                cuda_utils::copy_to_device(zif.data(), rows.data(), rows.size());
                cuda_utils::synchronize_stream();
            }
        }
        zf = DeviceArray<float>((std::size_t)a.lines * (nb - 1));
        out.zf_shape = state;
        out.has_zf = true;
    }
    detail::zkx_check(zkx_fir_f32(bf.data(), nb, xf.data(), (int)a.lines, a.samples,
                                  zi ? zif.data() : nullptr, y.data(), zi ? zf.data() : nullptr, nullptr));
    out.y = detail::axis_back(std::move(y), a, a.samples);
    if (zi) {
        if (a.transpose) {
            DeviceArray<float> t(zf.size());
            if (zf.size()) detail::zkx_check(zkx_transpose_f32(zf.data(), (int)a.lines, nb - 1, t.data(), nullptr));
            out.zf = std::move(t);
        } else {
            out.zf = std::move(zf);
        }
    }
}

/// One-dimensional FP32 FIR with caller-owned output (a single kernel, no staging).
inline void firfilter_fp32_resident_device(const DeviceArray<float>& b, const DeviceArray<float>& x,
                                           DeviceArray<float>& y)
{
    if (b.empty()) throw std::invalid_argument("firfilter coefficients");
    if (y.size() != x.size()) throw std::invalid_argument("firfilter resident output size mismatch");
    if (x.empty()) return;
    detail::zkx_check(zkx_fir_f32(b.data(), (int)b.size(), x.data(), 1, (int)x.size(), nullptr, y.data(),
                                  nullptr, nullptr));
}

/// Upsample by up, filter with h, downsample by down (causal, zero extension).
template <typename T>
void upfirdn_device(const DeviceArray<T>& h, const DeviceArray<T>& x, int up, int down,
                    UpfirdnDeviceResult& out, const UpfirdnOptions& options = {})
{
    if (h.empty()) throw std::invalid_argument("upfirdn coefficients");
    if (up < 1 || down < 1) throw std::invalid_argument("upfirdn factors");
    const auto a = detail::axis_layout(x.size(), options.shape, options.axis, "upfirdn");
    if (a.shape.size() > 2) throw std::invalid_argument("upfirdn rank");
    const long long nout = zkx_upfirdn_length(a.samples, (int)h.size(), up, down);
    if (nout < 0 || nout > 2147483647LL) throw std::invalid_argument("upfirdn output sample count");
    out = UpfirdnDeviceResult{};
    out.shape = a.shape;
    out.shape[a.axis] = (int)nout;
    auto hf = detail::staged_f32<T>(h.data(), h.size());
    auto xf = detail::axis_last(detail::staged_f32<T>(x.data(), x.size()), a);
    DeviceArray<float> y((std::size_t)a.lines * nout);
    if (a.lines > 0 && nout > 0)
        detail::zkx_check(zkx_upfirdn_f32(hf.data(), (int)h.size(), xf.data(), (int)a.lines, a.samples, up,
                                          down, y.data(), nullptr));
    auto yf = detail::axis_back(std::move(y), a, (int)nout);
    if constexpr (std::is_same_v<T, std::int32_t>) {
        out.dtype = UpfirdnOutputDtype::fp64;
        out.fp64 = detail::widened(yf);
    } else {
        out.dtype = UpfirdnOutputDtype::fp32;
        cuda_utils::synchronize_stream();
        out.fp32 = std::move(yf);
    }
}

namespace detail {

// up * coefficient with the reference's promotion and wrap rules for custom taps
// (filtering_typed.cpp:103-157), evaluated on the host.
template <typename T>
double scaled_custom_tap(T v, int up)
{
    if constexpr (std::is_same_v<T, float>) {
        return up < 65536 ? (double)(v * (float)up) : (double)v * (double)up;
    } else if constexpr (std::is_same_v<T, __half>) {
        const float f = __half2float(v);
        if (up <= 255) return (double)__half2float(__float2half_rn(f * (float)up));
        return up < 65536 ? (double)(f * (float)up) : (double)f * (double)up;
    } else {
        auto wrap = [](long long value, int bits) {
            const unsigned long long mod = 1ULL << bits;
            unsigned long long u = (unsigned long long)value & (mod - 1);
            return (double)(u >= (mod >> 1) ? (long long)u - (long long)mod : (long long)u);
        };
        int bits = 32;
        if constexpr (std::is_same_v<T, std::int16_t>) bits = up < 32768 ? 16 : 32;
        if constexpr (std::is_same_v<T, std::int8_t>) bits = up <= 127 ? 8 : (up < 32768 ? 16 : 32);
        return wrap((long long)v * (long long)up, bits);
    }
}

}  // namespace detail

/// Rational resampling by up/down (gcd-reduced) with the reference's output dtypes:
/// identity keeps T, the default design stores FP64, custom taps FP32 or FP64.
template <typename T>
void resample_poly_device(const DeviceArray<T>& x, int up, int down, ResamplePolyDeviceResult& out,
                          const ResamplePolyOptions& options = {},
                          const DeviceArray<T>* coefficients = nullptr)
{
    if (up < 1 || down < 1) throw std::invalid_argument("resample_poly factors");
    out = ResamplePolyDeviceResult{};
    const std::vector<int> shape = options.shape.empty() ? std::vector<int>{(int)x.size()} : options.shape;
    long long prod = 1;
    for (int e : shape) {
        if (e < 0) throw std::invalid_argument("resample_poly input shape");
        prod *= e;
    }
    if (prod != (long long)x.size()) throw std::invalid_argument("resample_poly input shape product");
    const int g = std::gcd(up, down);
    if (up / g == 1 && down / g == 1) {
        out.shape = shape;
        if constexpr (std::is_same_v<T, float>) { out.dtype = ResamplePolyOutputDtype::fp32; out.fp32 = DeviceArray<float>(x.size()); cuda_utils::copy_device_to_device(out.fp32.data(), x.data(), x.size()); }
        else if constexpr (std::is_same_v<T, __half>) { out.dtype = ResamplePolyOutputDtype::fp16; out.fp16 = DeviceArray<__half>(x.size()); cuda_utils::copy_device_to_device(out.fp16.data(), x.data(), x.size()); }
        else if constexpr (std::is_same_v<T, std::int32_t>) { out.dtype = ResamplePolyOutputDtype::int32; out.int32 = DeviceArray<std::int32_t>(x.size()); cuda_utils::copy_device_to_device(out.int32.data(), x.data(), x.size()); }
        else if constexpr (std::is_same_v<T, std::int16_t>) { out.dtype = ResamplePolyOutputDtype::int16; out.int16 = DeviceArray<std::int16_t>(x.size()); cuda_utils::copy_device_to_device(out.int16.data(), x.data(), x.size()); }
        else { out.dtype = ResamplePolyOutputDtype::int8; out.int8 = DeviceArray<std::int8_t>(x.size()); cuda_utils::copy_device_to_device(out.int8.data(), x.data(), x.size()); }
        cuda_utils::synchronize_stream();
        return;
    }
    if (shape.size() < 1 || shape.size() > 2) throw std::invalid_argument("resample_poly nonidentity rank");
    const auto a = detail::axis_layout(x.size(), shape, options.axis, "resample_poly");
    const bool custom = coefficients != nullptr;
    zkx_resample_layout lay;
    detail::zkx_check(zkx_resample_poly_layout(a.samples, up, down, custom ? 1 : 0,
                                               custom ? (int)coefficients->size() : 0, &lay));
    std::vector<float> taps32;
    if (custom) {
        auto host = coefficients->to_host();
        taps32.resize(host.size());
        for (std::size_t i = 0; i < host.size(); ++i) taps32[i] = (float)detail::scaled_custom_tap<T>(host[i], lay.up);
    } else {
        std::vector<double> taps(lay.coefficient_count);
        if (options.window_mode == ResamplePolyWindowMode::kaiser) {
            detail::zkx_check(zkx_resample_poly_design(&lay, options.kaiser_beta, taps.data()));
        } else {
            std::vector<double> window(lay.coefficient_count);
            if (options.window_mode == ResamplePolyWindowMode::hamming) {
                for (int i = 0; i < lay.coefficient_count; ++i)
                    window[i] = 0.54 - 0.46 * std::cos(6.283185307179586476925286766559 * i / (lay.coefficient_count - 1));
            } else if (options.window_mode == ResamplePolyWindowMode::explicit_values) {
                if (options.design_window.size() != (std::size_t)lay.coefficient_count)
                    throw std::invalid_argument("resample_poly design window shape");
                window = options.design_window;
            } else {
                throw std::invalid_argument("resample_poly window mode");
            }
            detail::zkx_check(zkx_resample_poly_design_window(&lay, window.data(), taps.data()));
        }
        taps32.assign(taps.begin(), taps.end());
    }
    auto dtaps = DeviceArray<float>::from_host(taps32);
    auto xf = detail::axis_last(detail::staged_f32<T>(x.data(), x.size()), a);
    DeviceArray<float> y((std::size_t)a.lines * lay.output_samples);
    detail::zkx_check(zkx_resample_poly_f32(xf.data(), (int)a.lines, a.samples, &lay, dtaps.data(), y.data(), nullptr));
    auto yf = detail::axis_back(std::move(y), a, lay.output_samples);
    out.shape = a.shape;
    out.shape[a.axis] = lay.output_samples;
    bool fp64 = !custom;
    if (custom) {
        if constexpr (std::is_same_v<T, std::int32_t>) fp64 = true;
        else if constexpr (std::is_same_v<T, std::int16_t> || std::is_same_v<T, std::int8_t>) fp64 = lay.up >= 32768;
        else fp64 = lay.up >= 65536;
    }
    if (fp64) {
        out.dtype = ResamplePolyOutputDtype::fp64;
        out.fp64 = detail::widened(yf);
    } else {
        out.dtype = ResamplePolyOutputDtype::fp32;
        cuda_utils::synchronize_stream();
        out.fp32 = std::move(yf);
    }
}

/// Zero-phase FIR along options.axis (filtering_typed.cpp:1226-1302, 1631-1730): padding by
/// odd / even / constant reflection of padlen samples (default 3 * len(b)), forward and backward
/// FIR with steady-state initial conditions, crop.  FP32 result; FP64 storage for int32 input.
/// Odd-reflected pad values keep the rounding / integer wrap of T.
template <typename T>
void firfilter2_device(const DeviceArray<T>& b, const DeviceArray<T>& x, Firfilter2DeviceResult& out,
                       const Firfilter2Options& options = {})
{
    if (b.empty()) throw std::invalid_argument("firfilter2 coefficients");
    if (options.method == Firfilter2Method::gust)
        throw std::invalid_argument("firfilter2 gust is not supported by cuSignal 23.08.00");
    if (options.method != Firfilter2Method::pad) throw std::invalid_argument("firfilter2 method");
    const auto a = detail::axis_layout(x.size(), options.shape, options.axis, "firfilter2");
    for (int e : a.shape)
        if (e <= 0) throw std::invalid_argument("firfilter2 input shape");
    int rounding = ZKX_PAD_ROUND_F32;
    if constexpr (std::is_same_v<T, __half>) rounding = ZKX_PAD_ROUND_F16;
    else if constexpr (std::is_same_v<T, std::int8_t>) rounding = ZKX_PAD_ROUND_I8;
    else if constexpr (std::is_same_v<T, std::int16_t>) rounding = ZKX_PAD_ROUND_I16;
    else if constexpr (std::is_same_v<T, std::int32_t>) rounding = ZKX_PAD_ROUND_I32;
    auto bf = detail::staged_f32<T>(b.data(), b.size());
    auto xf = detail::axis_last(detail::staged_f32<T>(x.data(), x.size()), a);
    DeviceArray<float> y(x.size());
    detail::zkx_check(zkx_firfilter2_f32(bf.data(), static_cast<int>(b.size()), xf.data(), (int)a.lines,
                                         a.samples, static_cast<int>(options.padtype),
                                         options.padlen.has_value() ? 1 : 0, options.padlen.value_or(0),
                                         rounding, y.data(), nullptr));
    y = detail::axis_back(std::move(y), a, a.samples);
    out.shape = a.shape;
    if constexpr (std::is_same_v<T, std::int32_t>) {
        out.dtype = Firfilter2OutputDtype::fp64;
        out.fp32 = DeviceArray<float>();
        out.fp64 = detail::widened(y);
    } else {
        out.dtype = Firfilter2OutputDtype::fp32;
        out.fp64 = DeviceArray<double>();
        cuda_utils::synchronize_stream();
        out.fp32 = std::move(y);
    }
}

/// Analytic signal along options.axis with N = options.fft_length (default the axis length)
/// (filtering_typed.cpp:500-562, 1819-1872).  ComplexFP32; ComplexFP64 for integer inputs.
template <typename T>
void hilbert_device(const DeviceArray<T>& x, HilbertDeviceResult& out, const HilbertOptions& options = {})
{
    const auto a = detail::axis_layout(x.size(), options.shape, options.axis, "hilbert");
    const int nfft = options.fft_length.value_or(a.samples);
    if (nfft <= 0) throw std::invalid_argument("hilbert N must be positive");
    auto xf = detail::axis_last(detail::staged_f32<T>(x.data(), x.size()), a);
    const std::size_t count = static_cast<std::size_t>(a.lines) * static_cast<std::size_t>(nfft);
    DeviceArray<ComplexFloat> y(count);
    detail::zkx_check(zkx_hilbert_f32(xf.data(), (int)a.lines, a.samples, nfft, y.data(), nullptr));
    if (a.transpose) {
        DeviceArray<ComplexFloat> t(count);
        detail::zkx_check(zkx_transpose_c64(y.data(), a.shape[1], nfft, t.data(), nullptr));
        y = std::move(t);
    }
    out.shape = a.shape;
    out.shape[a.axis] = nfft;
    if constexpr (std::is_integral_v<T>) {
        out.dtype = HilbertOutputDtype::complex_fp64;
        out.complex_fp32 = DeviceArray<ComplexFloat>();
        DeviceArray<ComplexDouble> wide(count);
        if (count)
            detail::zkx_check(zkx_widen_f32_to_f64(reinterpret_cast<const float*>(y.data()), 2LL * (long long)count,
                                                   reinterpret_cast<double*>(wide.data()), nullptr));
        out.complex_fp64 = std::move(wide);
    } else {
        out.dtype = HilbertOutputDtype::complex_fp32;
        out.complex_fp64 = DeviceArray<ComplexDouble>();
        cuda_utils::synchronize_stream();
        out.complex_fp32 = std::move(y);
    }
}

// CPU references (declared for callers that link the reference's own CPU implementation).
template <typename T>
FirfilterCpuResult firfilter_typed_cpu(const std::vector<T>& b, const std::vector<T>& x,
                                       const FirfilterOptions& options = {}, const std::vector<T>* zi = nullptr);
template <typename T>
UpfirdnCpuResult upfirdn_typed_cpu(const std::vector<T>& h, const std::vector<T>& x, int up, int down,
                                   const UpfirdnOptions& options = {});
template <typename T>
Firfilter2CpuResult firfilter2_typed_cpu(const std::vector<T>& b, const std::vector<T>& x,
                                         const Firfilter2Options& options = {});
template <typename T>
HilbertCpuResult hilbert_typed_cpu(const std::vector<T>& x, const HilbertOptions& options = {});
template <typename T>
ResamplePolyCpuResult resample_poly_typed_cpu(const std::vector<T>& x, int up, int down,
                                              const ResamplePolyOptions& options = {},
                                              const std::vector<T>* coefficients = nullptr);

}  // namespace cusignal
