// FP32 <-> FP64 storage boundaries of the cusignal_cpp API (the interface of
// ZKX/cusignal_cpp/include/cusignal/runtime/host_output_finalize.h:12-118; Task1 narrows
// FP64 pulse-compression results through narrow_complex_fp64_to_fp32_on_host,
// ZKX/Task1/pipeline/src/task1_common.cu:21-48).
//
// The operators compute in FP32 and, where the reference's contract says FP64 storage,
// widen the FP32 result exactly.  finalize_* widen on the host or on the device
// (libzkx_rd's zkx_widen_f32_to_f64 kernel; exact, no FP64 arithmetic).  narrow_* bring
// FP64 storage back to FP32 on the host: NaN and infinities keep their class, a finite
// value outside the FP32 range throws std::overflow_error instead of turning into an
// infinity.
#pragma once

#include <zkx_rd.h>

#include <cusignal/backends/fft/fft_interface.h>
#include <cusignal/detail/zkx_call.h>
#include <cusignal/runtime/device_array.h>

#include <cmath>
#include <cstddef>
#include <limits>
#include <stdexcept>
#include <vector>

namespace cusignal::cuda_utils {

inline std::vector<double> finalize_fp64_on_host(const std::vector<float>& computed)
{
    return std::vector<double>(computed.begin(), computed.end());
}

inline std::vector<ComplexDouble> finalize_complex_fp64_on_host(const std::vector<ComplexFloat>& computed)
{
    std::vector<ComplexDouble> out(computed.size());
    for (std::size_t i = 0; i < computed.size(); ++i) out[i] = {computed[i].re, computed[i].im};
    return out;
}

inline DeviceArray<double> finalize_fp64_device_storage(const DeviceArray<float>& computed)
{
    DeviceArray<double> out(computed.size());
    if (!computed.empty())
        cusignal::detail::zkx_check(zkx_widen_f32_to_f64(computed.data(), static_cast<long long>(computed.size()),
                                                         out.data(), nullptr));
    return out;
}

inline DeviceArray<ComplexDouble> finalize_complex_fp64_device_storage(const DeviceArray<ComplexFloat>& computed)
{
    static_assert(sizeof(ComplexDouble) == 2 * sizeof(double), "interleaved complex storage");
    DeviceArray<ComplexDouble> out(computed.size());
    if (!computed.empty())
        cusignal::detail::zkx_check(zkx_widen_f32_to_f64(reinterpret_cast<const float*>(computed.data()),
                                                         2LL * static_cast<long long>(computed.size()),
                                                         reinterpret_cast<double*>(out.data()), nullptr));
    return out;
}

inline float narrow_fp64_value_to_fp32_on_host(double value)
{
    if (std::isfinite(value) && std::fabs(value) > static_cast<double>(std::numeric_limits<float>::max()))
        throw std::overflow_error("FP64-to-FP32 host boundary: finite value outside the FP32 range");
    return static_cast<float>(value);
}

inline std::vector<float> narrow_fp64_to_fp32_on_host(const std::vector<double>& storage)
{
    std::vector<float> out(storage.size());
    for (std::size_t i = 0; i < storage.size(); ++i) out[i] = narrow_fp64_value_to_fp32_on_host(storage[i]);
    return out;
}

inline std::vector<ComplexFloat> narrow_complex_fp64_to_fp32_on_host(const std::vector<ComplexDouble>& storage)
{
    std::vector<ComplexFloat> out(storage.size());
    for (std::size_t i = 0; i < storage.size(); ++i)
        out[i] = {narrow_fp64_value_to_fp32_on_host(storage[i].re), narrow_fp64_value_to_fp32_on_host(storage[i].im)};
    return out;
}

inline DeviceArray<float> narrow_fp64_device_storage_to_fp32_on_host(const DeviceArray<double>& storage)
{
    return DeviceArray<float>::from_host(narrow_fp64_to_fp32_on_host(storage.to_host()));
}

inline DeviceArray<ComplexFloat> narrow_complex_fp64_device_storage_to_fp32_on_host(
    const DeviceArray<ComplexDouble>& storage)
{
    return DeviceArray<ComplexFloat>::from_host(narrow_complex_fp64_to_fp32_on_host(storage.to_host()));
}

}  // namespace cusignal::cuda_utils
