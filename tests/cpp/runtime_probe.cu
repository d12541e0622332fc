// Exercises the runtime headers of the C++ API (include/cusignal/runtime/...): the error
// model, the FP64 storage boundaries, the allocation tracker, the 1-D launch helpers and
// the event timer.  `runtime_probe host` runs what needs no GPU; `runtime_probe device`
// the rest.  Prints one line per check and exits non-zero on the first failure.
#include <cusignal/runtime/cuda_utils.h>
#include <cusignal/runtime/device_allocation_tracker.h>
#include <cusignal/runtime/device_array.h>
#include <cusignal/runtime/errors.h>
#include <cusignal/runtime/host_output_finalize.h>
#include <cusignal/runtime/kernel_launch.h>
#include <cusignal/runtime/runtime_utils.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <vector>

namespace {

int g_fail = 0;

void check(bool ok, const char* what)
{
    std::printf("%s %s\n", ok ? "ok" : "FAIL", what);
    if (!ok) g_fail = 1;
}

__global__ void scale_kernel(const float* in, float* out, int count, float factor)
{
    const int i = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
    if (i < count) out[i] = in[i] * factor;
}

void host_checks()
{
    using namespace cusignal;
    check(parse_error_code("OUT_OF_MEMORY") == ErrorCode::OUT_OF_MEMORY, "parse_error_code");
    check(std::strcmp(error_code_name(ErrorCode::UPSTREAM_STEP_FAILED), "UPSTREAM_STEP_FAILED") == 0,
          "error_code_name");
    check(error_code_value(ErrorCode::CONFIG_ERROR) == 1005, "error_code_value");
    try {
        throw_error(ErrorCode::IO_ERROR, "", BackendError{"7", "E", "m"}, false);
    } catch (const ProjectError& e) {
        check(e.detail().code == ErrorCode::IO_ERROR && e.code() == ErrorCode::IO_ERROR &&
                  e.detail().backend.code == "7" && !e.detail().safe_exit && std::strlen(e.what()) > 0,
              "throw_error carries the Error");
    }
    try {
        (void)parse_error_code("NOT_A_CODE");
        check(false, "unknown code name rejected");
    } catch (const ProjectError& e) {
        check(e.code() == ErrorCode::CONFIG_ERROR, "unknown code name rejected");
    }

    using namespace cusignal::cuda_utils;
    const std::vector<float> f{1.5F, -0.25F, std::numeric_limits<float>::infinity()};
    const auto d = finalize_fp64_on_host(f);
    check(d.size() == 3 && d[0] == 1.5 && d[1] == -0.25 && std::isinf(d[2]), "finalize_fp64_on_host");
    const std::vector<ComplexFloat> cf{{1.0F, 2.0F}, {-3.0F, 0.5F}};
    const auto cd = finalize_complex_fp64_on_host(cf);
    check(cd[1].re == -3.0 && cd[1].im == 0.5, "finalize_complex_fp64_on_host");
    const auto back = narrow_complex_fp64_to_fp32_on_host(cd);
    check(back[0].re == 1.0F && back[1].im == 0.5F, "narrow_complex_fp64_to_fp32_on_host");
    check(std::isnan(narrow_fp64_value_to_fp32_on_host(std::nan(""))) &&
              std::isinf(narrow_fp64_value_to_fp32_on_host(-INFINITY)),
          "NaN and infinities keep their class");
    try {
        (void)narrow_fp64_to_fp32_on_host({1.0, 1e300});
        check(false, "finite overflow rejected");
    } catch (const std::overflow_error&) {
        check(true, "finite overflow rejected");
    }
    const auto cfg = make_1d_launch_config(1000, 256);
    check(cfg.grid.x == 4 && cfg.block.x == 256 && div_up(1000, 256) == 4, "make_1d_launch_config");
}

void device_checks()
{
    using namespace cusignal;
    using namespace cusignal::cuda_utils;
    const auto info = current_device_info();
    check(device_count() >= 1 && info.properties.major >= 10, "current_device_info");
    const auto mem = current_memory_info();
    check(mem.total_bytes > 0 && mem.free_bytes <= mem.total_bytes, "current_memory_info");

    reset_tracked_device_peak();
    const std::size_t before = tracked_device_current_bytes();
    const int count = 100000;
    std::vector<float> host(count);
    for (int i = 0; i < count; ++i) host[i] = static_cast<float>(i % 97);
    {
        auto in = DeviceArray<float>::from_host(host);
        DeviceArray<float> out(count);
        check(tracked_device_current_bytes() == before + 2 * count * sizeof(float), "tracked bytes live");
        EventTimer timer;
        timer.record_start();
        // size_t element count and double factor converted to the kernel's int and float
        launch_1d_kernel(scale_kernel, static_cast<std::size_t>(count), in.data(), out.data(),
                         static_cast<std::size_t>(count), 2.0);
        timer.record_stop();
        const float ms = timer.elapsed_ms();
        check(ms >= 0.0F, "EventTimer elapsed_ms");
        const auto got = out.to_host();
        bool same = true;
        for (int i = 0; i < count; ++i) same = same && got[i] == 2.0F * host[i];
        check(same, "launch_1d_kernel converts arguments to the kernel's types");
        launch_1d_kernel_with_config(scale_kernel, static_cast<std::size_t>(count), nullptr, 128U,
                                     out.data(), out.data(), count, 0.5F);
        check(out.to_host()[96] == host[96], "launch_1d_kernel_with_config");
        const auto wide = finalize_fp64_device_storage(out);
        check(wide.to_host()[50] == static_cast<double>(host[50]), "finalize_fp64_device_storage");
    }
    check(tracked_device_current_bytes() == before, "tracked bytes released");
    check(tracked_device_peak_bytes() >= before + 2 * count * sizeof(float) + count * sizeof(double),
          "tracked peak");
    try {
        launch_1d_kernel(scale_kernel, 0, static_cast<const float*>(nullptr), static_cast<float*>(nullptr), 0,
                         1.0F);
        check(false, "empty launch reported");
    } catch (const ProjectError& e) {
        check(e.code() == ErrorCode::CUDA_RUNTIME_ERROR, "empty launch reported");
    }
    check(cudaGetLastError() == cudaSuccess, "no sticky error left");
}

}  // namespace

int main(int argc, char** argv)
{
    const bool device = argc > 1 && std::strcmp(argv[1], "device") == 0;
    try {
        if (device) device_checks();
        else host_checks();
    } catch (const std::exception& e) {
        std::printf("FAIL exception: %s\n", e.what());
        return 1;
    }
    return g_fail;
}
