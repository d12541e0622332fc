// One-dimensional kernel launch helpers of the cusignal_cpp API (the interface of
// ZKX/cusignal_cpp/include/cusignal/runtime/kernel_launch.h:9-56; Task1 step 4 launches
// its power kernel through launch_1d_kernel, ZKX/Task1/pipeline/src/steps/step4/step4.cu:65).
//
// A launch covers `elements` work items with `block_size`-thread blocks (default 256) on
// the given stream (the legacy default stream for launch_1d_kernel) and reports launch
// errors through CUDA_KERNEL_CHECK.  The launch goes through cudaLaunchKernel with every
// argument first converted to the kernel's own parameter type, so these helpers also
// compile in plain C++ translation units (no <<< >>> syntax needed).
#pragma once

#include <cuda_runtime.h>

#include <cusignal/runtime/cuda_error.h>

#include <cstddef>
#include <tuple>
#include <utility>

namespace cusignal::cuda_utils {

template <typename IndexType>
constexpr IndexType div_up(IndexType value, IndexType divisor)
{
    return (value + divisor - 1) / divisor;
}

struct LaunchConfig1D {
    dim3 block;
    dim3 grid;
};

inline LaunchConfig1D make_1d_launch_config(std::size_t elements, unsigned int block_size = 256)
{
    const std::size_t blocks = div_up(elements, static_cast<std::size_t>(block_size));
    return LaunchConfig1D{dim3(block_size), dim3(static_cast<unsigned int>(blocks))};
}

namespace detail {

template <typename... Params, typename Tuple, std::size_t... I>
inline cudaError_t launch_converted(void (*kernel)(Params...), dim3 grid, dim3 block, cudaStream_t stream,
                                    Tuple& converted, std::index_sequence<I...>)
{
    void* argv[sizeof...(Params) + 1] = {static_cast<void*>(&std::get<I>(converted))..., nullptr};
    return cudaLaunchKernel(reinterpret_cast<const void*>(kernel), grid, block, argv, 0, stream);
}

}  // namespace detail

template <typename... Params, typename... Args>
inline void launch_1d_kernel_with_config(void (*kernel)(Params...), std::size_t elements, cudaStream_t stream,
                                         unsigned int block_size, Args&&... args)
{
    static_assert(sizeof...(Params) == sizeof...(Args), "argument count does not match the kernel");
    // zero elements give an empty grid, which the runtime rejects as an invalid
    // configuration (reported like any other launch error)
    const LaunchConfig1D cfg = make_1d_launch_config(elements, block_size);
    std::tuple<std::decay_t<Params>...> converted(std::forward<Args>(args)...);
    const cudaError_t st = detail::launch_converted(kernel, cfg.grid, cfg.block, stream, converted,
                                                    std::index_sequence_for<Params...>{});
    if (st != cudaSuccess) {
        (void)cudaGetLastError();
        throw_cuda_error(st, "cudaLaunchKernel", __FILE__, __LINE__);
    }
    CUDA_KERNEL_CHECK();
}

template <typename... Params, typename... Args>
inline void launch_1d_kernel(void (*kernel)(Params...), std::size_t elements, Args&&... args)
{
    launch_1d_kernel_with_config(kernel, elements, nullptr, 256U, std::forward<Args>(args)...);
}

}  // namespace cusignal::cuda_utils
