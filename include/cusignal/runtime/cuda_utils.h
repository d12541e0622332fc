// Host helpers of the cusignal_cpp runtime that callers use around the operators
// (ZKX/cusignal_cpp/include/cusignal/runtime/cuda_utils.h, copy_utils.h): copies on a
// stream and a default-stream synchronisation, plus the device queries and event timer
// (runtime_utils.h) and the 1-D launch helpers (kernel_launch.h) it gathers.
#pragma once

#include <cuda_runtime.h>

#include <cusignal/runtime/cuda_error.h>
#include <cusignal/runtime/device_array.h>
#include <cusignal/runtime/kernel_launch.h>
#include <cusignal/runtime/runtime_utils.h>

#include <cstddef>

namespace cusignal::cuda_utils {

template <typename T>
inline void copy_to_device(T* dst, const T* src, std::size_t count, cudaStream_t stream = nullptr)
{
    if (count) CUDA_CHECK(cudaMemcpyAsync(dst, src, count * sizeof(T), cudaMemcpyHostToDevice, stream));
}

template <typename T>
inline void copy_to_host(T* dst, const T* src, std::size_t count, cudaStream_t stream = nullptr)
{
    if (count) CUDA_CHECK(cudaMemcpyAsync(dst, src, count * sizeof(T), cudaMemcpyDeviceToHost, stream));
}

template <typename T>
inline void copy_device_to_device(T* dst, const T* src, std::size_t count, cudaStream_t stream = nullptr)
{
    if (count) CUDA_CHECK(cudaMemcpyAsync(dst, src, count * sizeof(T), cudaMemcpyDeviceToDevice, stream));
}

inline void synchronize_stream(cudaStream_t stream = nullptr) { CUDA_CHECK(cudaStreamSynchronize(stream)); }

}  // namespace cusignal::cuda_utils
