// Host helpers of the cusignal_cpp runtime that callers use around the operators
// (ZKX/cusignal_cpp/include/cusignal/runtime/copy_utils.h, runtime_utils.h): copies on a
// stream, a default-stream synchronisation and the device memory counters.
#pragma once

#include <cuda_runtime.h>

#include <cusignal/runtime/cuda_error.h>
#include <cusignal/runtime/device_array.h>

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

struct MemoryInfo {
    std::size_t free_bytes = 0;
    std::size_t total_bytes = 0;
};

inline MemoryInfo current_memory_info()
{
    MemoryInfo m;
    CUDA_CHECK(cudaMemGetInfo(&m.free_bytes, &m.total_bytes));
    return m;
}

}  // namespace cusignal::cuda_utils
