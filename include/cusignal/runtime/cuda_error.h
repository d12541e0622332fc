// CUDA_CHECK: throws ProjectError{CUDA_RUNTIME_ERROR or OUT_OF_MEMORY} on a failing CUDA
// runtime call; CUDA_KERNEL_CHECK(): the same for the error a kernel launch left behind
// (the contract of ZKX/cusignal_cpp/include/cusignal/runtime/cuda_error.h:5-56).
#pragma once

#include <cuda_runtime.h>

#include <cusignal/runtime/errors.h>

#include <string>

namespace cusignal::cuda_utils {

[[noreturn]] inline void throw_cuda_error(cudaError_t status, const char* expr, const char* file, int line)
{
    const ErrorCode code = status == cudaErrorMemoryAllocation ? ErrorCode::OUT_OF_MEMORY
                                                               : ErrorCode::CUDA_RUNTIME_ERROR;
    throw ProjectError(code, std::string(expr) + " failed at " + file + ":" + std::to_string(line) +
                                 ": " + cudaGetErrorString(status));
}

// Launch-time error of the last kernel launch on this thread (bad configuration, no
// device image), as CUDA_CHECK reports it; asynchronous faults surface at the next
// synchronising call instead.
inline void check_last_kernel_error(const char* file, int line)
{
    const cudaError_t status = cudaGetLastError();
    if (status != cudaSuccess) throw_cuda_error(status, "kernel launch", file, line);
}

}  // namespace cusignal::cuda_utils

#define CUDA_KERNEL_CHECK() ::cusignal::cuda_utils::check_last_kernel_error(__FILE__, __LINE__)

#define CUDA_CHECK(call)                                                                     \
    do {                                                                                     \
        const cudaError_t cusignal_status_ = (call);                                         \
        if (cusignal_status_ != cudaSuccess)                                                 \
            ::cusignal::cuda_utils::throw_cuda_error(cusignal_status_, #call, __FILE__, __LINE__); \
    } while (0)
