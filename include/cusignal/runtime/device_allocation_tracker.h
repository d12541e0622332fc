// Allocation accounting for device memory owned by this process (the interface of
// ZKX/cusignal_cpp/include/cusignal/runtime/device_allocation_tracker.h:21-87).
//
// tracked_cuda_malloc / tracked_cuda_free wrap cudaMalloc / cudaFree and keep the bytes
// currently live and the high-water mark since the last reset_tracked_device_peak().
// DeviceArray<T> allocates through them, so the figures cover every array the API hands
// out; memory the library allocates for its own workspaces (replica spectra, chirp-z
// buffers, serving blocks) is not counted.  Counting allocation events instead of polling
// cudaMemGetInfo cannot miss short-lived buffers and ignores other processes on the GPU.
// Thread-safe (one mutex); the state is per process, shared by all devices.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <mutex>
#include <unordered_map>

namespace cusignal::cuda_utils {

namespace detail {

struct DeviceAllocationLedger {
    std::mutex lock;
    std::unordered_map<void*, std::size_t> live;
    std::size_t current = 0;
    std::size_t peak = 0;
};

inline DeviceAllocationLedger& device_allocation_ledger()
{
    static DeviceAllocationLedger ledger;
    return ledger;
}

}  // namespace detail

inline cudaError_t tracked_cuda_malloc(void** pointer, std::size_t bytes)
{
    const cudaError_t st = cudaMalloc(pointer, bytes);
    if (st == cudaSuccess && pointer != nullptr && *pointer != nullptr) {
        auto& l = detail::device_allocation_ledger();
        std::lock_guard<std::mutex> g(l.lock);
        l.live[*pointer] = bytes;
        l.current += bytes;
        l.peak = std::max(l.peak, l.current);
    }
    return st;
}

template <typename T>
inline cudaError_t tracked_cuda_malloc(T** pointer, std::size_t bytes)
{
    return tracked_cuda_malloc(reinterpret_cast<void**>(pointer), bytes);
}

inline cudaError_t tracked_cuda_free(void* pointer)
{
    const cudaError_t st = cudaFree(pointer);
    if (st == cudaSuccess && pointer != nullptr) {
        auto& l = detail::device_allocation_ledger();
        std::lock_guard<std::mutex> g(l.lock);
        const auto it = l.live.find(pointer);
        if (it != l.live.end()) {
            l.current -= it->second;
            l.live.erase(it);
        }
    }
    return st;
}

// Restart the high-water mark at the bytes live now.
inline void reset_tracked_device_peak()
{
    auto& l = detail::device_allocation_ledger();
    std::lock_guard<std::mutex> g(l.lock);
    l.peak = l.current;
}

inline std::size_t tracked_device_current_bytes()
{
    auto& l = detail::device_allocation_ledger();
    std::lock_guard<std::mutex> g(l.lock);
    return l.current;
}

inline std::size_t tracked_device_peak_bytes()
{
    auto& l = detail::device_allocation_ledger();
    std::lock_guard<std::mutex> g(l.lock);
    return l.peak;
}

}  // namespace cusignal::cuda_utils
