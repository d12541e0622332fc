// Device queries and a CUDA-event stopwatch for callers of the cusignal_cpp API (the
// interface of ZKX/cusignal_cpp/include/cusignal/runtime/runtime_utils.h:7-93, which
// Task1 includes through task1_common.h and uses as cuda_utils::EventTimer).
//
// EventTimer brackets work on one stream with two events and reports the time between
// them in milliseconds; elapsed_ms() waits for the stop event.  Every CUDA failure
// throws ProjectError through CUDA_CHECK.
#pragma once

#include <cuda_runtime.h>

#include <cusignal/runtime/cuda_error.h>

#include <cstddef>

namespace cusignal::cuda_utils {

struct DeviceInfo {
    int ordinal = 0;
    cudaDeviceProp properties{};
};

struct MemoryInfo {
    std::size_t free_bytes = 0;
    std::size_t total_bytes = 0;
};

inline DeviceInfo current_device_info()
{
    DeviceInfo info;
    CUDA_CHECK(cudaGetDevice(&info.ordinal));
    CUDA_CHECK(cudaGetDeviceProperties(&info.properties, info.ordinal));
    return info;
}

inline int device_count()
{
    int n = 0;
    CUDA_CHECK(cudaGetDeviceCount(&n));
    return n;
}

inline MemoryInfo current_memory_info()
{
    MemoryInfo info;
    CUDA_CHECK(cudaMemGetInfo(&info.free_bytes, &info.total_bytes));
    return info;
}

class EventTimer {
public:
    EventTimer()
    {
        CUDA_CHECK(cudaEventCreate(&events_[0]));
        const cudaError_t st = cudaEventCreate(&events_[1]);
        if (st != cudaSuccess) {
            (void)cudaEventDestroy(events_[0]);
            events_[0] = nullptr;
            CUDA_CHECK(st);
        }
    }
    ~EventTimer() noexcept
    {
        for (cudaEvent_t e : events_)
            if (e) (void)cudaEventDestroy(e);
    }
    EventTimer(const EventTimer&) = delete;
    EventTimer& operator=(const EventTimer&) = delete;
    EventTimer(EventTimer&&) = delete;
    EventTimer& operator=(EventTimer&&) = delete;

    void record_start(cudaStream_t stream = nullptr) { CUDA_CHECK(cudaEventRecord(events_[0], stream)); }
    void record_stop(cudaStream_t stream = nullptr) { CUDA_CHECK(cudaEventRecord(events_[1], stream)); }

    // Milliseconds between the two recorded events; blocks until the stop event completes.
    float elapsed_ms()
    {
        CUDA_CHECK(cudaEventSynchronize(events_[1]));
        float ms = 0.0F;
        CUDA_CHECK(cudaEventElapsedTime(&ms, events_[0], events_[1]));
        return ms;
    }

private:
    cudaEvent_t events_[2] = {nullptr, nullptr};
};

}  // namespace cusignal::cuda_utils
