// DeviceArray<T>: move-only owner of a cudaMalloc'd array with explicit host transfers,
// the container of the cusignal_cpp API (ZKX/cusignal_cpp/include/cusignal/runtime/
// device_array.h:19-121).  from_host/to_host copy on the legacy default stream and wait.
// Allocations go through the tracked allocator (device_allocation_tracker.h), so
// tracked_device_current_bytes / tracked_device_peak_bytes cover every array.
#pragma once

#include <cuda_runtime.h>

#include <cusignal/runtime/cuda_error.h>
#include <cusignal/runtime/device_allocation_tracker.h>

#include <cstddef>
#include <vector>

namespace cusignal {

template <typename T>
class DeviceArray {
public:
    DeviceArray() = default;
    explicit DeviceArray(std::size_t count) { allocate(count); }
    ~DeviceArray() noexcept { release(); }
    DeviceArray(const DeviceArray&) = delete;
    DeviceArray& operator=(const DeviceArray&) = delete;
    DeviceArray(DeviceArray&& o) noexcept : data_(o.data_), size_(o.size_)
    {
        o.data_ = nullptr;
        o.size_ = 0;
    }
    DeviceArray& operator=(DeviceArray&& o) noexcept
    {
        if (this != &o) {
            release();
            data_ = o.data_;
            size_ = o.size_;
            o.data_ = nullptr;
            o.size_ = 0;
        }
        return *this;
    }

    static DeviceArray from_host(const std::vector<T>& host)
    {
        DeviceArray out(host.size());
        if (!host.empty()) {
            CUDA_CHECK(cudaMemcpyAsync(out.data_, host.data(), host.size() * sizeof(T),
                                       cudaMemcpyHostToDevice, nullptr));
            CUDA_CHECK(cudaStreamSynchronize(nullptr));
        }
        return out;
    }

    std::vector<T> to_host() const
    {
        std::vector<T> host(size_);
        if (size_ != 0) {
            CUDA_CHECK(cudaMemcpyAsync(host.data(), data_, size_ * sizeof(T), cudaMemcpyDeviceToHost,
                                       nullptr));
            CUDA_CHECK(cudaStreamSynchronize(nullptr));
        }
        return host;
    }

    void reset()
    {
        if (data_) {
            const cudaError_t st = cuda_utils::tracked_cuda_free(data_);
            data_ = nullptr;
            size_ = 0;
            CUDA_CHECK(st);
        }
    }
    void reset(std::size_t count) { allocate(count); }

    [[nodiscard]] std::size_t size() const noexcept { return size_; }
    [[nodiscard]] bool empty() const noexcept { return size_ == 0; }
    [[nodiscard]] T* data() noexcept { return data_; }
    [[nodiscard]] const T* data() const noexcept { return data_; }

private:
    void allocate(std::size_t count)
    {
        reset();
        if (count == 0) return;
        CUDA_CHECK(cuda_utils::tracked_cuda_malloc(&data_, count * sizeof(T)));
        size_ = count;
    }
    void release() noexcept
    {
        if (data_) {
            (void)cuda_utils::tracked_cuda_free(data_);
            data_ = nullptr;
            size_ = 0;
        }
    }

    T* data_ = nullptr;
    std::size_t size_ = 0;
};

}  // namespace cusignal
