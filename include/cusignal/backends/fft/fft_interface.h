// Complex types and the batched device FFT of the cusignal_cpp FFT backend
// (ZKX/cusignal_cpp/include/cusignal/backends/fft/fft_interface.h:104-117, 499-536):
// forward transforms are unnormalised, inverse transforms scale by 1/N.  Lengths are
// powers of two up to 65536 and any other length up to 32768 (chirp-z on power-of-two
// FFTs, like the reference backend); the device calls run the B200 shared-memory FFT on
// the legacy default stream.
#pragma once

#include <cusignal/detail/zkx_call.h>
#include <cusignal/runtime/device_array.h>

#include <cstddef>
#include <stdexcept>

typedef struct {
    float re;
    float im;
} ComplexFloat;

typedef struct {
    double re;
    double im;
} ComplexDouble;

namespace cusignal {

class FFTInterface {
public:
    struct BatchOnly {};

    explicit FFTInterface(int n) : n_(n) { validate(); }
    FFTInterface(int n, BatchOnly) : n_(n) { validate(); }
    FFTInterface(const FFTInterface&) = delete;
    FFTInterface& operator=(const FFTInterface&) = delete;

    void fft_device(const DeviceArray<ComplexFloat>& in, DeviceArray<ComplexFloat>& out)
    {
        fft_batch_device(in, out, 1);
    }
    void ifft_device(const DeviceArray<ComplexFloat>& in, DeviceArray<ComplexFloat>& out)
    {
        ifft_batch_device(in, out, 1);
    }
    void fft_device(const ComplexFloat* in, ComplexFloat* out, std::size_t count)
    {
        fft_batch_device(in, out, 1, count);
    }
    void ifft_device(const ComplexFloat* in, ComplexFloat* out, std::size_t count)
    {
        ifft_batch_device(in, out, 1, count);
    }
    void fft_inplace_device(DeviceArray<ComplexFloat>& data)
    {
        run(data.data(), data.data(), static_cast<int>(data.size() / n_), data.size(), false);
    }
    void ifft_inplace_device(DeviceArray<ComplexFloat>& data)
    {
        run(data.data(), data.data(), static_cast<int>(data.size() / n_), data.size(), true);
    }
    void fft_batch_device(const DeviceArray<ComplexFloat>& in, DeviceArray<ComplexFloat>& out, int batch)
    {
        check_sizes(in.size(), out.size(), batch);
        run(in.data(), out.data(), batch, in.size(), false);
    }
    void ifft_batch_device(const DeviceArray<ComplexFloat>& in, DeviceArray<ComplexFloat>& out, int batch)
    {
        check_sizes(in.size(), out.size(), batch);
        run(in.data(), out.data(), batch, in.size(), true);
    }
    void fft_batch_device(const ComplexFloat* in, ComplexFloat* out, int batch, std::size_t count)
    {
        run(in, out, batch, count, false);
    }
    void ifft_batch_device(const ComplexFloat* in, ComplexFloat* out, int batch, std::size_t count)
    {
        run(in, out, batch, count, true);
    }

private:
    void validate() const
    {
        if (n_ < 1) throw std::invalid_argument("FFT length must be positive");
    }
    void check_sizes(std::size_t in, std::size_t out, int batch) const
    {
        if (batch < 1 || in < static_cast<std::size_t>(batch) * n_ || out < static_cast<std::size_t>(batch) * n_)
            throw std::invalid_argument("FFT batch size mismatch");
    }
    void run(const ComplexFloat* in, ComplexFloat* out, int batch, std::size_t count, bool inverse) const
    {
        if (batch < 1 || count < static_cast<std::size_t>(batch) * n_)
            throw std::invalid_argument("FFT batch size mismatch");
        detail::zkx_check(zkx_fft_c2c_c64(in, batch, n_, inverse ? 1 : 0, out, nullptr));
    }
    int n_;
};

}  // namespace cusignal
