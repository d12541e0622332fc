// Pulse compression without any device allocation.
//
// zkx_pulse_compression_c64 keeps the replica spectrum in a library-owned scratch
// buffer that it obtains with cudaMalloc the first time (and again whenever a longer
// transform is requested).  Some callers cannot let a library allocate: processing
// loops that must not allocate once they are running (cudaMalloc and cudaFree can
// block and synchronise the device, which breaks a fixed per-CPI time budget), and
// hosts whose device memory is entirely owned and accounted for by another allocator
// or a fixed budget.  For them this file provides one entry point whose scratch is a
// file-scope device array reserved when the library is loaded, so no call allocates.
//
// The array holds the spectrum of the longest supported transform (16384 complex64,
// 128 KiB) on every GPU that loads the library, until the process exits.
#include "fft_core.cuh"
#include "zkx_internal.h"

#include <mutex>
#include <string>

namespace zkx {
namespace {

constexpr int kNoAllocMaxNfft = 1 << kMaxSmemFftLog;  // 16384

// Scratch for the replica spectrum.  Every call rewrites all nfft entries it uses
// before reading them, so nothing has to be cleared between calls; calls that
// overlap on the GPU (different streams, or different host threads) race on it.
static __device__ __align__(256) float2 g_noalloc_spectrum[kNoAllocMaxNfft];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
float2* g_noalloc_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device, looked up once per
// device with that device current (the symbol's host-side name is only a stand-in).
int noalloc_scratch(float2** out)
{
    int dev = 0;
    ZKX_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return fail(ZKX_INTERNAL_ERROR, "device index out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
        float2* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_noalloc_spectrum);
        if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(no-allocation scratch)");
        g_noalloc_ptr[dev] = p;
    }
    *out = g_noalloc_ptr[dev];
    return ZKX_SUCCESS;
}

}  // namespace
}  // namespace zkx

using namespace zkx;

extern "C" int zkx_pulse_compression_c64_noalloc(const void* x, int P, int N, const void* replica,
                                                 int L, int nfft, int normalize, int kind,
                                                 const float* w, void* y, zkx_stream_t stream)
{
    if (nfft == -1) nfft = N;
    if (nfft > kNoAllocMaxNfft)
        return fail(ZKX_INVALID_ARGUMENT,
                    "pulse_compression_noalloc: nfft " + std::to_string(nfft) +
                        " exceeds the no-allocation scratch maximum of 16384");
    const long long in = (long long)P * N, outc = (long long)P * nfft;
    if (P < 1 || N < 1 || nfft < 1 || L < 1 || in > 2147483647LL || outc > 2147483647LL)
        return fail(ZKX_INVALID_SHAPE, "pulse_compression_noalloc shape is invalid");
    const bool is_explicit = kind == ZKX_WINDOW_EXPLICIT_FP32 || kind == ZKX_WINDOW_EXPLICIT_FP64;
    if (kind < ZKX_WINDOW_NONE || kind > ZKX_WINDOW_EXPLICIT_FP64 || is_explicit != (w != nullptr))
        return fail(ZKX_INVALID_ARGUMENT, "pulse_compression_noalloc window is invalid");
    if (!x || !replica || !y) return fail(ZKX_INVALID_ARGUMENT, "pulse_compression_noalloc: null pointer");
    if (!is_pow2(nfft))
        return fail(ZKX_UNSUPPORTED_OPERATION, "pulse_compression_noalloc: nfft must be a power of two");
    ZKX_TRY(ensure_device_ready());
    float2* spec = nullptr;
    ZKX_TRY(noalloc_scratch(&spec));
    ZKX_TRY(launch_replica_spectrum(static_cast<const float2*>(replica), L, nfft, normalize, kind, w,
                                    spec, stream));
    return launch_pulse_compression(static_cast<const float2*>(x), P, N, nfft, spec,
                                    static_cast<float2*>(y), stream);
}
