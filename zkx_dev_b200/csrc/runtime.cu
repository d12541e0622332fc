// Library runtime: error reporting, per-device initialisation (FP64-generated
// twiddle table) and grow-only per-device scratch buffers.
#include "fft_core.cuh"
#include "zkx_internal.h"

#include <mutex>
#include <string>
#include <vector>

namespace zkx {

namespace {
__device__ float2 g_twiddle[kTwiddleSize];

thread_local std::string g_error;

// exp(-2 pi i j / 65536) evaluated in FP64 and rounded once to FP32.
__global__ void twiddle_init_kernel(float2* table)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= kTwiddleSize) return;
    double s, c;
    sincospi(-2.0 * (double)j / (double)kTwiddleSize, &s, &c);
    table[j] = make_float2((float)c, (float)s);
}

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
bool g_ready[kMaxDevices] = {};
const float2* g_table[kMaxDevices] = {};
struct ScratchEntry {
    void* ptr = nullptr;
    std::size_t bytes = 0;
};
ScratchEntry g_scratch[kMaxDevices][kScratchSlots];
}  // namespace

void set_error(const std::string& msg) { g_error = msg; }

int fail(int code, const std::string& msg)
{
    g_error = msg;
    return code;
}

int cuda_status(cudaError_t e, const char* what)
{
    g_error = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? ZKX_OUT_OF_MEMORY : ZKX_CUDA_RUNTIME_ERROR;
}

bool is_pow2(long long n) { return n > 0 && (n & (n - 1)) == 0; }

int ilog2_host(long long n)
{
    int l = 0;
    while ((1LL << (l + 1)) <= n) ++l;
    return l;
}

int ensure_device_ready()
{
    int dev = 0;
    ZKX_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return fail(ZKX_INTERNAL_ERROR, "device index out of range");
    std::lock_guard<std::mutex> lock(g_mutex);
    if (g_ready[dev]) return ZKX_SUCCESS;
    float2* table = nullptr;
    ZKX_CUDA(cudaGetSymbolAddress(reinterpret_cast<void**>(&table), g_twiddle));
    // Generated on a private stream and waited for, so every later launch on any
    // stream of this device sees the finished table.
    cudaStream_t s;
    ZKX_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    twiddle_init_kernel<<<kTwiddleSize / 256, 256, 0, s>>>(table);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    if (e != cudaSuccess) return cuda_status(e, "twiddle table initialisation");
    g_table[dev] = table;
    g_ready[dev] = true;
    return ZKX_SUCCESS;
}

const float2* twiddle_table()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
    return g_table[dev];
}

int scratch(ScratchSlot slot, std::size_t bytes, void** out)
{
    int dev = 0;
    ZKX_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return fail(ZKX_INTERNAL_ERROR, "device index out of range");
    std::lock_guard<std::mutex> lock(g_mutex);
    ScratchEntry& e = g_scratch[dev][slot];
    if (e.bytes < bytes) {
        if (e.ptr) {
            // The old buffer may still be read by queued work on any stream.
            ZKX_CUDA(cudaDeviceSynchronize());
            ZKX_CUDA(cudaFree(e.ptr));
            e.ptr = nullptr;
            e.bytes = 0;
        }
        ZKX_CUDA(cudaMalloc(&e.ptr, bytes));
        e.bytes = bytes;
    }
    *out = e.ptr;
    return ZKX_SUCCESS;
}

}  // namespace zkx

extern "C" const char* zkx_last_error(void) { return zkx::g_error.c_str(); }
extern "C" const char* zkx_version(void) { return "zkx_rd 0.1.0 (sm_100a)"; }
