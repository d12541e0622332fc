// Library runtime: error reporting, per-device initialisation (FP64-generated
// twiddle table) and grow-only per-device scratch buffers.
#include "fft_core.cuh"
#include "tma.cuh"
#include "zkx_internal.h"

#include <cudaTypedefs.h>

#include <mutex>
#include <string>
#include <vector>

namespace zkx {

namespace {
__device__ float2 g_twiddle[kTwiddleSize];
__device__ int g_kernel_error;

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
int* g_error_word[kMaxDevices] = {};
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::once_flag g_encode_once;
struct ScratchEntry {
    void* ptr = nullptr;
    std::size_t bytes = 0;
};
ScratchEntry g_scratch[kMaxDevices][kScratchSlots];
cudaMemPool_t g_pool[kMaxDevices] = {};
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
    int* word = nullptr;
    ZKX_CUDA(cudaGetSymbolAddress(reinterpret_cast<void**>(&word), g_kernel_error));
    ZKX_CUDA(cudaMemset(word, 0, sizeof(int)));
    g_error_word[dev] = word;
    g_table[dev] = table;
    g_ready[dev] = true;
    return ZKX_SUCCESS;
}

int* kernel_error_word()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
    return g_error_word[dev];
}

bool encode_tensor_map_2d_f32(CUtensorMap* map, const void* base, uint64_t inner, uint64_t outer,
                              uint64_t row_pitch_bytes, uint32_t box_inner, uint32_t box_outer)
{
    std::call_once(g_encode_once, [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    });
    if (!g_encode) return false;
    const cuuint64_t dims[2] = {inner, outer};
    const cuuint64_t strides[1] = {row_pitch_bytes};
    const cuuint32_t box[2] = {box_inner, box_outer};
    const cuuint32_t estr[2] = {1, 1};
    return g_encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void*>(base), dims, strides,
                    box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
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

int stream_workspace(std::size_t bytes, cudaStream_t stream, void** out)
{
    int dev = 0;
    ZKX_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return fail(ZKX_INTERNAL_ERROR, "device index out of range");
    cudaMemPool_t pool;
    {
        std::lock_guard<std::mutex> lock(g_mutex);
        if (!g_pool[dev]) {
            cudaMemPoolProps props{};
            props.allocType = cudaMemAllocationTypePinned;
            props.location.type = cudaMemLocationTypeDevice;
            props.location.id = dev;
            ZKX_CUDA(cudaMemPoolCreate(&g_pool[dev], &props));
            std::uint64_t keep = ~std::uint64_t(0);  // keep freed blocks for the next launch
            ZKX_CUDA(cudaMemPoolSetAttribute(g_pool[dev], cudaMemPoolAttrReleaseThreshold, &keep));
        }
        pool = g_pool[dev];
    }
    ZKX_CUDA(cudaMallocFromPoolAsync(out, bytes, pool, stream));
    return ZKX_SUCCESS;
}

}  // namespace zkx

namespace zkx {
namespace {

// The failure path of every bulk-copy wait, exercised on purpose: thread 0 arms the
// barrier for 16 bytes that no copy will deliver (none is issued, so nothing is in flight
// when the CTA leaves), every thread waits with the bounded wait the kernels use, the CTA
// agrees on the timeout and records it in the error word exactly as they do.
__global__ void wait_timeout_selftest_kernel(long long limit, int* err)
{
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        mbar_arrive_expect_tx(&bar, 16);
    }
    __syncthreads();
    const bool ok = mbar_wait_bounded(&bar, 0, limit);
    if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0) atomicCAS(err, 0, (int)kKernelTmaTimeout);
        return;
    }
}

}  // namespace
}  // namespace zkx

extern "C" int zkx_selftest_wait_timeout(long long limit_clocks, zkx_stream_t stream)
{
    using namespace zkx;
    if (limit_clocks < 1000 || limit_clocks > (1LL << 31))
        return fail(ZKX_INVALID_ARGUMENT, "selftest_wait_timeout: limit must be 1000 .. 2^31 clocks");
    ZKX_TRY(ensure_device_ready());
    wait_timeout_selftest_kernel<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>(limit_clocks,
                                                                                 kernel_error_word());
    ZKX_LAUNCHED("wait_timeout_selftest_kernel");
    return ZKX_SUCCESS;
}

extern "C" const char* zkx_last_error(void) { return zkx::g_error.c_str(); }

extern "C" int zkx_kernel_status(int clear, int* code)
{
    using namespace zkx;
    if (!code) return fail(ZKX_INVALID_ARGUMENT, "kernel_status: null pointer");
    ZKX_TRY(ensure_device_ready());
    int* word = kernel_error_word();
    ZKX_CUDA(cudaDeviceSynchronize());
    ZKX_CUDA(cudaMemcpy(code, word, sizeof(int), cudaMemcpyDeviceToHost));
    if (clear) ZKX_CUDA(cudaMemset(word, 0, sizeof(int)));
    return ZKX_SUCCESS;
}
extern "C" const char* zkx_version(void) { return "zkx_rd 0.1.0 (sm_100a)"; }
