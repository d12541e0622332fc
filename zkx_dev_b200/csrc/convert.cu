// Dtype staging used by the C++ operator shims: business dtypes (FP16 and signed
// integers) to the FP32 compute type, and exact FP32 -> FP64 widening for the
// operators whose public result storage is FP64.  Grid-stride loops over `count`
// scalars (complex data count their real and imaginary parts).
#include <cuda_fp16.h>

#include "zkx_internal.h"

namespace zkx {
namespace {

template <typename T>
__device__ __forceinline__ float to_f32(T v) { return static_cast<float>(v); }
template <>
__device__ __forceinline__ float to_f32<__half>(__half v) { return __half2float(v); }

template <typename T>
__global__ void convert_kernel(const T* __restrict__ src, long long count, float* __restrict__ dst)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x)
        dst[i] = to_f32(src[i]);
}

__global__ void widen_kernel(const float* __restrict__ src, long long count, double* __restrict__ dst)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x)
        dst[i] = static_cast<double>(src[i]);
}

unsigned grid_for(long long count)
{
    const long long blocks = (count + 255) / 256;
    return (unsigned)(blocks < 148 * 32 ? (blocks > 0 ? blocks : 1) : 148 * 32);
}

}  // namespace
}  // namespace zkx

using namespace zkx;

extern "C" int zkx_convert_to_f32(const void* src, int dtype, long long count, float* dst,
                                  zkx_stream_t stream)
{
    if (count < 0) return fail(ZKX_INVALID_SHAPE, "convert: negative count");
    if (count == 0) return ZKX_SUCCESS;
    if (!src || !dst) return fail(ZKX_INVALID_ARGUMENT, "convert: null pointer");
    const unsigned g = grid_for(count);
    switch (dtype) {
    case ZKX_DTYPE_F32:
        ZKX_CUDA(cudaMemcpyAsync(dst, src, (size_t)count * sizeof(float), cudaMemcpyDeviceToDevice, stream));
        return ZKX_SUCCESS;
    case ZKX_DTYPE_F16: convert_kernel<__half><<<g, 256, 0, stream>>>(static_cast<const __half*>(src), count, dst); break;
    case ZKX_DTYPE_I32: convert_kernel<int32_t><<<g, 256, 0, stream>>>(static_cast<const int32_t*>(src), count, dst); break;
    case ZKX_DTYPE_I16: convert_kernel<int16_t><<<g, 256, 0, stream>>>(static_cast<const int16_t*>(src), count, dst); break;
    case ZKX_DTYPE_I8: convert_kernel<int8_t><<<g, 256, 0, stream>>>(static_cast<const int8_t*>(src), count, dst); break;
    default: return fail(ZKX_INVALID_ARGUMENT, "convert: unknown dtype");
    }
    ZKX_LAUNCHED("convert_kernel");
    return ZKX_SUCCESS;
}

extern "C" int zkx_widen_f32_to_f64(const float* src, long long count, double* dst, zkx_stream_t stream)
{
    if (count < 0) return fail(ZKX_INVALID_SHAPE, "widen: negative count");
    if (count == 0) return ZKX_SUCCESS;
    if (!src || !dst) return fail(ZKX_INVALID_ARGUMENT, "widen: null pointer");
    widen_kernel<<<grid_for(count), 256, 0, stream>>>(src, count, dst);
    ZKX_LAUNCHED("widen_kernel");
    return ZKX_SUCCESS;
}

namespace zkx {
namespace {

// Integral CA-CFAR decision (radartools_kernels.cuh:24-37): NaN thresholds never detect,
// infinities detect only when negative, thresholds outside the dtype's range saturate,
// otherwise x > floor(threshold) in the integer domain.
template <typename T>
__global__ void detect_int_kernel(const T* __restrict__ x, const float* __restrict__ thr, long long count,
                                  float lo, float hi, uint8_t* __restrict__ det)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x) {
        const float t = thr[i];
        bool hit;
        if (isnan(t)) hit = false;
        else if (isinf(t)) hit = t < 0.0f;
        else if (t < lo) hit = true;
        else if (t >= hi) hit = false;
        else hit = (long long)x[i] > (long long)floorf(t);
        det[i] = hit ? 1 : 0;
    }
}

// 32 x 32 tiles through shared memory: coalesced reads and writes.
template <class T>
__global__ void transpose_kernel(const T* __restrict__ src, int rows, int cols, T* __restrict__ dst)
{
    __shared__ T tile[32][33];
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int r = r0 + i, c = c0 + threadIdx.x;
        if (r < rows && c < cols) tile[i][threadIdx.x] = src[(size_t)r * cols + c];
    }
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int c = c0 + i, r = r0 + threadIdx.x;
        if (r < rows && c < cols) dst[(size_t)c * rows + r] = tile[threadIdx.x][i];
    }
}

}  // namespace
}  // namespace zkx

extern "C" int zkx_cfar_detect_int(const void* x, int dtype, const float* threshold, long long count,
                                   uint8_t* detections, zkx_stream_t stream)
{
    if (count < 0) return fail(ZKX_INVALID_SHAPE, "cfar_detect_int: negative count");
    if (count == 0) return ZKX_SUCCESS;
    if (!x || !threshold || !detections) return fail(ZKX_INVALID_ARGUMENT, "cfar_detect_int: null pointer");
    const unsigned g = grid_for(count);
    switch (dtype) {
    case ZKX_DTYPE_I32:
        detect_int_kernel<int32_t><<<g, 256, 0, stream>>>(static_cast<const int32_t*>(x), threshold, count,
                                                          -2147483648.0f, 2147483647.0f, detections);
        break;
    case ZKX_DTYPE_I16:
        detect_int_kernel<int16_t><<<g, 256, 0, stream>>>(static_cast<const int16_t*>(x), threshold, count,
                                                          -32768.0f, 32767.0f, detections);
        break;
    case ZKX_DTYPE_I8:
        detect_int_kernel<int8_t><<<g, 256, 0, stream>>>(static_cast<const int8_t*>(x), threshold, count,
                                                         -128.0f, 127.0f, detections);
        break;
    default: return fail(ZKX_INVALID_ARGUMENT, "cfar_detect_int: dtype must be an integer type");
    }
    ZKX_LAUNCHED("detect_int_kernel");
    return ZKX_SUCCESS;
}

namespace {
template <class T>
int transpose(const T* src, int rows, int cols, T* dst, cudaStream_t stream)
{
    if (rows < 0 || cols < 0) return fail(ZKX_INVALID_SHAPE, "transpose: negative extent");
    if ((long long)rows * cols == 0) return ZKX_SUCCESS;
    if (!src || !dst || src == dst) return fail(ZKX_INVALID_ARGUMENT, "transpose: null or aliased pointer");
    if ((rows + 31) / 32 > 65535) return fail(ZKX_UNSUPPORTED_OPERATION, "transpose: too many rows");
    dim3 grid((cols + 31) / 32, (rows + 31) / 32);
    transpose_kernel<T><<<grid, dim3(32, 8), 0, stream>>>(src, rows, cols, dst);
    ZKX_LAUNCHED("transpose_kernel");
    return ZKX_SUCCESS;
}
}  // namespace

extern "C" int zkx_transpose_f32(const float* src, int rows, int cols, float* dst, zkx_stream_t stream)
{
    return transpose(src, rows, cols, dst, stream);
}

extern "C" int zkx_transpose_c64(const void* src, int rows, int cols, void* dst, zkx_stream_t stream)
{
    return transpose(static_cast<const float2*>(src), rows, cols, static_cast<float2*>(dst), stream);
}
