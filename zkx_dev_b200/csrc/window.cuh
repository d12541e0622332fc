// Window taps evaluated on the device (the reference's RadarWindowKind,
// radartools_typed.h:39-47).
#pragma once

#include <cuda_runtime.h>

#include "../../include/zkx_rd.h"

namespace zkx {

__device__ __forceinline__ float window_value(int kind, const float* explicit_window, int i,
                                              int length)
{
    // Hann/Hamming evaluated in FP64 and rounded once (the reference evaluates the
    // same formulas in FP32, radartools_kernels.cuh:150-160).
    if (kind == ZKX_WINDOW_EXPLICIT_FP32 || kind == ZKX_WINDOW_EXPLICIT_FP64) return explicit_window[i];
    if (kind == ZKX_WINDOW_NONE || length <= 1) return 1.0f;
    const double c = cospi(2.0 * (double)i / (double)(length - 1));
    if (kind == ZKX_WINDOW_HANN) return (float)(0.5 - 0.5 * c);
    return (float)(0.54 - 0.46 * c);
}

}  // namespace zkx
