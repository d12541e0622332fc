// Where the pulses of a range-compression launch come from: one contiguous
// [pulses, samples] array, or a table of per-CPI arrays (a batch of CPIs that live in
// separate buffers, read in place instead of being gathered first).  Both are passed
// to the kernels by value.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace zkx {

constexpr int kMaxRowTable = 64;  // CPIs per table launch (520-byte kernel parameter)

struct RowsContiguous {
    const float2* base;
    int samples;
    __host__ __device__ __forceinline__ const float2* row(int pulse) const
    {
        return base + (size_t)pulse * samples;
    }
};

struct RowsTable {
    const float2* cpi[kMaxRowTable];
    int pulses;  // pulses per CPI
    int samples;
    __host__ __device__ __forceinline__ const float2* row(int pulse) const
    {
        const int c = pulse / pulses;
        return cpi[c] + (size_t)(pulse - c * pulses) * samples;
    }
};

}  // namespace zkx
