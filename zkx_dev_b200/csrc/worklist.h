// Work-list execution of the range-Doppler chain over CPIs of mixed shapes: the parameter
// blocks of the three stage kernels and their launchers.  A stage is one launch over every
// (CPI, tile) entry of up to kWlGroups shape groups (a group = the CPIs of one plan) per
// resource class: compression and Doppler lengths with up to 16 values per thread (class
// 0) and with 32 (class 1) run in separate launches, each kernel sized for its own lengths.
// A CTA finds its group from the groups' first entries, then runs that group's code path
// (a switch over the transform length inside the kernel).  The per-group constants, the
// bulk-copy tensor maps included, travel in the kernel's parameter block.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace zkx {

constexpr int kWlGroups = 24;               // shape groups per launch
constexpr int kWlCompressionThreads = 256;  // compression CTA: 256 / T(nfft) pulses
constexpr int kWlDopplerThreads = 256;      // Doppler CTA: 256 / T(nfft) range columns

struct WlCompressionGroup {
    const float2* const* xs;   // device array: the group's CPI inputs (pulses x samples each)
    const float2* spectrum;    // nfft bins
    float2* y;                 // the group's compressed cube: rows x nfft
    int pulses, samples, nfft;
    int rows;                  // CPIs x pulses
    int entry0;                // first CTA of the group
};
struct WlCompressionParams {
    WlCompressionGroup g[kWlGroups];
    int groups;
    int cls;                   // resource class of every group of the launch
};

struct WlDopplerGroup {
    CUtensorMap map;           // the group's compressed cube, 2 nr floats x rows; box 2C x min(nd, 256)
    const float* window;       // pulses weights or null
    float* power;              // the group's power planes: CPIs x nd x nr
    int pulses, nr, nd;
    int tiles_x;               // column tiles per CPI
    int entry0;
};
struct WlDopplerParams {
    WlDopplerGroup g[kWlGroups];
    int groups;
    int cls;
};

struct WlCfarGroup {
    CUtensorMap map;           // the group's power planes, nr x (CPIs x nd); box of the tile geometry
    float* const* thr;         // device array: each CPI's threshold plane
    uint8_t* const* det;       // device array: each CPI's detection plane
    double scale64;            // alpha / reference cells
    float scale32;
    int rows, cols;            // nd, nr
    int tiles_x, tiles_y;
    int entry0;
};
struct WlCfarParams {
    WlCfarGroup g[kWlGroups];
    int groups;
};

// Range lengths the work-list compression kernel runs (powers of two 64 .. 8192), the
// resource class of a length (compression and Doppler), the CTAs for `rows` pulses of
// length n, and the launch of one class.
bool wl_compression_length(int n);
int wl_length_class(int n);
int wl_compression_ctas(int n, int rows);
int launch_compression_worklist(const WlCompressionParams& p, int ctas, int cls, cudaStream_t stream);

// Doppler lengths the work-list Doppler kernel runs (powers of two 64 .. 1024), its
// columns per CTA and bulk-copy box height, and its launch.
bool wl_doppler_length(int n);
int wl_doppler_columns(int n);
int wl_doppler_box_rows(int n);
int launch_doppler_worklist(const WlDopplerParams& p, int ctas, int cls, cudaStream_t stream);

// CFAR window geometries with the tiled kernel, the tile's halo box (floats), and the launch
// over `tiles` entries (persistent CTAs, two halo buffers each).
bool wl_cfar_geometry(int gr, int gc, int rr, int rc, uint32_t* box_w, uint32_t* box_h);
int launch_cfar_worklist(const WlCfarParams& p, int tiles, int gr, int gc, int rr, int rc, cudaStream_t stream);

}  // namespace zkx
