// 2-D cell-averaging CFAR for sm_100a, two modes.
//
// Accurate mode (the chain's default).  A CTA owns a 64 x 64 tile of cells and
// stages the tile plus its (guard + training) halo in shared memory once.  The
// training-ring sum of a cell is assembled from separable pieces that are all sums
// of non-negative terms (no outer-minus-inner cancellation):
//   A[r][c] = sum of the 2*RR training rows of column c around row r
//   B[r][c] = sum of the 2*GR+1 guard rows of column c around row r
//   ring    = sum_{|dc|<=MC} A[r][c+dc] + sum_{GC<|dc|<=MC} B[r][c+dc]
// Every window sum is formed as (suffix of one W-block) + (prefix of the next), so a
// window costs one add after two adds of preparation per element and its relative
// error stays below W units in the last place.  The FP32 threshold is therefore
// within ~3e-6 (relative) of the FP64 one; every cell whose power lies within 1e-5
// of its threshold is re-decided with the ring summed in FP64, so the mask equals an
// FP64 CFAR on the same input.
//
// Compat mode reproduces the reference's FP32 integral image bit for bit
// (radartools_kernels.cuh:40-134): a column running sum, then a row running sum, in
// the same order and with the same corner formula.  It exists for parity checks
// against the reference; it is slower (the running sums are sequential).
//
// Algorithmic HBM traffic of the accurate kernel: 4 B read + 4 B threshold + 1 B
// mask = 9 B per cell.
#include "fft_core.cuh"
#include "tma.cuh"
#include "zkx_internal.h"
#include "worklist.h"

namespace zkx {
namespace {

constexpr int kCfarTY = 64;
constexpr int kCfarTX = 64;
constexpr int kCfarThreads = 256;
constexpr float kRecheckBand = 1e-5f;

// out[i] = v[i] + ... + v[i+W-1], i in [0, LEN-W], as suffix(block) + prefix(next block).
template <int W, int LEN>
__device__ __forceinline__ void window_sums(const float* v, float* out)
{
    static_assert(LEN >= W && W >= 1, "window");
    float pre[LEN], suf[LEN];
    static_for<0, LEN>([&](auto I) {
        constexpr int i = decltype(I)::value;
        if constexpr (i % W == 0) pre[i] = v[i];
        else pre[i] = pre[i - 1] + v[i];
    });
    static_for<0, LEN>([&](auto I) {
        constexpr int i = LEN - 1 - decltype(I)::value;
        constexpr int end = (i / W) * W + W - 1 < LEN - 1 ? (i / W) * W + W - 1 : LEN - 1;
        if constexpr (i == end) suf[i] = v[i];
        else suf[i] = suf[i + 1] + v[i];
    });
    static_for<0, LEN - W + 1>([&](auto I) {
        constexpr int i = decltype(I)::value;
        if constexpr (i % W == 0) out[i] = pre[i + W - 1];
        else out[i] = suf[i] + pre[i + W - 1];
    });
}

template <int GR, int GC, int RR, int RC>
__global__ void __launch_bounds__(kCfarThreads)
cfar_accurate_kernel(const float* __restrict__ x, int rows, int cols, float scale32,
                     double scale64, float* __restrict__ thr, uint8_t* __restrict__ det)
{
    constexpr int MR = GR + RR, MC = GC + RC;
    constexpr int TY = kCfarTY, TX = kCfarTX;
    constexpr int HR = TY + 2 * MR, HC = TX + 2 * MC;
    constexpr int PITCH = HC | 1;  // odd row pitch: a warp walking 32 rows hits 32 banks
    extern __shared__ float csm[];
    float* P = csm;                       // [HR][PITCH] input tile with halo
    float* SA = P + HR * PITCH;           // [TY][PITCH] training-row column sums
    float* SB = SA + TY * PITCH;          // [TY][PITCH] guard-row column sums
    const int r0 = blockIdx.y * TY;
    const int c0 = blockIdx.x * TX;
    x += (size_t)blockIdx.z * rows * cols;  // map of a stacked batch
    thr += (size_t)blockIdx.z * rows * cols;
    det += (size_t)blockIdx.z * rows * cols;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int WARPS = kCfarThreads / 32;

    // 1. halo tile: every thread issues all of its (float2 or scalar) loads before the
    //    shared stores, so each SM keeps ~14 loads per thread in flight
    const bool vec = ((MC & 1) == 0) && ((cols & 1) == 0) &&
                     ((reinterpret_cast<uintptr_t>(x) & 7) == 0);
    if (vec) {
        constexpr int H2 = HC / 2;
        constexpr int ITEMS = HR * H2;
        constexpr int PER = (ITEMS + kCfarThreads - 1) / kCfarThreads;
        float2 tmp[PER];
#pragma unroll
        for (int u = 0; u < PER; ++u) {
            const int e = u * kCfarThreads + threadIdx.x;
            const int hr = e / H2, h2 = e - hr * H2;
            const int gr = r0 - MR + hr, gc = c0 - MC + 2 * h2;
            float2 v = make_float2(0.f, 0.f);
            if (e < ITEMS && gr >= 0 && gr < rows) {
                const float* xrow = x + (size_t)gr * cols;
                if (gc >= 0 && gc + 1 < cols) v = __ldg(reinterpret_cast<const float2*>(xrow + gc));
                else {
                    if (gc >= 0 && gc < cols) v.x = __ldg(xrow + gc);
                    if (gc + 1 >= 0 && gc + 1 < cols) v.y = __ldg(xrow + gc + 1);
                }
            }
            tmp[u] = v;
        }
#pragma unroll
        for (int u = 0; u < PER; ++u) {
            const int e = u * kCfarThreads + threadIdx.x;
            if (e < ITEMS) {
                const int hr = e / H2, h2 = e - hr * H2;
                P[hr * PITCH + 2 * h2] = tmp[u].x;
                P[hr * PITCH + 2 * h2 + 1] = tmp[u].y;
            }
        }
    } else {
        for (int hr = warp; hr < HR; hr += WARPS) {
            const int gr = r0 - MR + hr;
            for (int hc = lane; hc < HC; hc += 32) {
                const int gc = c0 - MC + hc;
                P[hr * PITCH + hc] = (gr >= 0 && gr < rows && gc >= 0 && gc < cols)
                                         ? __ldg(x + (size_t)gr * cols + gc) : 0.f;
            }
        }
    }
    __syncthreads();

    // 2. vertical pieces: one thread per (halo column, 16-row segment)
    constexpr int SEG = 16;
    constexpr int VL = SEG + 2 * MR;
    for (int item = threadIdx.x; item < HC * (TY / SEG); item += kCfarThreads) {
        const int seg = item / HC;
        const int hc = item - seg * HC;
        const int rb = seg * SEG;
        float v[VL];
#pragma unroll
        for (int i = 0; i < VL; ++i) v[i] = P[(rb + i) * PITCH + hc];
        float wt[VL - RR + 1], wg[VL - 2 * GR];
        window_sums<RR, VL>(v, wt);
        window_sums<2 * GR + 1, VL>(v, wg);
#pragma unroll
        for (int r = 0; r < SEG; ++r) {
            SA[(rb + r) * PITCH + hc] = wt[r] + wt[r + MR + GR + 1];
            SB[(rb + r) * PITCH + hc] = wg[r + MR - GR];
        }
    }
    __syncthreads();

    // 3. horizontal: a warp walks 32 rows of one 16-column segment
    constexpr int CS = 16;
    constexpr int HL = CS + 2 * MC;
    const int r = threadIdx.x % TY;
    const int cb = (threadIdx.x / TY) * CS;
    const int grow = r0 + r;
    if (grow >= rows) return;
    float a[HL], b[HL];
#pragma unroll
    for (int i = 0; i < HL; ++i) {
        a[i] = SA[r * PITCH + cb + i];
        b[i] = SB[r * PITCH + cb + i];
    }
    float wa[HL - 2 * MC], wb[HL - RC + 1];
    window_sums<2 * MC + 1, HL>(a, wa);
    window_sums<RC, HL>(b, wb);
    const bool row_interior = grow >= MR && grow < rows - MR;
    float tout[CS];
    uint8_t dout[CS];
#pragma unroll
    for (int j = 0; j < CS; ++j) {
        const int gcol = c0 + cb + j;
        const float xv = P[(r + MR) * PITCH + cb + j + MC];
        float t = 0.f;
        bool hit;
        if (row_interior && gcol >= MC && gcol < cols - MC) {
            const float ring = wa[j] + (wb[j] + wb[j + MC + GC + 1]);
            t = scale32 * ring;
            hit = xv > t;
            if (fabsf(xv - t) <= kRecheckBand * t) {
                // re-decide in FP64 from the staged tile
                double s = 0.0;
                for (int dr = -MR; dr <= MR; ++dr)
                    for (int dc = -MC; dc <= MC; ++dc)
                        if (dr < -GR || dr > GR || dc < -GC || dc > GC)
                            s += (double)P[(r + MR + dr) * PITCH + cb + j + MC + dc];
                const double t64 = scale64 * s;
                hit = (double)xv > t64;
                t = (float)t64;
            }
        } else {
            hit = xv > 0.f;
        }
        tout[j] = t;
        dout[j] = hit ? 1 : 0;
    }
    const int cstart = c0 + cb;
    float* trow = thr + (size_t)grow * cols + cstart;
    uint8_t* drow = det + (size_t)grow * cols + cstart;
    const bool full = cstart + CS <= cols;
    if (full && ((reinterpret_cast<uintptr_t>(trow) & 15) == 0)) {
        float4* tp = reinterpret_cast<float4*>(trow);
#pragma unroll
        for (int q = 0; q < CS / 4; ++q)
            tp[q] = make_float4(tout[4 * q], tout[4 * q + 1], tout[4 * q + 2], tout[4 * q + 3]);
    } else {
#pragma unroll
        for (int j = 0; j < CS; ++j)
            if (cstart + j < cols) trow[j] = tout[j];
    }
    if (full && ((reinterpret_cast<uintptr_t>(drow) & 15) == 0)) {
        uint4 packed;
        unsigned w[4];
#pragma unroll
        for (int q = 0; q < 4; ++q)
            w[q] = dout[4 * q] | (dout[4 * q + 1] << 8) | (dout[4 * q + 2] << 16) |
                   ((unsigned)dout[4 * q + 3] << 24);
        packed.x = w[0]; packed.y = w[1]; packed.z = w[2]; packed.w = w[3];
        *reinterpret_cast<uint4*>(drow) = packed;
    } else {
#pragma unroll
        for (int j = 0; j < CS; ++j)
            if (cstart + j < cols) drow[j] = dout[j];
    }
}

// TMA variant of the accurate kernel: the halo tile arrives as one 2-D bulk copy (box
// of BOXW x HR floats starting OFF columns left of the halo, so its x coordinate is a
// 16-byte multiple; rows and columns outside the image are zero-filled by the copy
// engine), which leaves the threads only the arithmetic.
template <int GR, int GC, int RR, int RC>
struct CfarTmaGeom {
    static constexpr int MR = GR + RR, MC = GC + RC;
    static constexpr int HR = kCfarTY + 2 * MR, HC = kCfarTX + 2 * MC;
    static constexpr int OFF = ((MC + 3) & ~3) - MC;       // leading pad columns
    static constexpr int BOXW = (HC + OFF + 3) & ~3;        // box width (floats)
    static constexpr int PITCH = HC | 1;                    // SA/SB pitch
    static constexpr size_t smem_bytes()
    {
        return (size_t)HR * BOXW * sizeof(float) + (size_t)2 * kCfarTY * PITCH * sizeof(float) + 16;
    }
};

// Vertical pieces of a staged 64 x 64 tile: one item per (halo column, 32-row segment), a
// round of the CTA's threads for the 2/8 window (84 halo columns x 2 segments); longer
// segments sum fewer halo rows per cell.  (Three segments of 22/21/21 rows, which keep 252
// of the 256 threads busy instead of 168, measured slower: 260.2 against 253.5 us for the
// 1024 x 16384 chain.)
template <int GR, int GC, int RR, int RC>
__device__ __forceinline__ void full_tile_vertical(const float* P, float* SA, float* SB)
{
    using G = CfarTmaGeom<GR, GC, RR, RC>;
    constexpr int MR = G::MR, HC = G::HC, OFF = G::OFF, BOXW = G::BOXW, PITCH = G::PITCH;
    constexpr int SEG = 32;
    constexpr int VL = SEG + 2 * MR;
    for (int item = threadIdx.x; item < HC * (kCfarTY / SEG); item += kCfarThreads) {
        const int seg = item / HC;
        const int hc = item - seg * HC;
        const int rb = seg * SEG;
        float v[VL];
#pragma unroll
        for (int i = 0; i < VL; ++i) v[i] = P[(rb + i) * BOXW + hc + OFF];
        float wt[VL - RR + 1], wg[VL - 2 * GR];
        window_sums<RR, VL>(v, wt);
        window_sums<2 * GR + 1, VL>(v, wg);
#pragma unroll
        for (int r = 0; r < SEG; ++r) {
            SA[(rb + r) * PITCH + hc] = wt[r] + wt[r + MR + GR + 1];
            SB[(rb + r) * PITCH + hc] = wg[r + MR - GR];
        }
    }
}

// Horizontal pass of a staged tile at (r0, c0) of a rows x cols map: thread t owns 16
// cells of tile row t % 64; writes their thresholds and detections (thr, det point at the
// map).  Rows below the map are skipped.
template <int GR, int GC, int RR, int RC>
__device__ __forceinline__ void full_tile_horizontal(const float* P, const float* SA, const float* SB, int r0,
                                                     int c0, int rows, int cols, float scale32, double scale64,
                                                     float* __restrict__ thr, uint8_t* __restrict__ det)
{
    using G = CfarTmaGeom<GR, GC, RR, RC>;
    constexpr int MR = G::MR, MC = G::MC, OFF = G::OFF, BOXW = G::BOXW, PITCH = G::PITCH;
    constexpr int CS = 16;
    constexpr int HL = CS + 2 * MC;
    const int r = threadIdx.x % kCfarTY;
    const int cb = (threadIdx.x / kCfarTY) * CS;
    const int grow = r0 + r;
    if (grow >= rows) return;
    float a[HL], b[HL];
#pragma unroll
    for (int i = 0; i < HL; ++i) {
        a[i] = SA[r * PITCH + cb + i];
        b[i] = SB[r * PITCH + cb + i];
    }
    float wa[HL - 2 * MC], wb[HL - RC + 1];
    window_sums<2 * MC + 1, HL>(a, wa);
    window_sums<RC, HL>(b, wb);
    // cell values: columns cb..cb+15 of tile row r (aligned 128-bit loads when possible)
    float xv[CS];
    const float* prow = P + (r + MR) * BOXW + cb + MC + OFF;
    if constexpr (((MC + OFF) & 3) == 0 && (BOXW & 3) == 0) {
#pragma unroll
        for (int q = 0; q < CS / 4; ++q) {
            const float4 f = reinterpret_cast<const float4*>(prow)[q];
            xv[4 * q] = f.x; xv[4 * q + 1] = f.y; xv[4 * q + 2] = f.z; xv[4 * q + 3] = f.w;
        }
    } else {
#pragma unroll
        for (int j = 0; j < CS; ++j) xv[j] = prow[j];
    }
    const bool row_interior = grow >= MR && grow < rows - MR;
    float tout[CS];
    uint8_t dout[CS];
#pragma unroll
    for (int j = 0; j < CS; ++j) {
        const int gcol = c0 + cb + j;
        float t = 0.f;
        bool hit;
        if (row_interior && gcol >= MC && gcol < cols - MC) {
            const float ring = wa[j] + (wb[j] + wb[j + MC + GC + 1]);
            t = scale32 * ring;
            hit = xv[j] > t;
            if (fabsf(xv[j] - t) <= kRecheckBand * t) {
                double s = 0.0;
                for (int dr = -MR; dr <= MR; ++dr)
                    for (int dc = -MC; dc <= MC; ++dc)
                        if (dr < -GR || dr > GR || dc < -GC || dc > GC)
                            s += (double)P[(r + MR + dr) * BOXW + cb + j + MC + OFF + dc];
                const double t64 = scale64 * s;
                hit = (double)xv[j] > t64;
                t = (float)t64;
            }
        } else {
            hit = xv[j] > 0.f;
        }
        tout[j] = t;
        dout[j] = hit ? 1 : 0;
    }
    const int cstart = c0 + cb;
    float* trow = thr + (size_t)grow * cols + cstart;
    uint8_t* drow = det + (size_t)grow * cols + cstart;
    const bool full = cstart + CS <= cols;
    if (full && ((reinterpret_cast<uintptr_t>(trow) & 15) == 0)) {
        float4* tp = reinterpret_cast<float4*>(trow);
#pragma unroll
        for (int q = 0; q < CS / 4; ++q)
            tp[q] = make_float4(tout[4 * q], tout[4 * q + 1], tout[4 * q + 2], tout[4 * q + 3]);
    } else {
#pragma unroll
        for (int j = 0; j < CS; ++j)
            if (cstart + j < cols) trow[j] = tout[j];
    }
    if (full && ((reinterpret_cast<uintptr_t>(drow) & 15) == 0)) {
        unsigned w[4];
#pragma unroll
        for (int q = 0; q < 4; ++q)
            w[q] = dout[4 * q] | (dout[4 * q + 1] << 8) | (dout[4 * q + 2] << 16) |
                   ((unsigned)dout[4 * q + 3] << 24);
        *reinterpret_cast<uint4*>(drow) = make_uint4(w[0], w[1], w[2], w[3]);
    } else {
#pragma unroll
        for (int j = 0; j < CS; ++j)
            if (cstart + j < cols) drow[j] = dout[j];
    }
}

template <int GR, int GC, int RR, int RC>
__global__ void __launch_bounds__(kCfarThreads, 3)
cfar_accurate_tma_kernel(const __grid_constant__ CUtensorMap tmap, int rows, int cols,
                         float scale32, double scale64, float* __restrict__ thr,
                         uint8_t* __restrict__ det, int* err)
{
    using G = CfarTmaGeom<GR, GC, RR, RC>;
    constexpr int BOXW = G::BOXW, PITCH = G::PITCH;
    extern __shared__ __align__(128) float csm[];
    float* P = csm;                           // [HR][BOXW]; halo column hc at P[.. + hc + OFF]
    float* SA = P + G::HR * BOXW;             // [TY][PITCH]
    float* SB = SA + kCfarTY * PITCH;         // [TY][PITCH]
    uint64_t* bar = reinterpret_cast<uint64_t*>(SB + kCfarTY * PITCH);
    const int r0 = blockIdx.y * kCfarTY;
    const int c0 = blockIdx.x * kCfarTX;
    // map of a stacked batch: its rows follow the previous map's; halo rows that reach a
    // neighbouring map only feed border cells, whose threshold is 0
    const int map_row0 = blockIdx.z * rows;
    thr += (size_t)blockIdx.z * rows * cols;
    det += (size_t)blockIdx.z * rows * cols;
    if (threadIdx.x == 0) mbar_init(bar, 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        mbar_arrive_expect_tx(bar, (uint32_t)(G::HR * BOXW * sizeof(float)));
        tma_load_2d(P, &tmap, c0 - G::MC - G::OFF, map_row0 + r0 - G::MR, bar);
    }
    const bool ok = mbar_wait_bounded(bar, 0);
    if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0) atomicCAS(err, 0, (int)kKernelTmaTimeout);
        return;
    }
    full_tile_vertical<GR, GC, RR, RC>(P, SA, SB);
    __syncthreads();
    full_tile_horizontal<GR, GC, RR, RC>(P, SA, SB, r0, c0, rows, cols, scale32, scale64, thr, det);
}

// Persistent form of the full-tile kernel: two CTAs per SM walk the tiles (column tile
// fastest, then row tile, then map) in steps of the grid, with two halo buffers, so the
// halo copy of the CTA's next tile is in flight during the arithmetic of the current one.
// Each tile is computed exactly as by cfar_accurate_tma_kernel.
template <int GR, int GC, int RR, int RC>
struct CfarStreamGeom {
    using G = CfarTmaGeom<GR, GC, RR, RC>;
    static constexpr int HALO = G::HR * G::BOXW;              // floats of one halo copy
    static constexpr int STRIDE = (HALO + 31) / 32 * 32;       // buffers on 128-byte boundaries
    static constexpr size_t smem_bytes()
    {
        return (size_t)2 * STRIDE * sizeof(float) + (size_t)2 * kCfarTY * G::PITCH * sizeof(float) + 16;
    }
};

template <int GR, int GC, int RR, int RC>
__global__ void __launch_bounds__(kCfarThreads, 2)
cfar_accurate_stream_kernel(const __grid_constant__ CUtensorMap tmap, int rows, int cols, int tiles_x,
                            int tiles_y, int batch, float scale32, double scale64, float* __restrict__ thr,
                            uint8_t* __restrict__ det, int* err)
{
    using G = CfarTmaGeom<GR, GC, RR, RC>;
    using GS = CfarStreamGeom<GR, GC, RR, RC>;
    extern __shared__ __align__(128) float csm[];
    // halo buffer b at csm + b * STRIDE
    float* SA = csm + 2 * GS::STRIDE;         // [TY][PITCH]
    float* SB = SA + kCfarTY * G::PITCH;      // [TY][PITCH]
    uint64_t* full = reinterpret_cast<uint64_t*>(SB + kCfarTY * G::PITCH);   // full[0], full[1]
    const int tiles = tiles_x * tiles_y * batch;
    const int step = (int)gridDim.x;
    auto issue = [&](int tile, int b) {
        const int tx = tile % tiles_x, rest = tile / tiles_x;
        const int ty = rest % tiles_y, z = rest / tiles_y;
        mbar_arrive_expect_tx(&full[b], (uint32_t)(GS::HALO * sizeof(float)));
        tma_load_2d(csm + b * GS::STRIDE, &tmap, tx * kCfarTX - G::MC - G::OFF, z * rows + ty * kCfarTY - G::MR, &full[b]);
    };
    if (threadIdx.x == 0) {
        mbar_init(&full[0], 1);
        mbar_init(&full[1], 1);
    }
    __syncthreads();
    const int first = (int)blockIdx.x;
    if (threadIdx.x == 0) {
        if (first < tiles) issue(first, 0);
        if (first + step < tiles) issue(first + step, 1);
    }
    int k = 0;
    for (int tile = first; tile < tiles; tile += step, ++k) {
        const int b = k & 1;
        const bool ok = mbar_wait_bounded(&full[b], (uint32_t)((k >> 1) & 1));
        if (__syncthreads_or(!ok)) {
            if (threadIdx.x == 0) {
                atomicCAS(err, 0, (int)kKernelTmaTimeout);
                // the copy that timed out and the one into the other buffer may still be in
                // flight: wait for them (bounded) before the shared memory is released
                mbar_wait_bounded(&full[b], (uint32_t)((k >> 1) & 1));
                if (tile + step < tiles) mbar_wait_bounded(&full[b ^ 1], (uint32_t)(((k + 1) >> 1) & 1));
            }
            return;
        }
        const int tx = tile % tiles_x, rest = tile / tiles_x;
        const int ty = rest % tiles_y, z = rest / tiles_y;
        const float* P = csm + b * GS::STRIDE;
        full_tile_vertical<GR, GC, RR, RC>(P, SA, SB);
        __syncthreads();
        full_tile_horizontal<GR, GC, RR, RC>(P, SA, SB, ty * kCfarTY, tx * kCfarTX, rows, cols, scale32,
                                             scale64, thr + (size_t)z * rows * cols, det + (size_t)z * rows * cols);
        __syncthreads();   // halo buffer b, SA and SB are free
        if (threadIdx.x == 0 && tile + 2 * step < tiles) issue(tile + 2 * step, b);
    }
}

// Second TMA variant: the same tile, halo copy, separable sums and FP64 re-check, with the
// row-sum planes built and consumed in two 32-row halves, so they take half the shared
// memory (about 55 KB per CTA: four CTAs per SM instead of three, at most 64 registers per
// thread), and the horizontal pass reads them with 128-bit loads (plane pitch = 4 modulo
// 32 words: eight consecutive rows of a quarter-warp land on distinct bank groups).
// A thread of the horizontal pass owns 8 cells of one row; a vertical item is 16 rows of
// one halo column.
template <int GR, int GC, int RR, int RC>
struct CfarTma2Geom {
    using G = CfarTmaGeom<GR, GC, RR, RC>;
    static constexpr int HALF = kCfarTY / 2;
    static constexpr int PITCH = ((G::HC + 27) / 32) * 32 + 4;   // >= HC, = 4 (mod 32)
    static constexpr size_t smem_bytes()
    {
        return (size_t)G::HR * G::BOXW * sizeof(float) + (size_t)2 * HALF * PITCH * sizeof(float) + 16;
    }
    static_assert(PITCH >= G::HC && PITCH % 32 == 4, "plane pitch");
};

template <int GR, int GC, int RR, int RC>
__global__ void __launch_bounds__(kCfarThreads, 4)
cfar_accurate_tma2_kernel(const __grid_constant__ CUtensorMap tmap, int rows, int cols,
                          float scale32, double scale64, float* __restrict__ thr,
                          uint8_t* __restrict__ det, int* err)
{
    using G = CfarTmaGeom<GR, GC, RR, RC>;
    using G2 = CfarTma2Geom<GR, GC, RR, RC>;
    constexpr int MR = G::MR, MC = G::MC, HC = G::HC, OFF = G::OFF, BOXW = G::BOXW;
    constexpr int PITCH = G2::PITCH, HALF = G2::HALF, TY = kCfarTY, TX = kCfarTX;
    static_assert(((MC + OFF) & 3) == 0 && (BOXW & 3) == 0, "128-bit cell loads");
    extern __shared__ __align__(128) float csm[];
    float* P = csm;                        // [HR][BOXW]; halo column hc at P[.. + hc + OFF]
    float* SA = P + G::HR * BOXW;          // [HALF][PITCH]
    float* SB = SA + HALF * PITCH;         // [HALF][PITCH]
    uint64_t* bar = reinterpret_cast<uint64_t*>(SB + HALF * PITCH);
    const int r0 = blockIdx.y * TY;
    const int c0 = blockIdx.x * TX;
    const int map_row0 = blockIdx.z * rows;
    thr += (size_t)blockIdx.z * rows * cols;
    det += (size_t)blockIdx.z * rows * cols;
    if (threadIdx.x == 0) mbar_init(bar, 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        mbar_arrive_expect_tx(bar, (uint32_t)(G::HR * BOXW * sizeof(float)));
        tma_load_2d(P, &tmap, c0 - MC - OFF, map_row0 + r0 - MR, bar);
    }
    const bool ok = mbar_wait_bounded(bar, 0);
    if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0) atomicCAS(err, 0, (int)kKernelTmaTimeout);
        return;
    }
    constexpr int SEG = 16, VL = SEG + 2 * MR;
    constexpr int CS = 8, HL = CS + 2 * MC, HL4 = (HL + 3) / 4;
    const int hr = threadIdx.x & 31;          // horizontal: row within the half
    const int cb = (threadIdx.x >> 5) * CS;    // horizontal: first of 8 columns
    for (int h = 0; h < 2; ++h) {
        // vertical pieces of rows [h HALF, h HALF + HALF): one item per (halo column, 16 rows)
        for (int item = threadIdx.x; item < HC * (HALF / SEG); item += kCfarThreads) {
            const int seg = item / HC;
            const int hc = item - seg * HC;
            const int rb = h * HALF + seg * SEG;
            float v[VL];
#pragma unroll
            for (int i = 0; i < VL; ++i) v[i] = P[(rb + i) * BOXW + hc + OFF];
            float wt[VL - RR + 1], wg[VL - 2 * GR];
            window_sums<RR, VL>(v, wt);
            window_sums<2 * GR + 1, VL>(v, wg);
#pragma unroll
            for (int r = 0; r < SEG; ++r) {
                SA[(seg * SEG + r) * PITCH + hc] = wt[r] + wt[r + MR + GR + 1];
                SB[(seg * SEG + r) * PITCH + hc] = wg[r + MR - GR];
            }
        }
        __syncthreads();
        const int tr = h * HALF + hr;          // row within the tile
        const int grow = r0 + tr;
        if (grow < rows) {
            float a[HL4 * 4], b[HL4 * 4];
#pragma unroll
            for (int q = 0; q < HL4; ++q) {
                const float4 fa = *reinterpret_cast<const float4*>(SA + hr * PITCH + cb + 4 * q);
                const float4 fb = *reinterpret_cast<const float4*>(SB + hr * PITCH + cb + 4 * q);
                a[4 * q] = fa.x; a[4 * q + 1] = fa.y; a[4 * q + 2] = fa.z; a[4 * q + 3] = fa.w;
                b[4 * q] = fb.x; b[4 * q + 1] = fb.y; b[4 * q + 2] = fb.z; b[4 * q + 3] = fb.w;
            }
            float wa[HL - 2 * MC], wb[HL - RC + 1];
            window_sums<2 * MC + 1, HL>(a, wa);
            window_sums<RC, HL>(b, wb);
            float xv[CS];
            const float* prow = P + (tr + MR) * BOXW + cb + MC + OFF;
#pragma unroll
            for (int q = 0; q < CS / 4; ++q) {
                const float4 f = reinterpret_cast<const float4*>(prow)[q];
                xv[4 * q] = f.x; xv[4 * q + 1] = f.y; xv[4 * q + 2] = f.z; xv[4 * q + 3] = f.w;
            }
            const bool row_interior = grow >= MR && grow < rows - MR;
            float tout[CS];
            unsigned dlo = 0, dhi = 0;
#pragma unroll
            for (int j = 0; j < CS; ++j) {
                const int gcol = c0 + cb + j;
                float t = 0.f;
                bool hit;
                if (row_interior && gcol >= MC && gcol < cols - MC) {
                    const float ring = wa[j] + (wb[j] + wb[j + MC + GC + 1]);
                    t = scale32 * ring;
                    hit = xv[j] > t;
                    if (fabsf(xv[j] - t) <= kRecheckBand * t) {
                        double s = 0.0;
                        for (int dr = -MR; dr <= MR; ++dr)
                            for (int dc = -MC; dc <= MC; ++dc)
                                if (dr < -GR || dr > GR || dc < -GC || dc > GC)
                                    s += (double)P[(tr + MR + dr) * BOXW + cb + j + MC + OFF + dc];
                        const double t64 = scale64 * s;
                        hit = (double)xv[j] > t64;
                        t = (float)t64;
                    }
                } else {
                    hit = xv[j] > 0.f;
                }
                tout[j] = t;
                if (j < 4) dlo |= (hit ? 1u : 0u) << (8 * j);
                else dhi |= (hit ? 1u : 0u) << (8 * (j - 4));
            }
            const int cstart = c0 + cb;
            float* trow = thr + (size_t)grow * cols + cstart;
            uint8_t* drow = det + (size_t)grow * cols + cstart;
            if (cstart + CS <= cols && ((reinterpret_cast<uintptr_t>(trow) & 15) == 0) &&
                ((reinterpret_cast<uintptr_t>(drow) & 7) == 0)) {
                reinterpret_cast<float4*>(trow)[0] = make_float4(tout[0], tout[1], tout[2], tout[3]);
                reinterpret_cast<float4*>(trow)[1] = make_float4(tout[4], tout[5], tout[6], tout[7]);
                *reinterpret_cast<uint2*>(drow) = make_uint2(dlo, dhi);
            } else {
#pragma unroll
                for (int j = 0; j < CS; ++j)
                    if (cstart + j < cols) {
                        trow[j] = tout[j];
                        drow[j] = (uint8_t)(((j < 4 ? dlo : dhi) >> (8 * (j & 3))) & 1u);
                    }
            }
        }
        __syncthreads();  // the next half's vertical pass overwrites SA and SB
    }
}

// CA-CFAR of every map of a work list, whatever its shape: the persistent double-buffered
// walk of cfar_accurate_stream_kernel over the (group, map, 64 x 64 tile) entries of all
// groups, each tile computed exactly as by cfar_accurate_tma_kernel (so the thresholds
// equal the per-shape kernels'), each map writing its own threshold and detection planes.
template <int GR, int GC, int RR, int RC>
__global__ void __launch_bounds__(kCfarThreads, 2)
cfar_worklist_kernel(const __grid_constant__ WlCfarParams p, int tiles, int* err)
{
    using G = CfarTmaGeom<GR, GC, RR, RC>;
    using GS = CfarStreamGeom<GR, GC, RR, RC>;
    extern __shared__ __align__(128) float csm[];
    // halo buffer b at csm + b * STRIDE
    float* SA = csm + 2 * GS::STRIDE;         // [TY][PITCH]
    float* SB = SA + kCfarTY * G::PITCH;      // [TY][PITCH]
    uint64_t* full = reinterpret_cast<uint64_t*>(SB + kCfarTY * G::PITCH);
    const int step = (int)gridDim.x;
    // entry -> group, map, tile row, tile column
    auto locate = [&](int tile, int& gi, int& b, int& ty, int& tx) {
        gi = 0;
        while (gi + 1 < p.groups && tile >= p.g[gi + 1].entry0) ++gi;
        const WlCfarGroup& W = p.g[gi];
        const int local = tile - W.entry0;
        tx = local % W.tiles_x;
        const int rest = local / W.tiles_x;
        ty = rest % W.tiles_y;
        b = rest / W.tiles_y;
    };
    auto issue = [&](int tile, int buf) {
        int gi, b, ty, tx;
        locate(tile, gi, b, ty, tx);
        mbar_arrive_expect_tx(&full[buf], (uint32_t)(GS::HALO * sizeof(float)));
        tma_load_2d(csm + buf * GS::STRIDE, &p.g[gi].map, tx * kCfarTX - G::MC - G::OFF,
                    b * p.g[gi].rows + ty * kCfarTY - G::MR, &full[buf]);
    };
    if (threadIdx.x == 0) {
        mbar_init(&full[0], 1);
        mbar_init(&full[1], 1);
    }
    __syncthreads();
    const int first = (int)blockIdx.x;
    if (threadIdx.x == 0) {
        if (first < tiles) issue(first, 0);
        if (first + step < tiles) issue(first + step, 1);
    }
    int k = 0;
    for (int tile = first; tile < tiles; tile += step, ++k) {
        const int buf = k & 1;
        const bool ok = mbar_wait_bounded(&full[buf], (uint32_t)((k >> 1) & 1));
        if (__syncthreads_or(!ok)) {
            if (threadIdx.x == 0) {
                atomicCAS(err, 0, (int)kKernelTmaTimeout);
                // the copy that timed out and the one into the other buffer may still be in
                // flight: wait for them (bounded) before the shared memory is released
                mbar_wait_bounded(&full[buf], (uint32_t)((k >> 1) & 1));
                if (tile + step < tiles) mbar_wait_bounded(&full[buf ^ 1], (uint32_t)(((k + 1) >> 1) & 1));
            }
            return;
        }
        int gi, b, ty, tx;
        locate(tile, gi, b, ty, tx);
        const WlCfarGroup& W = p.g[gi];
        const float* P = csm + buf * GS::STRIDE;
        full_tile_vertical<GR, GC, RR, RC>(P, SA, SB);
        __syncthreads();
        full_tile_horizontal<GR, GC, RR, RC>(P, SA, SB, ty * kCfarTY, tx * kCfarTX, W.rows, W.cols, W.scale32,
                                             W.scale64, W.thr[b], W.det[b]);
        __syncthreads();   // halo buffer buf, SA and SB are free
        if (threadIdx.x == 0 && tile + 2 * step < tiles) issue(tile + 2 * step, buf);
    }
}

template <int GR, int GC, int RR, int RC>
int cfar_worklist_impl(const WlCfarParams& p, int tiles, cudaStream_t s)
{
    using GS = CfarStreamGeom<GR, GC, RR, RC>;
    const size_t smem = GS::smem_bytes();
    auto k = cfar_worklist_kernel<GR, GC, RR, RC>;
    ZKX_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int dev = 0, sms = 0, per_sm = 0;
    ZKX_CUDA(cudaGetDevice(&dev));
    ZKX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    ZKX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kCfarThreads, smem));
    const int ctas = std::max(1, std::min(tiles, sms * std::max(per_sm, 1)));
    k<<<ctas, kCfarThreads, smem, s>>>(p, tiles, kernel_error_word());
    ZKX_LAUNCHED("cfar_worklist_kernel");
    return ZKX_SUCCESS;
}

template <int GR, int GC, int RR, int RC>
void cfar_box(uint32_t* w, uint32_t* h)
{
    using G = CfarTmaGeom<GR, GC, RR, RC>;
    *w = (uint32_t)G::BOXW;
    *h = (uint32_t)G::HR;
}

// Any window geometry with guard + train up to 32 cells each way: a 32 x 32 tile per CTA,
// the tile and its halo staged in shared memory once, the training ring summed separably in
// FP64 (per halo column the training-row and guard-row sums, then per cell the column sums
// over the window's width), the threshold FP64 * alpha / N.  A cell within 1e-12 of its
// threshold is re-decided with the ring summed in the FP64 CFAR's own (row, column) order,
// so the mask equals an FP64 CFAR of the same input.  About (2 RR + 2 GR + 1) + (2 MC + 1 +
// 2 RC) FP64 adds per cell instead of the ring's (2 MR + 1)(2 MC + 1).
constexpr int kRtTile = 32;
constexpr int kRtMaxHalf = 32;

__host__ __device__ constexpr size_t cfar_rt_smem(int mr, int mc)
{
    return (size_t)2 * kRtTile * (kRtTile + 2 * mc) * sizeof(double) +
           (size_t)(kRtTile + 2 * mr) * ((kRtTile + 2 * mc) | 1) * sizeof(float);
}

__global__ void __launch_bounds__(256)
cfar_rt_kernel(const float* __restrict__ x, int rows, int cols, int gr, int gc, int rr, int rc,
               double scale64, float* __restrict__ thr, uint8_t* __restrict__ det)
{
    extern __shared__ __align__(16) double dsm[];
    const int MR = gr + rr, MC = gc + rc;
    const int HR = kRtTile + 2 * MR, HC = kRtTile + 2 * MC, HP = HC | 1;
    double* A = dsm;                                  // [32][HC] training-row sums
    double* B = A + kRtTile * HC;                     // [32][HC] guard-row sums
    float* P = reinterpret_cast<float*>(B + kRtTile * HC);   // [HR][HP] tile + halo
    const int r0 = blockIdx.y * kRtTile, c0 = blockIdx.x * kRtTile;
    x += (size_t)blockIdx.z * rows * cols;
    thr += (size_t)blockIdx.z * rows * cols;
    det += (size_t)blockIdx.z * rows * cols;
    for (int i = threadIdx.x; i < HR * HC; i += blockDim.x) {
        const int hr = i / HC, hc = i - (i / HC) * HC;
        const int r = r0 - MR + hr, c = c0 - MC + hc;
        P[hr * HP + hc] = (r >= 0 && r < rows && c >= 0 && c < cols) ? __ldg(&x[(size_t)r * cols + c]) : 0.f;
    }
    __syncthreads();
    // halo rows of cell row r (tile row): training rows r .. r+RR-1 and r+MR+GR+1 .. r+2MR,
    // guard rows r+MR-GR .. r+MR+GR
    for (int i = threadIdx.x; i < kRtTile * HC; i += blockDim.x) {
        const int r = i / HC, hc = i - (i / HC) * HC;
        double a = 0.0, b = 0.0;
        for (int k = 0; k < rr; ++k) a += (double)P[(r + k) * HP + hc];
        for (int k = 0; k < rr; ++k) a += (double)P[(r + MR + gr + 1 + k) * HP + hc];
        for (int k = -gr; k <= gr; ++k) b += (double)P[(r + MR + k) * HP + hc];
        A[r * HC + hc] = a;
        B[r * HC + hc] = b;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kRtTile * kRtTile; i += blockDim.x) {
        const int r = i / kRtTile, c = i - (i / kRtTile) * kRtTile;
        const int grow = r0 + r, gcol = c0 + c;
        if (grow >= rows || gcol >= cols) continue;
        const float xv = P[(r + MR) * HP + c + MC];
        float t = 0.f;
        bool hit;
        if (grow >= MR && grow < rows - MR && gcol >= MC && gcol < cols - MC) {
            double ring = 0.0;
            for (int dc = -MC; dc <= MC; ++dc) ring += A[r * HC + c + MC + dc];
            for (int dc = -MC; dc < -gc; ++dc) ring += B[r * HC + c + MC + dc];
            for (int dc = gc + 1; dc <= MC; ++dc) ring += B[r * HC + c + MC + dc];
            double t64 = scale64 * ring;
            if (fabs((double)xv - t64) <= 1e-12 * t64) {
                double s = 0.0;
                for (int dr = -MR; dr <= MR; ++dr)
                    for (int dc = -MC; dc <= MC; ++dc)
                        if (dr < -gr || dr > gr || dc < -gc || dc > gc)
                            s += (double)P[(r + MR + dr) * HP + c + MC + dc];
                t64 = scale64 * s;
            }
            t = (float)t64;
            hit = (double)xv > t64;
        } else {
            hit = xv > 0.f;
        }
        thr[(size_t)grow * cols + gcol] = t;
        det[(size_t)grow * cols + gcol] = hit ? 1 : 0;
    }
}

// Windows wider than 32 cells each way (beyond cfar_rt_kernel's shared memory): one thread
// per cell, ring summed directly in FP64.
__global__ void cfar_generic_kernel(const float* __restrict__ x, int rows, int cols, int gr, int gc,
                                    int rr, int rc, double scale64, float* __restrict__ thr,
                                    uint8_t* __restrict__ det)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)rows * cols) return;
    x += (size_t)blockIdx.y * rows * cols;
    thr += (size_t)blockIdx.y * rows * cols;
    det += (size_t)blockIdx.y * rows * cols;
    const int r = (int)(i / cols), c = (int)(i % cols);
    const int mr = gr + rr, mc = gc + rc;
    const float xv = x[i];
    float t = 0.f;
    bool hit;
    if (r >= mr && r < rows - mr && c >= mc && c < cols - mc) {
        double s = 0.0;
        for (int dr = -mr; dr <= mr; ++dr)
            for (int dc = -mc; dc <= mc; ++dc)
                if (dr < -gr || dr > gr || dc < -gc || dc > gc) s += (double)x[(size_t)(r + dr) * cols + c + dc];
        const double t64 = scale64 * s;
        t = (float)t64;
        hit = (double)xv > t64;
    } else {
        hit = xv > 0.f;
    }
    thr[i] = t;
    det[i] = hit ? 1 : 0;
}

// --------------------------------------------------------------- compat mode

__global__ void compat_column_cumsum_kernel(const float* __restrict__ x, int rows, int cols,
                                            float* __restrict__ cum)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    float run = 0.f;
    // unrolled so the loads of several rows are in flight ahead of the sequential adds
#pragma unroll 16
    for (int r = 0; r < rows; ++r) {
        run = __fadd_rn(run, x[(size_t)r * cols + c]);
        cum[(size_t)r * cols + c] = run;
    }
}

// One warp per 32 rows; 32 x 32 tiles are staged through shared memory so the
// sequential row scan still reads and writes HBM in coalesced rows.  The next tile's loads
// are issued into registers before the current tile is scanned, so their latency overlaps
// the scan's dependent adds, which run on registers.
__global__ void compat_row_cumsum_kernel(float* __restrict__ cum, int rows, int cols)
{
    __shared__ float tile[32][33];
    const int lane = threadIdx.x;
    const int r0 = blockIdx.x * 32;
    float run = 0.f;
    float next[32];
#pragma unroll
    for (int i = 0; i < 32; ++i) {
        const int rr = r0 + i;
        next[i] = (rr < rows && lane < cols) ? cum[(size_t)rr * cols + lane] : 0.f;
    }
    for (int c0 = 0; c0 < cols; c0 += 32) {
#pragma unroll
        for (int i = 0; i < 32; ++i) tile[i][lane] = next[i];
        __syncwarp();
        if (c0 + 32 < cols) {
#pragma unroll
            for (int i = 0; i < 32; ++i) {
                const int rr = r0 + i, cc = c0 + 32 + lane;
                next[i] = (rr < rows && cc < cols) ? cum[(size_t)rr * cols + cc] : 0.f;
            }
        }
        // this lane's row of the tile in registers (conflict-free: bank (lane + j) % 32), the
        // dependent adds on registers, then back
        float v[32];
#pragma unroll
        for (int j = 0; j < 32; ++j) v[j] = tile[lane][j];
#pragma unroll
        for (int j = 0; j < 32; ++j) {
            if (c0 + j < cols) {
                run = __fadd_rn(run, v[j]);
                v[j] = run;
            }
        }
#pragma unroll
        for (int j = 0; j < 32; ++j) tile[lane][j] = v[j];
        __syncwarp();
#pragma unroll
        for (int i = 0; i < 32; ++i) {
            const int rr = r0 + i, cc = c0 + lane;
            if (rr < rows && cc < cols) cum[(size_t)rr * cols + cc] = tile[i][lane];
        }
        __syncwarp();
    }
}

__global__ void compat_cumsum_1d_kernel(const float* __restrict__ x, int n, float* __restrict__ cum)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    float run = 0.f;
    for (int i = 0; i < n; ++i) {
        run = __fadd_rn(run, x[i]);
        cum[i] = run;
    }
}

// Threshold from the integral image with the reference's operation order
// (radartools_kernels.cuh:85-133); explicit _rn intrinsics keep nvcc from fusing.
__global__ void compat_threshold_kernel(const float* __restrict__ x, const float* __restrict__ cum,
                                        int rank, int rows, int cols, int gr, int gc, int rr,
                                        int rc, float alpha, int nref, float* __restrict__ thr,
                                        uint8_t* __restrict__ det)
{
    const long long index = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long count = (long long)rows * cols;
    if (index >= count) return;
    const float scale = __fdiv_rn(alpha, (float)nref);
    float t = 0.f;
    if (rank == 1) {
        const int i = (int)index;
        const int m = gr + rr;
        if (i >= m && i < rows - m) {
            const int orr = i + m, ol = i - m - 1, ir = i + gr, il = i - gr - 1;
            const float outer = ol >= 0 ? __fsub_rn(cum[orr], cum[ol]) : cum[orr];
            const float inner = __fsub_rn(cum[ir], cum[il]);
            t = __fmul_rn(scale, __fsub_rn(outer, inner));
        }
    } else {
        const int r = (int)(index / cols), c = (int)(index % cols);
        const int rm = gr + rr, cm = gc + rc;
        if (r >= rm && r < rows - rm && c >= cm && c < cols - cm) {
#define AT(r_, c_) cum[(size_t)(r_) * cols + (c_)]
            const int ot = r + rm, ol = r - rm - 1, orc = c + cm, olc = c - cm - 1;
            float outer = AT(ot, orc);
            if (ol >= 0) outer = __fsub_rn(outer, AT(ol, orc));
            if (olc >= 0) outer = __fsub_rn(outer, AT(ot, olc));
            if (ol >= 0 && olc >= 0) outer = __fadd_rn(outer, AT(ol, olc));
            float inner = __fsub_rn(AT(r + gr, c + gc), AT(r - gr - 1, c + gc));
            inner = __fsub_rn(inner, AT(r + gr, c - gc - 1));
            inner = __fadd_rn(inner, AT(r - gr - 1, c - gc - 1));
#undef AT
            t = __fmul_rn(scale, __fsub_rn(outer, inner));
        }
    }
    thr[index] = t;
    det[index] = x[index] > t ? 1 : 0;
}

template <int GR, int GC, int RR, int RC>
int accurate_impl(const float* x, int rows, int cols, float s32, double s64, float* thr,
                  uint8_t* det, int batch, int tile, int ctas_per_sm, cudaStream_t s)
{
    dim3 grid((cols + kCfarTX - 1) / kCfarTX, (rows + kCfarTY - 1) / kCfarTY, batch);
    using G = CfarTmaGeom<GR, GC, RR, RC>;
    if ((cols & 3) == 0 && (reinterpret_cast<uintptr_t>(x) & 15) == 0) {
        CUtensorMap map;
        if (encode_tensor_map_2d_f32(&map, x, (uint64_t)cols, (uint64_t)rows * batch,
                                     (uint64_t)cols * sizeof(float), G::BOXW, G::HR)) {
            if (tile == ZKX_CFAR_TILE_HALVES) {
                using G2 = CfarTma2Geom<GR, GC, RR, RC>;
                const size_t smem = G2::smem_bytes();
                auto k = cfar_accurate_tma2_kernel<GR, GC, RR, RC>;
                ZKX_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
                k<<<grid, kCfarThreads, smem, s>>>(map, rows, cols, s32, s64, thr, det, kernel_error_word());
                ZKX_LAUNCHED("cfar_accurate_tma2_kernel");
                return ZKX_SUCCESS;
            }
            if (tile == ZKX_CFAR_TILE_STREAM || tile == ZKX_CFAR_TILE_DEFAULT) {
                using GS = CfarStreamGeom<GR, GC, RR, RC>;
                const size_t smem = GS::smem_bytes();
                auto k = cfar_accurate_stream_kernel<GR, GC, RR, RC>;
                ZKX_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
                int dev = 0, sms = 0, per_sm = 0;
                ZKX_CUDA(cudaGetDevice(&dev));
                ZKX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
                ZKX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kCfarThreads, smem));
                per_sm = std::max(per_sm, 1);
                if (ctas_per_sm > 0) per_sm = std::min(per_sm, ctas_per_sm);
                const long long tiles = (long long)grid.x * grid.y * grid.z;
                const int ctas = (int)std::min<long long>(tiles, (long long)sms * per_sm);
                k<<<ctas, kCfarThreads, smem, s>>>(map, rows, cols, (int)grid.x, (int)grid.y, batch, s32, s64,
                                                   thr, det, kernel_error_word());
                ZKX_LAUNCHED("cfar_accurate_stream_kernel");
                return ZKX_SUCCESS;
            }
            const size_t smem = G::smem_bytes();
            auto k = cfar_accurate_tma_kernel<GR, GC, RR, RC>;
            ZKX_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            k<<<grid, kCfarThreads, smem, s>>>(map, rows, cols, s32, s64, thr, det, kernel_error_word());
            ZKX_LAUNCHED("cfar_accurate_tma_kernel");
            return ZKX_SUCCESS;
        }
    }
    constexpr int HR = kCfarTY + 2 * (GR + RR), HC = kCfarTX + 2 * (GC + RC);
    constexpr int PITCH = HC | 1;
    const size_t smem = (size_t)(HR + 2 * kCfarTY) * PITCH * sizeof(float);
    auto k = cfar_accurate_kernel<GR, GC, RR, RC>;
    ZKX_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k<<<grid, kCfarThreads, smem, s>>>(x, rows, cols, s32, s64, thr, det);
    ZKX_LAUNCHED("cfar_accurate_kernel");
    return ZKX_SUCCESS;
}

}  // namespace

int launch_ca_cfar_accurate(const float* x, int rows, int columns, int gr, int gc, int rr, int rc,
                            double alpha, int nref, float* threshold, uint8_t* detections,
                            int batch, int tile, cudaStream_t stream, int ctas_per_sm)
{
    if (batch < 1 || batch > 65535) return fail(ZKX_UNSUPPORTED_OPERATION, "ca_cfar: batch must be 1..65535");
    const double s64 = alpha / (double)nref;
    const float s32 = (float)s64;
#define ZKX_CFAR_CASE(A, B, C, D) \
    if (gr == A && gc == B && rr == C && rc == D) return accurate_impl<A, B, C, D>(x, rows, columns, s32, s64, threshold, detections, batch, tile, ctas_per_sm, stream);
    ZKX_CFAR_CASE(2, 2, 8, 8)
    ZKX_CFAR_CASE(1, 1, 4, 4)
    ZKX_CFAR_CASE(2, 2, 4, 4)
    ZKX_CFAR_CASE(1, 1, 2, 2)
    ZKX_CFAR_CASE(1, 2, 2, 6)
#undef ZKX_CFAR_CASE
    if (gr + rr <= kRtMaxHalf && gc + rc <= kRtMaxHalf) {
        const size_t smem = cfar_rt_smem(gr + rr, gc + rc);
        ZKX_CUDA(cudaFuncSetAttribute(cfar_rt_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        const dim3 grid((columns + kRtTile - 1) / kRtTile, (rows + kRtTile - 1) / kRtTile, batch);
        cfar_rt_kernel<<<grid, 256, smem, stream>>>(x, rows, columns, gr, gc, rr, rc, s64, threshold, detections);
        ZKX_LAUNCHED("cfar_rt_kernel");
        return ZKX_SUCCESS;
    }
    const long long count = (long long)rows * columns;
    cfar_generic_kernel<<<dim3((unsigned)((count + 255) / 256), batch), 256, 0, stream>>>(
        x, rows, columns, gr, gc, rr, rc, s64, threshold, detections);
    ZKX_LAUNCHED("cfar_generic_kernel");
    return ZKX_SUCCESS;
}

int launch_ca_cfar_compat(const float* x, int rank, int rows, int columns, int gr, int gc, int rr,
                          int rc, float alpha, int nref, float* cum, float* threshold,
                          uint8_t* detections, cudaStream_t stream)
{
    if (rank == 1) {
        compat_cumsum_1d_kernel<<<1, 1, 0, stream>>>(x, rows, cum);
        ZKX_LAUNCHED("compat_cumsum_1d_kernel");
        columns = 1;
    } else {
        compat_column_cumsum_kernel<<<(columns + 255) / 256, 256, 0, stream>>>(x, rows, columns, cum);
        ZKX_LAUNCHED("compat_column_cumsum_kernel");
        compat_row_cumsum_kernel<<<(rows + 31) / 32, 32, 0, stream>>>(cum, rows, columns);
        ZKX_LAUNCHED("compat_row_cumsum_kernel");
    }
    const long long count = (long long)rows * columns;
    compat_threshold_kernel<<<(unsigned)((count + 255) / 256), 256, 0, stream>>>(
        x, cum, rank, rows, columns, gr, gc, rr, rc, alpha, nref, threshold, detections);
    ZKX_LAUNCHED("compat_threshold_kernel");
    return ZKX_SUCCESS;
}

bool wl_cfar_geometry(int gr, int gc, int rr, int rc, uint32_t* box_w, uint32_t* box_h)
{
#define ZKX_CFAR_CASE(A, B, C, D) \
    if (gr == A && gc == B && rr == C && rc == D) { cfar_box<A, B, C, D>(box_w, box_h); return true; }
    ZKX_CFAR_CASE(2, 2, 8, 8)
    ZKX_CFAR_CASE(1, 1, 4, 4)
    ZKX_CFAR_CASE(2, 2, 4, 4)
    ZKX_CFAR_CASE(1, 1, 2, 2)
    ZKX_CFAR_CASE(1, 2, 2, 6)
#undef ZKX_CFAR_CASE
    return false;
}

int launch_cfar_worklist(const WlCfarParams& p, int tiles, int gr, int gc, int rr, int rc, cudaStream_t stream)
{
#define ZKX_CFAR_CASE(A, B, C, D) \
    if (gr == A && gc == B && rr == C && rc == D) return cfar_worklist_impl<A, B, C, D>(p, tiles, stream);
    ZKX_CFAR_CASE(2, 2, 8, 8)
    ZKX_CFAR_CASE(1, 1, 4, 4)
    ZKX_CFAR_CASE(2, 2, 4, 4)
    ZKX_CFAR_CASE(1, 1, 2, 2)
    ZKX_CFAR_CASE(1, 2, 2, 6)
#undef ZKX_CFAR_CASE
    return fail(ZKX_UNSUPPORTED_OPERATION, "cfar work list: window geometry without a tiled kernel");
}

}  // namespace zkx
