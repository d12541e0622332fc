// Internal host-side helpers shared by the library's translation units: status
// codes, the thread-local error message, CUDA error mapping and the per-device
// initialisation (twiddle table, cached scratch buffers).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <string>

#include "../../include/zkx_rd.h"
#include "rows.cuh"

namespace zkx {

void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int cuda_status(cudaError_t e, const char* what);

// Throw-free wrappers: evaluate, map a CUDA failure to ZKX_CUDA_RUNTIME_ERROR or
// ZKX_OUT_OF_MEMORY and return it from the enclosing function.
#define ZKX_CUDA(call)                                              \
    do {                                                            \
        cudaError_t zkx_e_ = (call);                                \
        if (zkx_e_ != cudaSuccess) return ::zkx::cuda_status(zkx_e_, #call); \
    } while (0)
#define ZKX_LAUNCHED(what)                                          \
    do {                                                            \
        cudaError_t zkx_e_ = cudaGetLastError();                    \
        if (zkx_e_ != cudaSuccess) return ::zkx::cuda_status(zkx_e_, what); \
    } while (0)
#define ZKX_TRY(call)                                               \
    do {                                                            \
        int zkx_rc_ = (call);                                       \
        if (zkx_rc_ != ZKX_SUCCESS) return zkx_rc_;                 \
    } while (0)

// Generate the FP64-accurate twiddle table on the current device (once).
int ensure_device_ready();
// Device address of the current device's twiddle table (after ensure_device_ready).
const float2* twiddle_table();
// Device address of the current device's kernel error word (after ensure_device_ready).
int* kernel_error_word();

// Grow-only per-device scratch buffer identified by a slot number; the returned
// pointer stays valid until the same slot is requested with a larger size on the
// same device.  Callers on one device must order their use of a slot on one stream.
enum ScratchSlot { kScratchReplica = 0, kScratchDopplerWindow = 1, kScratchCfarIntegral = 2,
                   kScratchPolyTaps = 3, kScratchAmbgfun = 4, kScratchSlots = 5 };
int scratch(ScratchSlot slot, std::size_t bytes, void** out);

// Stream-ordered workspace from the library's per-device pool (memory kept by the pool
// between uses): valid for work queued on `stream` after the call until released, so
// concurrent streams never share it.  Usable inside CUDA graph capture.
int stream_workspace(std::size_t bytes, cudaStream_t stream, void** out);
struct StreamWorkspace {
    void* ptr = nullptr;
    cudaStream_t stream = nullptr;
    StreamWorkspace() = default;
    StreamWorkspace(const StreamWorkspace&) = delete;
    StreamWorkspace& operator=(const StreamWorkspace&) = delete;
    ~StreamWorkspace()
    {
        if (ptr) cudaFreeAsync(ptr, stream);
    }
};

bool is_pow2(long long n);
int ilog2_host(long long n);

// Launchers implemented in the .cu files (all asynchronous on `stream`).
int launch_replica_spectrum(const float2* replica, int length, int nfft, int normalize,
                            int window_kind, const float* explicit_window, float2* spectrum,
                            cudaStream_t stream);
int launch_pulse_compression(const float2* x, int pulses, int samples, int nfft,
                             const float2* spectrum, float2* y, cudaStream_t stream);
// Tensor-core compression (tc_dft.cu): nfft 4096, 8192, 16384; natural-order spectrum.
int launch_pulse_compression_tc(const float2* x, int pulses, int samples, int nfft,
                                const float2* spectrum, float2* y, int precision,
                                cudaStream_t stream);
// Compression kernel choice: the library's default, the one-launch-per-pulse-group kernel,
// the persistent bulk-copy pipeline (N >= 4096, 16-byte aligned pulses) or the four-step
// kernels.  radix: values per thread of the first two (0 = the plan table's; the other of
// 16 / 32 at nfft 1024 .. 8192, which rounds differently); ctas_per_sm > 0 caps the
// persistent and four-step kernels' CTAs per SM (results unchanged).
int launch_pulse_compression_variant(const float2* x, int pulses, int samples, int nfft,
                                     const float2* spectrum, float2* y, int variant, cudaStream_t stream,
                                     int radix = 0, int ctas_per_sm = 0);
// columns: range columns per CTA of the bulk-copy Doppler kernel (8 or 16; 4 or 8 at 2048
// pulses, 2 or 4 at 4096, where 1 selects the per-thread-load kernel; 0 = by shape).
int launch_pulse_doppler(const float2* x, int pulses, int samples, int nfft,
                         const float* window, float2* out, float* power, int batch, int columns,
                         cudaStream_t stream);
int launch_fft_rows(const float2* x, int rows, int n, int inverse, float2* y, cudaStream_t stream);
// Lengths 32768 and 65536 (thread-block clusters, long_fft.cu); the spectrum of a long
// transform is kept in cluster order (bin k1 + R k2 at k1 * 16384 + k2, R = nfft / 16384).
int launch_long_replica_spectrum(const float2* replica, int length, int nfft, int normalize,
                                 int window_kind, const float* explicit_window, float2* spectrum,
                                 cudaStream_t stream);
// The concrete kernel ZKX_COMPRESSION_DEFAULT stands for at `pulses` pulses of a 32768- or
// 65536-point compression.
int resolve_long_compression_variant(int pulses, int nfft, int* resolved);
int launch_long_compression(const RowsContiguous& x, int pulses, int samples, int nfft,
                            const float2* spectrum, float2* y, int variant, cudaStream_t stream);
int launch_long_compression(const RowsTable& x, int pulses, int samples, int nfft,
                            const float2* spectrum, float2* y, int variant, cudaStream_t stream);
// The concrete ZKX_COMPRESSION_* kernel that `variant` stands for at `pulses` pulses of
// nfft points (ZKX_COMPRESSION_DEFAULT resolves by the four-step kernels' rule; any other
// value is returned as is).  Plans resolve it once from their per-CPI shape, so a CPI gives
// the same bits alone and inside any batch.
int resolve_compression_variant(int pulses, int nfft, int variant, int* resolved);
// Range compression of `count` CPIs [pulses_per_cpi, samples] read in place from
// separate buffers (count <= kMaxRowTable); y is [count * pulses_per_cpi, nfft].
// `variant` is a ZKX_COMPRESSION_* choice, as for launch_pulse_compression_variant.
int launch_pulse_compression_table(const float2* const* cpis, int count, int pulses_per_cpi,
                                   int samples, int nfft, const float2* spectrum, float2* y,
                                   int variant, cudaStream_t stream, int radix = 0, int ctas_per_sm = 0);
// The other radix plan the Stockham compression kernels have at nfft (0: none).
int compression_alt_radix(int nfft);
int launch_long_fft_rows(const float2* x, int rows, int n, int inverse, float2* y,
                         cudaStream_t stream);
int launch_doppler_window(int pulses, int window_kind, const float* explicit_window, float* out,
                          cudaStream_t stream);
// `tile` is a ZKX_CFAR_TILE_* kernel choice for the tiled window sizes; every choice gives
// the same detection mask (each re-decides near-threshold cells in FP64).
int launch_ca_cfar_accurate(const float* x, int rows, int columns, int guard_rows,
                            int guard_columns, int reference_rows, int reference_columns,
                            double alpha, int reference_count, float* threshold,
                            uint8_t* detections, int batch, int tile, cudaStream_t stream,
                            int ctas_per_sm = 0);
int launch_ca_cfar_compat(const float* x, int rank, int rows, int columns, int guard_rows,
                          int guard_columns, int reference_rows, int reference_columns,
                          float alpha, int reference_count, float* cumulative, float* threshold,
                          uint8_t* detections, cudaStream_t stream);
// method: ZKX_FIR_AUTO (by tap count), ZKX_FIR_DIRECT (register-blocked direct sums) or
// ZKX_FIR_FFT (overlap-save on the Stockham transforms, firfft.cu; up to 4096 taps).
int launch_fir(const float* b, int nb, const float* x, int lines, int n, const float* zi,
               float* y, float* zf, cudaStream_t stream, int method = ZKX_FIR_AUTO);
int launch_fir_fft(const float* b, int nb, const float* x, int lines, int n, const float* zi, float* y,
                   cudaStream_t stream);
// zkx_rd_execute_batch with an explicit compat-mode integral-image workspace
// (nd * nr floats; NULL = the plan's own), for callers that run one plan on several
// streams at once.  With a non-NULL `table` (batch <= kMaxRowTable entries) CPI b is
// read in place from table[b] and x is ignored.
int rd_execute_batch_ws(zkx_rd_plan p, const void* x, int batch, void* compressed, void* rd,
                        float* power, float* threshold, uint8_t* detections, float* cumulative,
                        cudaStream_t stream, const void* const* table = nullptr);
// Read-only view of a plan's resident state (capi.cu), for the work-list builder.
struct RdPlanView {
    zkx_rd_desc d;
    int range_nfft, doppler_nfft;
    const float2* spectrum;
    const float* doppler_window;   // null without a window
    float* cumulative;             // compat-mode integral image (null in accurate mode)
    double alpha;
    int nref;
    zkx_rd_tuning tuning;
};
int rd_plan_view(zkx_rd_plan p, RdPlanView* v);
// Transforms of any length (bluestein.cu): lengths that are not powers of two up to
// kMaxBluesteinLength by the chirp-z identity on power-of-two FFTs; spectra in natural order.
constexpr int kMaxBluesteinLength = 1 << 15;
int launch_dft_rows(const float2* x, int rows, int n, int inverse, float2* y, cudaStream_t stream);
int launch_replica_spectrum_any(const float2* replica, int length, int nfft, int normalize, int window_kind,
                                const float* explicit_window, float2* spectrum, cudaStream_t stream);
int launch_compression_any(const RowsContiguous& x, int pulses, int samples, int nfft, const float2* spectrum,
                           float2* y, cudaStream_t stream);
int launch_compression_any(const RowsTable& x, int pulses, int samples, int nfft, const float2* spectrum,
                           float2* y, cudaStream_t stream);
// Doppler transforms of any length up to 32768, and powers of two up to 65536 (transposed
// row passes; the single-CTA kernels cover powers of two up to 4096).
int launch_doppler_any(const float2* x, int pulses, int samples, int nfft, const float* window, float2* out,
                       float* power, int batch, cudaStream_t stream);
int launch_polyphase(const float* taps, int ntaps, int up, int down, long long offset,
                     const float* x, int lines, int n, float* y, int nout, cudaStream_t stream);

}  // namespace zkx
