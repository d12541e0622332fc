/*
 * zkx_rd.h -- C ABI of the B200 radar range-Doppler library (libzkx_rd.so).
 *
 * Every entry point takes plain device pointers, element counts and a CUDA stream,
 * returns an int status and never throws.  Status values are the reference
 * library's ErrorCode numbers (ZKX/cusignal_cpp/include/cusignal/runtime/errors.h:18-41)
 * so a C++ shim can rethrow them unchanged.  Complex data are interleaved
 * complex64 (float re, float im), the layout of the reference's ComplexFloat and
 * TypedComplex<float> (include/cusignal/backends/fft/fft_interface.h:104-107,
 * include/cusignal/operators/filtering/filtering_typed.h:13).
 *
 * Pointers named x/y/out/threshold/... are device pointers.  Calls are
 * asynchronous on `stream` (NULL = the legacy default stream, which is what the
 * reference uses everywhere); host-side parameter errors are reported before any
 * work is queued.  The last failure's message is available per host thread from
 * zkx_last_error().
 *
 * Transform lengths (nfft), along range and along pulses: powers of two from 1 to 65536
 * (range lengths above 16384 run on clusters of two or four CTAs), and any other length
 * up to 32768 (Bluestein's chirp-z transform on power-of-two FFTs, as the reference's FFT
 * backend does for such lengths; its workspace comes from a stream-ordered pool).
 */
#ifndef ZKX_RD_H
#define ZKX_RD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define ZKX_API __attribute__((visibility("default")))
#else
#define ZKX_API
#endif

typedef struct CUstream_st* zkx_stream_t; /* identical to cudaStream_t */

enum {
    ZKX_SUCCESS = 0,
    ZKX_INVALID_ARGUMENT = 1001,
    ZKX_INVALID_SHAPE = 1002,
    ZKX_UNSUPPORTED_OPERATION = 1004,
    ZKX_CUDA_RUNTIME_ERROR = 2002,
    ZKX_OUT_OF_MEMORY = 2003,
    ZKX_BACKEND_ERROR = 2099,
    ZKX_RESOURCE_FAILED = 3002,
    ZKX_INTERNAL_ERROR = 9001
};

/* Window kinds, numbered as the reference's RadarWindowKind
 * (include/cusignal/operators/radartools/radartools_typed.h:59-65). */
enum {
    ZKX_WINDOW_NONE = 0,
    ZKX_WINDOW_HANN = 1,
    ZKX_WINDOW_HAMMING = 2,
    ZKX_WINDOW_EXPLICIT_FP32 = 3,
    ZKX_WINDOW_EXPLICIT_FP64 = 4
};

/* Business dtypes of the reference's operators (TypedComplex<T> components). */
enum {
    ZKX_DTYPE_F32 = 0,
    ZKX_DTYPE_F16 = 1,
    ZKX_DTYPE_I32 = 2,
    ZKX_DTYPE_I16 = 3,
    ZKX_DTYPE_I8 = 4
};

/* CA-CFAR evaluation modes. */
enum {
    /* Separable training-ring sums in FP32 with every cell whose power lies within
     * 1e-5 (relative) of its threshold re-decided in FP64: the detection mask equals
     * an FP64 CFAR evaluated on the same input. */
    ZKX_CFAR_ACCURATE = 0,
    /* The reference's FP32 integral image, summed in the reference's order: thresholds
     * and mask are bit-identical to ca_cfar_typed_cpu<float>. */
    ZKX_CFAR_COMPAT = 1
};

/* DFT arithmetic of range compression. */
enum {
    ZKX_PRECISION_FP32 = 0,     /* FP32 shared-memory FFT (all lengths) */
    /* The DFT passes as tcgen05 tensor-core GEMMs on split hi + lo operands accumulated in
     * FP32 (nfft 4096, 8192 or 16384): hi + lo FP16 with per-pulse power-of-two range
     * scaling (error close to FP32), or hi + lo BF16 (no scaling, about 16 significant
     * bits per operand). */
    ZKX_PRECISION_TC_F16 = 1,
    ZKX_PRECISION_TC_BF16 = 2
};

ZKX_API const char* zkx_last_error(void);
ZKX_API const char* zkx_version(void);

/* Device-side status of the library's kernels on the current device: waits for the
 * device to go idle and reports in *code the first error a kernel recorded since the
 * last clear (0 = none; 1 = a bulk-copy wait ran out of its ~1 s bound and the CTA
 * left without computing).  clear != 0 resets the word.  No counterpart in the
 * reference, whose kernels have no device-side waits. */
ZKX_API int zkx_kernel_status(int clear, int* code);

/* Self-test of that failure path (for tests and health checks; no counterpart in the
 * reference): one 32-thread CTA waits on a barrier that no copy completes, gives up
 * after limit_clocks SM clocks (1000 .. 2^31), records code 1 in the error word and
 * returns.  Nothing is left running; read the result with zkx_kernel_status. */
ZKX_API int zkx_selftest_wait_timeout(long long limit_clocks, zkx_stream_t stream);

/* pulse_compression: y[p, :] = IFFT(FFT(x[p, :nfft]) * conj(FFT(w*h/||w*h||, nfft))).
 * Replaces cusignal::pulse_compression_device<float>
 * (include/cusignal/operators/radartools/radartools_typed.h:257-262; computation
 * src/operators/radartools/radartools_typed.cu:184-223).
 * x [num_pulses, samples_per_pulse] complex64, replica [replica_length] complex64,
 * explicit_window [replica_length] float (only for the explicit kinds, else NULL),
 * y [num_pulses, nfft] complex64; nfft = -1 means samples_per_pulse.
 * Uses a library-owned per-device scratch buffer for the replica spectrum. */
ZKX_API int zkx_pulse_compression_c64(const void* x, int num_pulses, int samples_per_pulse,
                              const void* replica, int replica_length, int nfft, int normalize,
                              int window_kind, const float* explicit_window, void* y,
                              zkx_stream_t stream);

/* pulse_compression that allocates no device memory, for callers that cannot let a
 * library allocate: processing loops that must not call cudaMalloc/cudaFree once they
 * run (those calls can block and synchronise the device) and hosts whose device
 * memory is owned by another allocator or a fixed budget.  Same arguments and result
 * as zkx_pulse_compression_c64 (the caller passes inputs and outputs); the replica
 * spectrum goes to a file-scope device array of 16384 complex64 (128 KiB) that every
 * GPU loading the library holds until the process exits.  nfft above 16384 is
 * rejected with ZKX_INVALID_ARGUMENT, and an nfft that is not a power of two (with
 * nfft = -1: a samples_per_pulse that is not one) with ZKX_UNSUPPORTED_OPERATION, since
 * the chirp-z transform the allocating entry uses for those lengths needs a workspace.
 * The first call on a device initialises the library's twiddle table there (a
 * synchronous set-up) and looks up the array's device address, so make that first call
 * before any stream capture.  All calls share the array: calls that overlap on the GPU
 * (other streams or host threads) race.
 * No counterpart in the reference. */
ZKX_API int zkx_pulse_compression_c64_noalloc(const void* x, int num_pulses, int samples_per_pulse,
                                              const void* replica, int replica_length, int nfft,
                                              int normalize, int window_kind,
                                              const float* explicit_window, void* y,
                                              zkx_stream_t stream);

/* The replica spectrum alone: spectrum[k] = conj(FFT(w*h/||w*h||, nfft))[k] / nfft,
 * the per-bin factor that zkx_pulse_compression_spectrum_c64 applies.  For nfft above
 * 16384 the bins are stored in cluster order (bin k1 + R*k2 at index k1*16384 + k2,
 * R = nfft / 16384), the order the long compression kernel consumes them in.  Lets callers
 * keep a spectrum resident per waveform (no counterpart call in the reference, which
 * recomputes it inside radartools_typed.cu:199-215). */
ZKX_API int zkx_replica_spectrum_c64(const void* replica, int replica_length, int nfft, int normalize,
                             int window_kind, const float* explicit_window, void* spectrum,
                             zkx_stream_t stream);

/* pulse_compression with a precomputed spectrum from zkx_replica_spectrum_c64. */
ZKX_API int zkx_pulse_compression_spectrum_c64(const void* x, int num_pulses, int samples_per_pulse,
                                       int nfft, const void* spectrum, void* y,
                                       zkx_stream_t stream);

/* zkx_pulse_compression_spectrum_c64 with a chosen DFT arithmetic (ZKX_PRECISION_*); the
 * spectrum is the natural-order one of zkx_replica_spectrum_c64.  No counterpart in the
 * reference (its compression is FP32 only). */
ZKX_API int zkx_pulse_compression_spectrum_ex_c64(const void* x, int num_pulses, int samples_per_pulse,
                                                  int nfft, const void* spectrum, int precision,
                                                  void* y, zkx_stream_t stream);

/* pulse_doppler: out[k, n] = sum_p w[p] x[p, n] exp(-2 pi i k p / nfft), nfft = -1 means
 * num_pulses; optional power[k, n] = |out[k, n]|^2 (NULL to skip; out may also be NULL
 * when only the power is wanted).  Replaces cusignal::pulse_doppler_device<float>
 * (radartools_typed.h:294-311; computation radartools_typed.cu:225-244).
 * x [num_pulses, samples_per_pulse] complex64, out [nfft, samples_per_pulse] complex64. */
ZKX_API int zkx_pulse_doppler_c64(const void* x, int num_pulses, int samples_per_pulse, int nfft,
                          int window_kind, const float* explicit_window, void* out,
                          float* power, zkx_stream_t stream);

/* Batched complex-to-complex FFT of `batch` contiguous rows of n complex64 (n a power of
 * two up to 65536, or any length up to 32768); forward unnormalised, inverse scaled by 1/n;
 * x == y allowed.
 * Replaces FFTInterface::fft_batch_device / ifft_batch_device
 * (include/cusignal/backends/fft/fft_interface.h:499-536; fft_interface.cpp:385-470). */
ZKX_API int zkx_fft_c2c_c64(const void* x, int batch, int n, int inverse, void* y,
                            zkx_stream_t stream);

/* ambgfun: normalised ambiguity function of x against y (y = NULL means y = x) and its
 * cuts.  Replaces cusignal::ambgfun_device<float> (include/cusignal/operators/radartools/
 * radartools_typed.h:133-137; radartools_typed.cpp:422-463, computation
 * radartools_typed.cu:30-126).  x [x_count] complex64 of which the first nx samples enter
 * the sums while the norm runs over all x_count (the reference's rule for high-rank
 * inputs, whose first extent is nx); y likewise.  cut 0 = 2-D, out [nx+ny-1, nfreq];
 * 1 = delay cut (cut_value = delay), out [nfreq]; 2 = Doppler cut (cut_value = Doppler
 * frequency), out [nx+ny-1]; nfreq = the next power of two >= nx+ny-1, at most 65536.
 * fs must be nonzero for the cuts.  FP32 results; a zero norm gives NaN. */
ZKX_API int zkx_ambgfun_c64(const void* x, int x_count, int nx, const void* y, int y_count, int ny,
                            int cut, double fs, double cut_value, float* out, zkx_stream_t stream);

/* Output geometry of zkx_ambgfun_c64 (host only): element count, rows = nx+ny-1, nfreq. */
ZKX_API int zkx_ambgfun_shape(int nx, int ny, int cut, long long* count, int* rows, int* nfreq);

/* ---------------------------------------------------------------- synthesis
 * Inputs generated on the device (no counterpart entry in the reference library; the
 * Task1 pair replaces the kernels of ZKX/Task1/pipeline/src/steps/step1/step1.cu:11-71). */

/* Task1 LFM waveform: out[i] = exp(i pi (B / T) t^2), t = i / fs - T / 2, T = length / fs
 * (phase in FP64). */
ZKX_API int zkx_lfm_waveform_c64(int length, double sample_rate, double bandwidth, void* out,
                                 zkx_stream_t stream);

/* Task1 echo [num_pulses, samples_per_pulse]: the waveform delayed by `delay` samples with
 * Doppler phase exp(2 pi i f_d (p / prf + n / fs)) times amplitude (noiseless), uniform
 * noise in [-noise_std, noise_std] from the reference's per-element hash of `seed`
 * (bit-identical), and their sum (echo).  Any of the three outputs may be NULL. */
ZKX_API int zkx_task1_echo_c64(const void* waveform, int pulse_samples, int num_pulses,
                               int samples_per_pulse, int delay, double doppler_hz, uint32_t seed,
                               double prf, double sample_rate, double amplitude, double noise_std,
                               void* noiseless, void* noise, void* echo, zkx_stream_t stream);

/* One point target of the synthetic CPI model. */
typedef struct {
    int delay;         /* range delay in samples */
    int doppler_bin;   /* Doppler ramp exp(2 pi i bin p / num_pulses) */
    double amplitude;
    double phase;      /* radians */
} zkx_synth_target;

/* Synthetic CPI [num_pulses, samples_per_pulse]: CN(0, noise_power) noise from a
 * counter-based generator keyed by `seed` (a pure function of seed and element index)
 * plus up to 64 targets, each amplitude * s[n - delay] * exp(i (2 pi bin p / P + phase))
 * with the chirp s[m] = exp(i pi (bandwidth / L) (m - L/2)^2), m < chirp_length. */
ZKX_API int zkx_synth_cpi_c64(int num_pulses, int samples_per_pulse, int chirp_length,
                              double bandwidth, const zkx_synth_target* targets, int n_targets,
                              uint64_t seed, double noise_power, void* out, zkx_stream_t stream);

/* CFAR threshold multiplier alpha = N_ref * (pfa^(-1/N_ref) - 1), on the host in FP64.
 * Replaces cusignal::cfar_alpha_typed_cpu / cfar_alpha_device (radartools_typed.h:207-222,
 * radartools_typed.cpp:592-617). */
ZKX_API int zkx_cfar_alpha(double pfa, int reference_count, double* alpha);

/* Number of training cells of a 2-D CA-CFAR window (radartools_typed.cpp:203-212). */
ZKX_API int zkx_cfar_reference_count(int rank, int guard_rows, int guard_columns, int reference_rows,
                             int reference_columns);

/* 1-D (rank 1, columns ignored) or 2-D CA-CFAR on row-major FP32 input.  threshold
 * is 0 where the window does not fit; detections[i] = x[i] > threshold[i] (0/1 bytes).
 * Replaces cusignal::ca_cfar_device<float> (radartools_typed.h:173-195; computation
 * radartools_typed.cu:128-170, validation radartools_typed.cpp:161-220).
 * mode is ZKX_CFAR_ACCURATE or ZKX_CFAR_COMPAT; rank-1 input always uses the compat
 * algorithm (a single FP32 prefix sum, as the reference).  Compat mode uses a
 * library-owned per-device scratch buffer of rows*columns floats. */
ZKX_API int zkx_ca_cfar_f32(const float* x, int rank, int rows, int columns, int guard_rows,
                    int guard_columns, int reference_rows, int reference_columns, double pfa,
                    int mode, float* threshold, uint8_t* detections, zkx_stream_t stream);

/* Causal FIR along the last axis of [lines, n]: y[l, i] = sum_k b[k] x[l, i-k]
 * (+ zi[l, i] for i < nb-1 when zi is given; then zf[l, j] receives the final state).
 * Replaces cusignal::firfilter_device<float> / firfilter_fp32_resident_device
 * (include/cusignal/operators/filtering/filtering_typed.h:552-567;
 * computation src/operators/filtering/filtering_typed.cu:118-184). */
ZKX_API int zkx_fir_f32(const float* b, int nb, const float* x, int lines, int n, const float* zi,
                float* y, float* zf, zkx_stream_t stream);

/* Padding of zkx_firfilter2_f32, in the order of the reference's Firfilter2PadType
 * (include/cusignal/operators/filtering/filtering_typed.h, Firfilter2PadType). */
enum {
    ZKX_PAD_ODD = 0,
    ZKX_PAD_EVEN = 1,
    ZKX_PAD_CONSTANT = 2,
    ZKX_PAD_NONE = 3
};
/* Rounding of an odd-reflected pad value 2*x[edge] - x[reflected]: as the input's element
 * type does it in the reference (filtering_typed.cpp:1597-1620): float arithmetic, half
 * (rounded to half), or the 8/16/32-bit integer wrap. */
enum {
    ZKX_PAD_ROUND_F32 = 0,
    ZKX_PAD_ROUND_F16 = 1,
    ZKX_PAD_ROUND_I8 = 2,
    ZKX_PAD_ROUND_I16 = 3,
    ZKX_PAD_ROUND_I32 = 4
};

/* Zero-phase FIR along the last axis of [lines, n] (n > edge): the line is extended by
 * edge samples each side (edge = padlen when has_padlen, else 3*nb; 0 for ZKX_PAD_NONE),
 * filtered forward and backward with steady-state initial conditions, and cropped to n.
 * At most 4096 coefficients.  Replaces cusignal::firfilter2_device (filtering_typed.h,
 * firfilter2_device; layout filtering_typed.cpp:1226-1302, algorithm 1631-1730; device
 * computation filtering_typed.cu:186-286).  Method "gust" is not provided, as in the
 * reference. */
ZKX_API int zkx_firfilter2_f32(const float* b, int nb, const float* x, int lines, int n, int padtype,
                               int has_padlen, int padlen, int pad_rounding, float* y,
                               zkx_stream_t stream);

/* zkx_firfilter2_f32 with an explicit method (ZKX_FIR_AUTO / DIRECT / FFT).  With padding at
 * least as long as the filter (padlen >= nb, as the default 3 nb is) the result is one
 * convolution of the padded line with the taps' autocorrelation, which the FFT method evaluates
 * by overlap-save; ZKX_FIR_FFT with shorter padding returns ZKX_UNSUPPORTED_OPERATION. */
ZKX_API int zkx_firfilter2_ex_f32(const float* b, int nb, const float* x, int lines, int n, int padtype,
                                  int has_padlen, int padlen, int pad_rounding, float* y, int method,
                                  zkx_stream_t stream);

/* Analytic signal along the last axis of [lines, n]: x zero-padded or truncated to nfft
 * (-1 = n), DFT, one-sided mask, inverse DFT; y is complex64 [lines, nfft].  nfft a power
 * of two up to 65536 or any length up to 32768.  Replaces cusignal::hilbert_device
 * (filtering_typed.h, hilbert_device; layout filtering_typed.cpp:500-562, algorithm
 * 1813-1872; device computation filtering_typed.cu:327-352). */
ZKX_API int zkx_hilbert_f32(const float* x, int lines, int n, int nfft, void* y, zkx_stream_t stream);

/* FIR evaluation method of zkx_fir_ex_f32. */
enum {
    ZKX_FIR_AUTO = 0,    /* by tap count */
    ZKX_FIR_DIRECT = 1,  /* direct sums, 16 outputs per thread from shared memory */
    ZKX_FIR_FFT = 2      /* overlap-save convolution, two lines per complex transform (<= 4096 taps) */
};
/* zkx_fir_f32 with an explicit evaluation method (same results within FP32 rounding). */
ZKX_API int zkx_fir_ex_f32(const float* b, int nb, const float* x, int lines, int n, const float* zi,
                           float* y, float* zf, int method, zkx_stream_t stream);

/* Output length of upfirdn: floor(((n-1)*up + nh - 1) / down) + 1
 * (src/operators/filtering/filtering_typed.cpp:1091-1098). */
ZKX_API long long zkx_upfirdn_length(int n, int nh, int up, int down);

/* Causal polyphase upfirdn along the last axis of [lines, n] with zero extension.
 * Replaces cusignal::upfirdn_device<float> (filtering_typed.h:745-749; computation
 * filtering_typed.cu:597-645).  y is [lines, zkx_upfirdn_length(n, nh, up, down)]. */
ZKX_API int zkx_upfirdn_f32(const float* h, int nh, const float* x, int lines, int n, int up,
                    int down, float* y, zkx_stream_t stream);

/* resample_poly layout after gcd reduction (filtering_typed.cpp:933-1044). */
typedef struct {
    int up, down;            /* reduced factors */
    int identity;            /* 1 when up == down after reduction (a copy) */
    int output_samples;      /* ceil(n * up / down) */
    int coefficient_count;   /* taps of the designed (or given) filter */
    int half_length;
    int prefix_zeros;
    int output_start;
} zkx_resample_layout;

ZKX_API int zkx_resample_poly_layout(int n, int up, int down, int custom_coefficients,
                             int coefficient_count, zkx_resample_layout* layout);

/* Default design: Kaiser(beta) windowed sinc, cutoff 1/max(up, down), scaled to
 * sum to up, computed on the host in FP64 (filtering_typed.cpp:159-222).
 * taps (host) must hold layout->coefficient_count doubles. */
ZKX_API int zkx_resample_poly_design(const zkx_resample_layout* layout, double kaiser_beta,
                             double* taps);

/* The same windowed-sinc design with a caller-supplied window of coefficient_count values
 * (the reference's Hamming and explicit design windows, filtering_typed.cpp:195-204). */
ZKX_API int zkx_resample_poly_design_window(const zkx_resample_layout* layout, const double* window,
                                            double* taps);

/* Centred polyphase resampling along the last axis of [lines, n] with FP32 device
 * taps (already scaled by up).  Replaces the compute half of
 * cusignal::resample_poly_device<float> (filtering_typed.h:765-770;
 * filtering_typed.cpp:2717-2779, filtering_typed.cu:661-681).  y is
 * [lines, layout->output_samples]. */
ZKX_API int zkx_resample_poly_f32(const float* x, int lines, int n, const zkx_resample_layout* layout,
                          const float* taps, float* y, zkx_stream_t stream);

/* dst[i] = (float)src[i] for `count` scalars of `dtype` (complex data: 2 scalars per
 * element).  Replaces the reference's dtype staging before FP32 compute
 * (src/operators/filtering/filtering_kernels.cuh:1277 convert_signal_kernel,
 * radartools_kernels.cuh:215-237 pack kernels). */
ZKX_API int zkx_convert_to_f32(const void* src, int dtype, long long count, float* dst,
                               zkx_stream_t stream);

/* Integral CA-CFAR decision of the reference (radartools_kernels.cuh:24-37) for int32/16/8
 * input x and FP32 thresholds: detections[i] = x[i] > floor(threshold[i]) with NaN and
 * range saturation rules. */
ZKX_API int zkx_cfar_detect_int(const void* x, int dtype, const float* threshold, long long count,
                                uint8_t* detections, zkx_stream_t stream);

/* dst[c, r] = src[r, c] for a row-major [rows, cols] FP32 array (moves a filtering axis
 * last; no counterpart in the reference, whose kernels take axis strides). */
ZKX_API int zkx_transpose_f32(const float* src, int rows, int cols, float* dst, zkx_stream_t stream);
/* The same for complex64 elements. */
ZKX_API int zkx_transpose_c64(const void* src, int rows, int cols, void* dst, zkx_stream_t stream);

/* dst[i] = (double)src[i]: exact widening of FP32 results to the reference's FP64 result
 * storage (src/runtime/fp64_storage_finalize.cu:45-87). */
ZKX_API int zkx_widen_f32_to_f64(const float* src, long long count, double* dst,
                                 zkx_stream_t stream);

/* ------------------------------------------------------------ the fused chain */

/* Chain description: pulse_compression -> pulse_doppler (+|.|^2) -> 2-D CA-CFAR on one
 * CPI, the path of the reference's Task1 steps 2-4 (ZKX/Task1/pipeline/src/steps/
 * step2/step2.cu:7-47, step3/step3.cu:7-49, step4/step4.cu:22-100). */
typedef struct {
    int num_pulses;          /* P */
    int samples_per_pulse;   /* N (range samples) */
    int range_nfft;          /* -1: N */
    int doppler_nfft;        /* -1: P */
    int replica_length;
    int normalize;
    int range_window;        /* ZKX_WINDOW_* applied to the replica */
    int doppler_window;      /* ZKX_WINDOW_* applied across pulses */
    int guard_cells[2];      /* Doppler, range */
    int reference_cells[2];  /* Doppler, range */
    double pfa;
    int cfar_mode;           /* ZKX_CFAR_ACCURATE or ZKX_CFAR_COMPAT */
    int precision;           /* ZKX_PRECISION_* of range compression (0 = FP32) */
} zkx_rd_desc;

typedef struct zkx_rd_plan_s* zkx_rd_plan;

/* Creates a plan on the current device: validates the description, computes the
 * replica spectrum and the Doppler window once and keeps them resident.
 * replica: device [replica_length] complex64; explicit windows are device arrays
 * (NULL unless the matching kind is explicit). */
ZKX_API int zkx_rd_plan_create(const zkx_rd_desc* desc, const void* replica,
                       const float* range_window, const float* doppler_window,
                       zkx_stream_t stream, zkx_rd_plan* plan);
ZKX_API int zkx_rd_plan_destroy(zkx_rd_plan plan);

/* Output sizes of a plan: compressed [P, range_nfft], rd and power/threshold/detections
 * [doppler_nfft, range_nfft]. */
ZKX_API int zkx_rd_plan_shape(zkx_rd_plan plan, int* range_bins, int* doppler_bins);

/* Runs the chain on one CPI x [P, N] complex64.  compressed may be NULL only if the
 * caller does not need it (it is still produced internally in a plan-owned buffer);
 * rd may be NULL to skip storing the complex range-Doppler map. */
ZKX_API int zkx_rd_execute(zkx_rd_plan plan, const void* x, void* compressed, void* rd, float* power,
                   float* threshold, uint8_t* detections, zkx_stream_t stream);

/* The chain on `batch` CPIs stored back to back (x [batch, P, N]; outputs [batch, ...]),
 * one launch per stage for the whole batch (no counterpart in the reference, which runs
 * one CPI per call). */
ZKX_API int zkx_rd_execute_batch(zkx_rd_plan plan, const void* x, int batch, void* compressed,
                                 void* rd, float* power, float* threshold, uint8_t* detections,
                                 zkx_stream_t stream);

/* ---------------------------------------------------------------- autotuning
 * Per-shape kernel choices of a plan (no counterpart in the reference).  0 in a field
 * means the library's shape heuristic. */
enum {
    ZKX_COMPRESSION_DEFAULT = 0,
    ZKX_COMPRESSION_PLAIN = 1,       /* one launch per group of pulses */
    ZKX_COMPRESSION_PERSISTENT = 2,  /* persistent CTAs prefetching the next pulse (N 4096 .. 16384);
                                        one cluster per pulse (N 32768, 65536) */
    ZKX_COMPRESSION_LOCAL = 3        /* persistent CTAs (clusters above 16384 points) with a four-step
                                        transform whose later passes stay inside warps and the
                                        spectrum in tensor memory (N 4096 .. 65536) */
};
enum {
    ZKX_CFAR_TILE_DEFAULT = 0,
    ZKX_CFAR_TILE_FULL = 1,    /* 64 x 64 tile, row-sum planes of the whole tile (3 CTAs per SM) */
    ZKX_CFAR_TILE_HALVES = 2,  /* 64 x 64 tile, row-sum planes built in two 32-row halves (4 CTAs per SM) */
    ZKX_CFAR_TILE_STREAM = 3   /* persistent full tiles, two CTAs per SM, next tile's halo copied during
                                  this one; the default (thresholds equal to ZKX_CFAR_TILE_FULL's) */
};
typedef struct {
    int compression_variant;  /* ZKX_COMPRESSION_* */
    int doppler_columns;      /* range columns per CTA of the bulk-copy Doppler kernel: 8 or 16
                                 (4 or 8 at 2048 Doppler bins; 2 or 4 at 4096, where 1 selects
                                 the per-thread-load kernel) */
    int cfar_tile;            /* ZKX_CFAR_TILE_* (accurate-mode CA-CFAR of the tiled window sizes) */
    int compression_radix;    /* values per thread (radix plan) of the Stockham compression kernels
                                 (variants 1, 2): 0 = the plan table's; 16 or 32 where the other
                                 exists (range nfft 1024 .. 8192; it rounds differently) */
    int compression_ctas_per_sm;  /* cap on the persistent / four-step compression CTAs per SM (0 = all
                                     that fit; results unchanged) */
    int cfar_ctas_per_sm;     /* cap on the persistent CA-CFAR CTAs per SM (0 = all that fit) */
} zkx_rd_tuning;

/* Times every candidate of each stage on `batch` CPIs at x (device, the plan's shape) on
 * `stream`, keeps the fastest in the plan and in a process-wide table keyed by the plan's
 * shape, which plans created later with that shape start from.  Synchronises the stream;
 * allocates and frees temporary device buffers; run it at set-up, not in a timed loop. */
ZKX_API int zkx_rd_plan_autotune(zkx_rd_plan plan, const void* x, int batch, zkx_stream_t stream,
                                 zkx_rd_tuning* chosen);
ZKX_API int zkx_rd_plan_get_tuning(zkx_rd_plan plan, zkx_rd_tuning* tuning);
ZKX_API int zkx_rd_plan_set_tuning(zkx_rd_plan plan, const zkx_rd_tuning* tuning);

/* A CUDA graph of one zkx_rd_execute_batch with fixed pointers: create runs the chain once
 * eagerly (allocating any plan-owned buffer), then captures and instantiates it; launch
 * replays it on `stream` with one call.  No counterpart in the reference. */
typedef struct zkx_rd_graph_s* zkx_rd_graph;
ZKX_API int zkx_rd_graph_create(zkx_rd_plan plan, const void* x, int batch, void* compressed,
                                void* rd, float* power, float* threshold, uint8_t* detections,
                                zkx_rd_graph* graph);
ZKX_API int zkx_rd_graph_launch(zkx_rd_graph graph, zkx_stream_t stream);
ZKX_API int zkx_rd_graph_destroy(zkx_rd_graph graph);

/* ---------------------------------------------------------------- work list
 * The chain over CPIs of mixed shapes with ONE launch per stage (no counterpart in the
 * reference, whose Task1 pipeline runs one CPI per call).  create groups the items by
 * plan, allocates the compressed cubes and power planes of every CPI (grouped by plan,
 * library-owned) and device tables of the items' pointers, and builds the stage kernels'
 * parameter blocks; launch enqueues on `stream`
 *   range compression  work-list kernels over every (CPI, 256-thread pulse group) entry
 *                      with a range nfft that is a power of two from 64 to 8192;
 *   Doppler + |.|^2    work-list kernels over every (CPI, column tile) entry with a
 *                      Doppler nfft that is a power of two from 64 to 1024;
 *   CA-CFAR            one work-list kernel over every (CPI, 64 x 64 tile) entry of the
 *                      accurate mode with the tiled window geometry of the first such plan;
 * compression and Doppler take one launch per resource class present (lengths with up to
 * 16 values per thread, and with 32), each class its own registers and shared memory; at
 * most 24 plans per launch (more plans take one launch per 24).  A plan whose stage
 * falls outside these (longer or non-power-of-two transforms, a tuning choice that rounds
 * differently from the work-list kernel, compat mode, another window geometry) runs that
 * stage with its own kernels, one launch per plan (per CPI for CFAR).  Every CPI's
 * threshold and detections equal zkx_rd_execute of that CPI alone with its plan, bit for
 * bit, and so does its power plane, copied to `power` when that is not NULL.  Plans must
 * have FP32 precision; items must stay valid (and the plans alive) until destroy.  The
 * kernel choices are taken from the plans' tunings at create (a later tuning change needs a
 * new list).  Launches of one list share its library-owned buffers, so they must be ordered
 * (one stream, or events between streams).  launch may be captured into a CUDA graph.
 * count: 1 .. 65535. */
typedef struct zkx_rd_worklist_s* zkx_rd_worklist;
typedef struct {
    zkx_rd_plan plan;
    const void* x;             /* device complex64 [num_pulses][samples_per_pulse] */
    float* power;              /* optional device [doppler_bins][range_bins] */
    float* threshold;          /* device [doppler_bins][range_bins] */
    uint8_t* detections;       /* device [doppler_bins][range_bins] */
} zkx_rd_work_item;
ZKX_API int zkx_rd_worklist_create(const zkx_rd_work_item* items, int count, zkx_rd_worklist* out);
ZKX_API int zkx_rd_worklist_launch(zkx_rd_worklist list, zkx_stream_t stream);
/* Launch calls one zkx_rd_worklist_launch makes (a plan's own stage launch of a
 * non-power-of-two transform or of compat-mode CFAR issues several kernels per call), the
 * plans (groups), and the library-owned scratch bytes; any pointer may be NULL. */
ZKX_API int zkx_rd_worklist_info(zkx_rd_worklist list, int* launches, int* groups, long long* scratch_bytes);
ZKX_API int zkx_rd_worklist_destroy(zkx_rd_worklist list);

/* ---------------------------------------------------------------- serving loop
 * A continuous-batching request loop over the chain (no counterpart in the reference,
 * whose Task1 pipeline runs one CPI per call on the default stream).  CPIs of any
 * supported shape are submitted as they arrive; a worker thread admits them while
 * device slots and the HBM budget allow, fuses pending CPIs of one shape and waveform
 * into one batched launch per stage, and spreads the batches over several CUDA
 * streams so copies and kernels of different batches overlap.  Replica spectra and
 * Doppler windows stay resident per (shape, waveform).  Each batch runs in a workspace
 * block the server owns: the smallest idle block that is large enough, else a new block
 * (cudaMalloc, sizes rounded up to classes 2^k x {1, 1.25, 1.5, 1.75}) after idle blocks
 * are freed to make room; a batch's completion callback returns its block to the idle
 * list, and zkx_rd_server_destroy frees them all.  Every block held (in flight or idle)
 * plus the resident plans stays within the HBM budget: a batch is admitted only when its
 * block fits, so once the blocks of a stream's sizes exist nothing more is allocated. */

/* Zero fields take the defaults named in the comments. */
typedef struct {
    int normalize;           /* replica normalisation (0/1) */
    int range_window;        /* ZKX_WINDOW_NONE / HANN / HAMMING on the replica */
    int doppler_window;      /* ZKX_WINDOW_NONE / HANN / HAMMING across pulses */
    int guard_cells[2];      /* Doppler, range */
    int reference_cells[2];  /* Doppler, range */
    double pfa;
    int cfar_mode;           /* ZKX_CFAR_ACCURATE or ZKX_CFAR_COMPAT */
    int streams;             /* compute streams batches are spread over (2); copies use
                                one copy-in and one copy-out stream besides */
    int max_inflight;        /* batches on the device at once (2 * streams) */
    int max_batch;           /* CPIs of one shape fused into one batch (32, at most 64) */
    double hbm_fraction;     /* budget = this fraction of the free HBM at creation (0.8) */
    size_t budget_bytes;     /* nonzero: a lower cap on the budget */
    int max_pending;         /* submitted requests waiting for admission (0 = no bound); a
                                submit beyond it is refused at once with ZKX_RESOURCE_FAILED,
                                so an overloaded server sheds load instead of queueing it */
} zkx_rd_server_desc;

/* One CPI.  x and the outputs may be host memory (page-locked for the copies to
 * overlap) or device memory (a device-resident x is read in place); they must stay
 * valid until the request completes.
 * Outputs are [P, N] (Doppler bin major, range nfft = N, Doppler nfft = P): detections
 * is required, the others may be NULL.  Requests with the same waveform_id must pass
 * the same replica (device memory, read when the id is first seen with this shape). */
typedef struct {
    int num_pulses;
    int samples_per_pulse;   /* and num_pulses: at most 32768, or a power of two up to 65536 */
    uint64_t waveform_id;
    const void* replica;     /* complex64 [replica_length] */
    int replica_length;
    const void* x;           /* complex64 [P, N] */
    uint8_t* detections;
    float* threshold;
    float* power;
    void* rd;                /* complex64 */
} zkx_rd_request;

typedef struct {
    uint64_t submitted, completed, failed, batches;
    double mean_batch;       /* CPIs per batch */
    double p50_us, p99_us, max_us, mean_us;  /* submit -> results in the caller's buffers */
    double cpis_per_s;       /* completed / (last completion - first submission) */
    size_t budget_bytes;
    size_t peak_bytes;       /* most workspace-block bytes held at once (in flight + idle) */
    size_t plan_bytes;       /* resident replica spectra and Doppler windows */
    int plans;
    uint64_t refused;        /* submits refused because max_pending requests were waiting */
} zkx_rd_server_stats;

typedef struct zkx_rd_server_s* zkx_rd_server;

/* Creates the loop on the current device (starts its worker thread). */
ZKX_API int zkx_rd_server_create(const zkx_rd_server_desc* desc, zkx_rd_server* server);
/* Finishes every submitted request, then releases the loop. */
ZKX_API int zkx_rd_server_destroy(zkx_rd_server server);
/* Queues one CPI and returns at once with its ticket.  A request whose workspace
 * alone exceeds the budget is refused with ZKX_OUT_OF_MEMORY; with max_pending set, a
 * request arriving while that many wait for admission is refused with
 * ZKX_RESOURCE_FAILED (no ticket; the caller may retry or drop it). */
ZKX_API int zkx_rd_submit(zkx_rd_server server, const zkx_rd_request* request, uint64_t* ticket);
/* *done = 1 and the request's status once it has completed (the ticket is then
 * released); *done = 0 if it is still pending after timeout_ms (0 = do not wait,
 * negative = wait until it completes). */
ZKX_API int zkx_rd_poll(zkx_rd_server server, uint64_t ticket, int timeout_ms, int* done);
ZKX_API int zkx_rd_server_stats_get(zkx_rd_server server, zkx_rd_server_stats* stats);
ZKX_API int zkx_rd_server_stats_reset(zkx_rd_server server);

#ifdef __cplusplus
}
#endif
#endif /* ZKX_RD_H */
