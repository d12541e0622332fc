/*
 * Test infrastructure only (the oracle).  A plain-C restatement of the reference
 * library's CPU algorithms for the radar range-Doppler chain, plus FP64 "truth"
 * variants of the same mathematics.  Only tests/, the smoke check and bench.py's
 * CPU-baseline leg may load it; the product library never links or calls it.
 *
 * Reference files cited (paths within the ZKX_dev checkout):
 *   rt.cpp = ZKX/cusignal_cpp/src/operators/radartools/radartools_typed.cpp
 *   ft.cpp = ZKX/cusignal_cpp/src/operators/filtering/filtering_typed.cpp
 *
 * Complex arrays are interleaved (re, im).  All functions return 0 on success
 * and 1001 (the reference's INVALID_ARGUMENT code) on invalid arguments.
 */
#ifndef ZKX_RD_ORACLE_H
#define ZKX_RD_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Window kinds, numbered as RadarWindowKind (include/.../radartools_typed.h:59-65). */
enum { OR_WINDOW_NONE = 0, OR_WINDOW_HANN = 1, OR_WINDOW_HAMMING = 2,
       OR_WINDOW_EXPLICIT_FP32 = 3, OR_WINDOW_EXPLICIT_FP64 = 4 };

/* FP32 window value exactly as rt.cpp:238-251 evaluates it (float phase, cosf). */
float or_radar_window_f32(int kind, int index, int length, const float* explicit_window);

/* pulse_compression, direct double-precision circular correlation (rt.cpp:618-675).
 * x [P, N] complex64, tmpl [L] complex64, out [P, nfft] complex double. */
int or_pulse_compression_direct(const float* x, int num_pulses, int samples_per_pulse,
                                const float* tmpl, int template_length, int nfft,
                                int normalize, int window_kind, const float* explicit_window,
                                double* out);

/* The same operation through double-precision FFTs (power-of-two nfft only):
 * the FP64 truth used at sizes where the direct sum is too slow.  The window
 * is taken as float values (window_f32, length L, may be NULL for none). */
int or_pulse_compression_fft64(const float* x, int num_pulses, int samples_per_pulse,
                               const float* tmpl, int template_length, int nfft,
                               int normalize, const float* window_f32, double* out);

/* pulse_doppler, direct DFT along pulses (rt.cpp:714-759), including the
 * reference's float-rounded pi in the phase.  out [nfft, N] complex double. */
int or_pulse_doppler_direct(const float* x, int num_pulses, int samples_per_pulse, int nfft,
                            int window_kind, const float* explicit_window, double* out);

/* FP64 truth Doppler through double FFTs (power-of-two nfft), exact pi.
 * x is complex double so a chain can stay in FP64. */
int or_pulse_doppler_fft64(const double* x, int num_pulses, int samples_per_pulse, int nfft,
                           const float* window_f32, double* out, double* power);

/* cfar_alpha (rt.cpp:592-603). */
int or_cfar_alpha(double pfa, int reference_count, double* alpha);

/* Reference cell count for a 2-D window (rt.cpp:203-212). */
int or_cfar_reference_count_2d(int guard_rows, int guard_columns,
                               int reference_rows, int reference_columns);

/* CA-CFAR bit-exact restatement of the FP32 integral-image algorithm
 * (rt.cpp:161-220 validation/alpha, rt.cpp:465-555 computation).
 * rank 1 uses rows only.  threshold float, detections 0/1. */
int or_ca_cfar_compat_f32(const float* x, int rank, int rows, int columns,
                          int guard_rows, int guard_columns,
                          int reference_rows, int reference_columns, double pfa,
                          float* threshold, uint8_t* detections);

/* CA-CFAR FP64 truth: the same window geometry and border rule, with the
 * reference-cell sum taken over the training ring in double and
 * T = alpha64 / N_ref * sum.  threshold64 (may be NULL), detections x > T. */
int or_ca_cfar_f64(const float* x, int rows, int columns,
                   int guard_rows, int guard_columns,
                   int reference_rows, int reference_columns, double pfa,
                   double* threshold64, uint8_t* detections);

/* The same FP64 truth for output rows [row_begin, row_end) only, with the ring sum
 * taken separably: per input row, the full-width and the two side-band column sums
 * (each a direct FP64 sum of its cells), then the ring = sum of full-width sums over
 * the training rows + sum of side-band sums over the guard rows.  Every term is an
 * input cell (no difference of partial sums), so for a power plane no cancellation
 * enters; the result equals
 * or_ca_cfar_f64 up to FP64 summation order.  threshold64 / detections point at the
 * band's first output row ([row_end - row_begin, columns]); bands are independent, so
 * callers may compute them on several threads at once. */
int or_ca_cfar_f64_rows(const float* x, int rows, int columns,
                        int guard_rows, int guard_columns,
                        int reference_rows, int reference_columns, double pfa,
                        int row_begin, int row_end,
                        double* threshold64, uint8_t* detections);

/* firfilter along the last axis of [rows, n] (ft.cpp:1536-1590): double
 * accumulation in tap order, rounded to float.  zi/zf are [rows, nb-1] or NULL. */
int or_firfilter(const float* b, int nb, const float* x, int rows, int n,
                 const float* zi, float* y, float* zf);

/* upfirdn output length (ft.cpp:1046-1117). */
int64_t or_upfirdn_length(int n, int nh, int up, int down);

/* upfirdn along the last axis, FP32 accumulation in tap order (ft.cpp:2548-2616). */
int or_upfirdn_f32(const float* h, int nh, const float* x, int rows, int n,
                   int up, int down, float* out);

/* resample_poly layout (ft.cpp:933-1044). */
typedef struct {
    int up, down;             /* after gcd reduction */
    int identity;
    int output_samples;
    int coefficient_count;
    int half_length;
    int prefix_zeros;
    int output_start;
} or_resample_layout;

int or_resample_poly_layout(int n, int up, int down, int custom, int ncoeffs,
                            or_resample_layout* layout);

/* Default Kaiser(beta) windowed-sinc design scaled to sum = up, with the
 * reference's own polynomial I0 (ft.cpp:159-222).  taps has coefficient_count. */
int or_resample_poly_design(const or_resample_layout* layout, double beta, double* taps);

/* Centred polyphase filtering with double taps and double accumulation
 * (the default-design branch of ft.cpp:2617-2716).  out [rows, output_samples]. */
int or_resample_poly_f64(const double* taps, const or_resample_layout* layout,
                         const float* x, int rows, int n, double* out);

/* Same indexing with float taps and FP32 accumulation (custom-coefficient FP32 branch). */
int or_resample_poly_f32(const float* taps, const or_resample_layout* layout,
                         const float* x, int rows, int n, float* out);

/* ambgfun (rt.cpp:330-463): x [x_count] complex64 of which the first nx samples enter
 * the sums (the norm runs over all x_count); y likewise (y = NULL means y = x).
 * cut 0 = 2-D [rows, nfreq], 1 = delay cut [nfreq], 2 = Doppler cut [rows], with
 * rows = nx + ny - 1 and nfreq the next power of two; values in double.  Direct
 * double-precision sums in the reference's order. */
int or_ambgfun(const float* x, int x_count, int nx, const float* y, int y_count, int ny,
               int cut, double fs, double cut_value, double* out);

/* Task1 step 1 echo (ZKX/Task1/pipeline/src/steps/step1/step1.cu:11-71): uniform noise
 * from the reference's per-element hash (exact FP32), target = amplitude * waveform delayed
 * with the Doppler phase in FP64.  noise, noiseless: [P * N] complex (float / double). */
int or_task1_echo(const float* waveform, int pulse_samples, int num_pulses, int samples_per_pulse,
                  int delay, double doppler_hz, uint32_t seed, double prf, double sample_rate,
                  double amplitude, float noise_std, double* noiseless, float* noise);

/* firfilter2 (filtering_typed.cpp:1226-1302 layout, 1631-1730 algorithm) along the last
 * axis of x [lines, n]: odd/even/constant/none padding by edge (padlen, default 3 nb), the
 * odd pad value 2 x0 - x[r] rounded as `rounding` says (0 float, 1 half, 2/3/4 the 8/16/32
 * bit integer wrap), forward and backward FIR with steady-state initial conditions in
 * double, crop.  out [lines, n] double.  Returns OR_INVALID on the reference's errors. */
int or_firfilter2(const float* b, int nb, const float* x, int lines, int n, int padtype, int has_padlen,
                  int padlen, int rounding, double* out);

/* hilbert (filtering_typed.cpp:500-562 layout, 1819-1872 algorithm) along the last axis of
 * x [lines, n]: zero-pad/truncate to nfft, direct double DFT, one-sided mask, direct
 * inverse DFT.  out [lines, nfft] complex, interleaved double. */
int or_hilbert(const float* x, int lines, int n, int nfft, double* out);

#ifdef __cplusplus
}
#endif
#endif
