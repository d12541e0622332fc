// Radar inputs synthesised on the device, so that CPIs are made where they are processed
// instead of crossing PCIe (a 2048 x 65536 CPI is 1 GiB):
//
//   * the Task1 LFM waveform and single-target echo with hashed uniform noise
//     (ZKX/Task1/pipeline/src/steps/step1/step1.cu:11-71): the same integer hash and FP32
//     noise scaling, so the noise is bit-identical; the chirp and Doppler phases are
//     evaluated in FP64 and rounded once (the reference evaluates them in FP32);
//   * the multi-target CPI model of the benchmarks and the serving load generator:
//     CN(0, noise_power) noise from a counter-based generator (SplitMix64 finaliser,
//     Box-Muller in FP64) plus point targets, each a delayed LFM chirp
//     s[m] = exp(i pi (B/L) (m - L/2)^2) with a Doppler ramp exp(i (2 pi k p / P + phi)).
//
// Every output element is a pure function of (seed, index), so any slice can be
// regenerated on any device.
#include <cstdint>

#include "fft_core.cuh"
#include "zkx_internal.h"

namespace zkx {
namespace {

// Task1's noise hash (step1.cu:11-25): a multiply-xorshift mix of the element index and
// the seed, kept identical so the noise sequence matches the reference.
__device__ __forceinline__ uint32_t task1_hash(uint32_t index, uint32_t seed)
{
    uint32_t h = seed ^ (index * 747796405u + 2891336453u);
    h = (h ^ (h >> 16)) * 2246822519u;
    h = (h ^ (h >> 13)) * 3266489917u;
    return h ^ (h >> 16);
}

// uniform in [-1, 1] from the low 16 bits, scaled by std, in the reference's FP32 order
__device__ __forceinline__ float task1_uniform(uint32_t index, uint32_t seed, float std_dev)
{
    return ((float)(task1_hash(index, seed) & 0xffffu) / 32767.5f - 1.0f) * std_dev;
}

__global__ void lfm_kernel(int length, double sample_rate, double bandwidth, float2* __restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= length) return;
    const double width = (double)length / sample_rate;
    const double t = (double)i / sample_rate - 0.5 * width;
    double s, c;
    sincospi(bandwidth / width * t * t, &s, &c);  // phase / pi = (B / T) t^2
    out[i] = make_float2((float)c, (float)s);
}

__global__ void task1_echo_kernel(const float2* __restrict__ waveform, int pulse_samples, long long count,
                                  int samples_per_pulse, int delay, double doppler_hz, uint32_t seed,
                                  double prf, double sample_rate, float amplitude, float noise_std,
                                  float2* __restrict__ noiseless, float2* __restrict__ noise,
                                  float2* __restrict__ echo)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < count;
         e += (long long)gridDim.x * blockDim.x) {
        const int pulse = (int)(e / samples_per_pulse);
        const int sample = (int)(e - (long long)pulse * samples_per_pulse);
        float2 target = make_float2(0.f, 0.f);
        const int src = sample - delay;
        if (src >= 0 && src < pulse_samples) {
            const double time = (double)pulse / prf + (double)sample / sample_rate;
            double s, c;
            sincospi(2.0 * doppler_hz * time, &s, &c);
            const float2 r = cmul(waveform[src], make_float2((float)c, (float)s));
            target = make_float2(amplitude * r.x, amplitude * r.y);
        }
        const uint32_t k = (uint32_t)(2 * e);
        const float2 n = make_float2(task1_uniform(k, seed, noise_std), task1_uniform(k + 1u, seed, noise_std));
        if (noiseless) noiseless[e] = target;
        if (noise) noise[e] = n;
        if (echo) echo[e] = make_float2(target.x + n.x, target.y + n.y);
    }
}

// ---- the CPI model

constexpr int kMaxSynthTargets = 64;

struct TargetTable {
    int count;
    int delay[kMaxSynthTargets];
    double amplitude[kMaxSynthTargets];
    double cycles[kMaxSynthTargets];  // Doppler cycles per pulse (bin / pulses)
    double phase[kMaxSynthTargets];   // initial phase / pi
};

__device__ __forceinline__ uint64_t splitmix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// Two N(0, 1) values for element e: u1 in (0, 1], u2 in [0, 1) (53-bit), Box-Muller in FP64.
__device__ __forceinline__ void gaussian_pair(uint64_t seed, uint64_t e, double& g1, double& g2)
{
    const uint64_t base = seed + (2 * e + 1) * 0x9e3779b97f4a7c15ull;
    const uint64_t a = splitmix64(base), b = splitmix64(base + 0x9e3779b97f4a7c15ull);
    const double u1 = ((double)(a >> 11) + 1.0) * 0x1.0p-53;
    const double u2 = (double)(b >> 11) * 0x1.0p-53;
    const double r = sqrt(-2.0 * log(u1));
    double s, c;
    sincospi(2.0 * u2, &s, &c);
    g1 = r * c;
    g2 = r * s;
}

__global__ void synth_cpi_kernel(int pulses, int samples, int chirp_length, double bandwidth,
                                 const TargetTable tt, uint64_t seed, double noise_scale,
                                 float2* __restrict__ out)
{
    const long long count = (long long)pulses * samples;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < count;
         e += (long long)gridDim.x * blockDim.x) {
        const int p = (int)(e / samples);
        const int n = (int)(e - (long long)p * samples);
        double re = 0.0, im = 0.0;
        if (noise_scale != 0.0) {
            double g1, g2;
            gaussian_pair(seed, (uint64_t)e, g1, g2);
            re = g1 * noise_scale;
            im = g2 * noise_scale;
        }
        for (int k = 0; k < tt.count; ++k) {
            const int m = n - tt.delay[k];
            if (m < 0 || m >= chirp_length) continue;
            const double d = (double)m - 0.5 * chirp_length;
            // chirp phase / pi + Doppler phase / pi
            double s, c;
            sincospi(bandwidth / chirp_length * d * d + 2.0 * tt.cycles[k] * p + tt.phase[k], &s, &c);
            re += tt.amplitude[k] * c;
            im += tt.amplitude[k] * s;
        }
        out[e] = make_float2((float)re, (float)im);
    }
}

unsigned grid_for(long long n)
{
    const long long b = (n + 255) / 256;
    return (unsigned)(b < 148LL * 64 ? (b > 0 ? b : 1) : 148LL * 64);
}

}  // namespace
}  // namespace zkx

using namespace zkx;

extern "C" int zkx_lfm_waveform_c64(int length, double sample_rate, double bandwidth, void* out,
                                    zkx_stream_t stream)
{
    if (length < 1 || !(sample_rate > 0) || !(bandwidth > 0) || !out)
        return fail(ZKX_INVALID_ARGUMENT, "lfm_waveform: length, sample_rate and bandwidth must be positive");
    ZKX_TRY(ensure_device_ready());
    lfm_kernel<<<(length + 255) / 256, 256, 0, stream>>>(length, sample_rate, bandwidth,
                                                        static_cast<float2*>(out));
    ZKX_LAUNCHED("lfm_kernel");
    return ZKX_SUCCESS;
}

extern "C" int zkx_task1_echo_c64(const void* waveform, int pulse_samples, int num_pulses,
                                  int samples_per_pulse, int delay, double doppler_hz, uint32_t seed,
                                  double prf, double sample_rate, double amplitude, double noise_std,
                                  void* noiseless, void* noise, void* echo, zkx_stream_t stream)
{
    if (!waveform || (!noiseless && !noise && !echo))
        return fail(ZKX_INVALID_ARGUMENT, "task1_echo: null pointer");
    if (num_pulses < 1 || samples_per_pulse < 1 || pulse_samples < 1 || pulse_samples > samples_per_pulse ||
        delay < 0 || delay + pulse_samples > samples_per_pulse)
        return fail(ZKX_INVALID_SHAPE, "task1_echo: the pulse must lie inside the receive window");
    if (!(prf > 0) || !(sample_rate > 0) || !(amplitude > 0) || !(noise_std >= 0))
        return fail(ZKX_INVALID_ARGUMENT, "task1_echo: prf, sample_rate, amplitude must be positive");
    ZKX_TRY(ensure_device_ready());
    const long long count = (long long)num_pulses * samples_per_pulse;
    task1_echo_kernel<<<grid_for(count), 256, 0, stream>>>(
        static_cast<const float2*>(waveform), pulse_samples, count, samples_per_pulse, delay, doppler_hz,
        seed, prf, sample_rate, (float)amplitude, (float)noise_std, static_cast<float2*>(noiseless),
        static_cast<float2*>(noise), static_cast<float2*>(echo));
    ZKX_LAUNCHED("task1_echo_kernel");
    return ZKX_SUCCESS;
}

extern "C" int zkx_synth_cpi_c64(int num_pulses, int samples_per_pulse, int chirp_length, double bandwidth,
                                 const zkx_synth_target* targets, int n_targets, uint64_t seed,
                                 double noise_power, void* out, zkx_stream_t stream)
{
    if (!out || (n_targets > 0 && !targets)) return fail(ZKX_INVALID_ARGUMENT, "synth_cpi: null pointer");
    if (num_pulses < 1 || samples_per_pulse < 1 || chirp_length < 1)
        return fail(ZKX_INVALID_SHAPE, "synth_cpi: shape must be positive");
    if (n_targets < 0 || n_targets > kMaxSynthTargets)
        return fail(ZKX_INVALID_ARGUMENT, "synth_cpi: at most 64 targets");
    if (!(noise_power >= 0)) return fail(ZKX_INVALID_ARGUMENT, "synth_cpi: noise_power must be >= 0");
    TargetTable tt{};
    tt.count = n_targets;
    for (int k = 0; k < n_targets; ++k) {
        tt.delay[k] = targets[k].delay;
        tt.amplitude[k] = targets[k].amplitude;
        tt.cycles[k] = (double)targets[k].doppler_bin / (double)num_pulses;
        tt.phase[k] = targets[k].phase / 3.141592653589793238462643383279502884;
    }
    ZKX_TRY(ensure_device_ready());
    const long long count = (long long)num_pulses * samples_per_pulse;
    synth_cpi_kernel<<<grid_for(count), 256, 0, stream>>>(num_pulses, samples_per_pulse, chirp_length,
                                                         bandwidth, tt, seed, sqrt(0.5 * noise_power),
                                                         static_cast<float2*>(out));
    ZKX_LAUNCHED("synth_cpi_kernel");
    return ZKX_SUCCESS;
}
