/*
 * Test infrastructure only (the oracle): plain-C restatement of the reference's
 * CPU algorithms for the range-Doppler chain, and FP64 truth variants.
 * See rd_oracle.h for the contract and the reference citations.
 *
 * Built with -ffp-contract=off so that float/double expressions round exactly
 * as the reference's host code does (x86-64, no fused multiply-add).
 */
#include "rd_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define OR_OK 0
#define OR_INVALID 1001

static const float kPiF = 3.14159265358979323846F;  /* rt.cpp:14 */
static const double kPi = 3.141592653589793238462643383279502884;

/* ---------------------------------------------------------------- windows */

float or_radar_window_f32(int kind, int index, int length, const float* explicit_window)
{
    /* rt.cpp:238-251 */
    if (kind == OR_WINDOW_EXPLICIT_FP32 || kind == OR_WINDOW_EXPLICIT_FP64)
        return explicit_window[index];
    if (kind == OR_WINDOW_NONE || length <= 1) return 1.0F;
    const float phase = 2.0F * kPiF * (float)index / (float)(length - 1);
    if (kind == OR_WINDOW_HANN) return 0.5F - 0.5F * cosf(phase);
    if (kind == OR_WINDOW_HAMMING) return 0.54F - 0.46F * cosf(phase);
    return 1.0F;
}

static int valid_window(int kind, const float* explicit_window)
{
    if (kind < OR_WINDOW_NONE || kind > OR_WINDOW_EXPLICIT_FP64) return 0;
    const int is_explicit = kind == OR_WINDOW_EXPLICIT_FP32 || kind == OR_WINDOW_EXPLICIT_FP64;
    return is_explicit == (explicit_window != NULL);
}

/* ------------------------------------------------------- double FFT (truth) */

static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

/* In-place iterative radix-2 FFT on interleaved doubles; sign -1 forward, +1 inverse
 * (unscaled).  Twiddles are evaluated directly with cos/sin per index. */
static void fft64_inplace(double* a, int n, int sign)
{
    for (int i = 1, j = 0; i < n; ++i) {
        int bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            double tr = a[2 * i], ti = a[2 * i + 1];
            a[2 * i] = a[2 * j]; a[2 * i + 1] = a[2 * j + 1];
            a[2 * j] = tr; a[2 * j + 1] = ti;
        }
    }
    for (int len = 2; len <= n; len <<= 1) {
        const int half = len >> 1;
        for (int k = 0; k < half; ++k) {
            const double ang = sign * 2.0 * kPi * (double)k / (double)len;
            const double wr = cos(ang), wi = sin(ang);
            for (int base = 0; base < n; base += len) {
                double* u = a + 2 * (base + k);
                double* v = a + 2 * (base + k + half);
                const double vr = v[0] * wr - v[1] * wi;
                const double vi = v[0] * wi + v[1] * wr;
                v[0] = u[0] - vr; v[1] = u[1] - vi;
                u[0] = u[0] + vr; u[1] = u[1] + vi;
            }
        }
    }
}

/* ------------------------------------------------------ pulse compression */

int or_pulse_compression_direct(const float* x, int P, int N, const float* tmpl, int L,
                                int nfft, int normalize, int window_kind,
                                const float* explicit_window, double* out)
{
    /* rt.cpp:618-675 */
    if (nfft == -1) nfft = N;
    if (P < 1 || N < 1 || nfft < 1 || L < 1 || !valid_window(window_kind, explicit_window))
        return OR_INVALID;
    double* tr = (double*)malloc(sizeof(double) * (size_t)L);
    double* ti = (double*)malloc(sizeof(double) * (size_t)L);
    double norm = 0.0;
    for (int i = 0; i < L; ++i) {
        const double w = or_radar_window_f32(window_kind, i, L, explicit_window);
        tr[i] = (double)tmpl[2 * i] * w;
        ti[i] = (double)tmpl[2 * i + 1] * w;
        norm += tr[i] * tr[i] + ti[i] * ti[i];
    }
    norm = normalize ? sqrt(norm) : 1.0;
    for (int p = 0; p < P; ++p) {
        for (int o = 0; o < nfft; ++o) {
            double re = 0.0, im = 0.0;
            for (int tap = 0; tap < nfft && tap < L; ++tap) {
                const int s = (o + tap) % nfft;
                const size_t src = (size_t)p * N + s;
                const double xr = s < N ? (double)x[2 * src] : 0.0;
                const double xi = s < N ? (double)x[2 * src + 1] : 0.0;
                const double hr = tr[tap] / norm;
                const double hi = -ti[tap] / norm;
                re += xr * hr - xi * hi;
                im += xr * hi + xi * hr;
            }
            const size_t t = (size_t)p * nfft + o;
            out[2 * t] = re;
            out[2 * t + 1] = im;
        }
    }
    free(tr);
    free(ti);
    return OR_OK;
}

int or_pulse_compression_fft64(const float* x, int P, int N, const float* tmpl, int L,
                               int nfft, int normalize, const float* window_f32, double* out)
{
    if (nfft == -1) nfft = N;
    if (P < 1 || N < 1 || L < 1 || !is_pow2(nfft)) return OR_INVALID;
    double* h = (double*)calloc((size_t)2 * nfft, sizeof(double));
    double norm = 0.0;
    for (int i = 0; i < L; ++i) {
        const double w = window_f32 ? (double)window_f32[i] : 1.0;
        const double r = (double)tmpl[2 * i] * w, m = (double)tmpl[2 * i + 1] * w;
        norm += r * r + m * m;
        if (i < nfft) { h[2 * i] = r; h[2 * i + 1] = m; }
    }
    norm = normalize ? sqrt(norm) : 1.0;
    fft64_inplace(h, nfft, -1);
    double* row = (double*)malloc(sizeof(double) * 2 * (size_t)nfft);
    for (int p = 0; p < P; ++p) {
        for (int s = 0; s < nfft; ++s) {
            const size_t src = (size_t)p * N + s;
            row[2 * s] = s < N ? (double)x[2 * src] : 0.0;
            row[2 * s + 1] = s < N ? (double)x[2 * src + 1] : 0.0;
        }
        fft64_inplace(row, nfft, -1);
        for (int k = 0; k < nfft; ++k) {
            /* X * conj(H) / norm */
            const double ar = row[2 * k], ai = row[2 * k + 1];
            const double br = h[2 * k] / norm, bi = -h[2 * k + 1] / norm;
            row[2 * k] = ar * br - ai * bi;
            row[2 * k + 1] = ar * bi + ai * br;
        }
        fft64_inplace(row, nfft, +1);
        for (int o = 0; o < nfft; ++o) {
            out[2 * ((size_t)p * nfft + o)] = row[2 * o] / nfft;
            out[2 * ((size_t)p * nfft + o) + 1] = row[2 * o + 1] / nfft;
        }
    }
    free(row);
    free(h);
    return OR_OK;
}

/* ---------------------------------------------------------- pulse doppler */

int or_pulse_doppler_direct(const float* x, int P, int N, int nfft, int window_kind,
                            const float* explicit_window, double* out)
{
    /* rt.cpp:714-759; note the phase uses the float-rounded pi of rt.cpp:14. */
    if (nfft == -1) nfft = P;
    if (P < 1 || N < 1 || nfft < 1 || !valid_window(window_kind, explicit_window))
        return OR_INVALID;
    for (int f = 0; f < nfft; ++f) {
        for (int s = 0; s < N; ++s) {
            double re = 0.0, im = 0.0;
            for (int p = 0; p < P && p < nfft; ++p) {
                const double w = or_radar_window_f32(window_kind, p, P, explicit_window);
                const double angle = -2.0 * (double)kPiF * f * p / nfft;
                const double c = cos(angle), sn = sin(angle);
                const size_t src = (size_t)p * N + s;
                const double xr = (double)x[2 * src] * w;
                const double xi = (double)x[2 * src + 1] * w;
                re += xr * c - xi * sn;
                im += xr * sn + xi * c;
            }
            const size_t t = (size_t)f * N + s;
            out[2 * t] = re;
            out[2 * t + 1] = im;
        }
    }
    return OR_OK;
}

int or_pulse_doppler_fft64(const double* x, int P, int N, int nfft, const float* window_f32,
                           double* out, double* power)
{
    if (nfft == -1) nfft = P;
    if (P < 1 || N < 1 || !is_pow2(nfft)) return OR_INVALID;
    double* col = (double*)malloc(sizeof(double) * 2 * (size_t)nfft);
    for (int s = 0; s < N; ++s) {
        for (int p = 0; p < nfft; ++p) {
            if (p < P) {
                const double w = window_f32 ? (double)window_f32[p] : 1.0;
                col[2 * p] = x[2 * ((size_t)p * N + s)] * w;
                col[2 * p + 1] = x[2 * ((size_t)p * N + s) + 1] * w;
            } else {
                col[2 * p] = 0.0;
                col[2 * p + 1] = 0.0;
            }
        }
        fft64_inplace(col, nfft, -1);
        for (int f = 0; f < nfft; ++f) {
            const size_t t = (size_t)f * N + s;
            out[2 * t] = col[2 * f];
            out[2 * t + 1] = col[2 * f + 1];
            if (power) power[t] = col[2 * f] * col[2 * f] + col[2 * f + 1] * col[2 * f + 1];
        }
    }
    free(col);
    return OR_OK;
}

/* ------------------------------------------------------------------- CFAR */

int or_cfar_alpha(double pfa, int reference_count, double* alpha)
{
    /* rt.cpp:592-603 */
    if (reference_count < 1 || !isfinite(pfa) || pfa <= 0.0 || pfa > 1.0) return OR_INVALID;
    *alpha = (double)reference_count * (pow(pfa, -1.0 / (double)reference_count) - 1.0);
    return OR_OK;
}

int or_cfar_reference_count_2d(int gr, int gc, int rr, int rc)
{
    /* rt.cpp:206-209 */
    return 2 * rr * (2 * rc + 2 * gc + 1) + 2 * (2 * gr + 1) * rc;
}

static int validate_cfar(int rank, int rows, int columns, int gr, int gc, int rr, int rc,
                         double pfa)
{
    /* rt.cpp:161-200 (rank 1 and 2) */
    if (rank < 1 || rank > 2) return 0;
    if (gr < 0 || rr < 1 || rows <= 2 * (gr + rr)) return 0;
    if (rank == 2 && (gc < 0 || rc < 1 || columns <= 2 * (gc + rc))) return 0;
    if (!isfinite(pfa) || pfa <= 0.0 || pfa > 1.0) return 0;
    return 1;
}

int or_ca_cfar_compat_f32(const float* x, int rank, int rows, int columns, int gr, int gc,
                          int rr, int rc, double pfa, float* threshold, uint8_t* detections)
{
    if (!validate_cfar(rank, rows, columns, gr, gc, rr, rc, pfa)) return OR_INVALID;
    if (rank == 1) columns = 1;
    const int count_ref = rank == 2 ? or_cfar_reference_count_2d(gr, gc, rr, rc) : 2 * rr;
    const double nref = (double)count_ref;
    const float alpha = (float)(nref * (pow(pfa, -1.0 / nref) - 1.0)); /* rt.cpp:216-218 */
    const size_t count = (size_t)rows * columns;
    float* cum = (float*)malloc(sizeof(float) * count);
    for (size_t i = 0; i < count; ++i) threshold[i] = 0.0F;
    const float scale = alpha / (float)count_ref;
    if (rank == 1) {
        /* rt.cpp:477-499 */
        float running = 0.0F;
        for (int i = 0; i < rows; ++i) { running += x[i]; cum[i] = running; }
        const int m = gr + rr;
        for (int i = m; i < rows - m; ++i) {
            const int orr = i + m, ol = i - m - 1, ir = i + gr, il = i - gr - 1;
            const float outer = ol >= 0 ? cum[orr] - cum[ol] : cum[orr];
            const float inner = cum[ir] - cum[il];
            threshold[i] = scale * (outer - inner);
        }
    } else {
        /* rt.cpp:500-548: column cumsum, then row cumsum, then 4+4 corner differences */
        for (int c = 0; c < columns; ++c) {
            float running = 0.0F;
            for (int r = 0; r < rows; ++r) {
                const size_t i = (size_t)r * columns + c;
                running += x[i];
                cum[i] = running;
            }
        }
        for (int r = 0; r < rows; ++r) {
            float running = 0.0F;
            for (int c = 0; c < columns; ++c) {
                const size_t i = (size_t)r * columns + c;
                running += cum[i];
                cum[i] = running;
            }
        }
        const int rm = gr + rr, cm = gc + rc;
#define AT(r_, c_) cum[(size_t)(r_) * columns + (c_)]
        for (int r = rm; r < rows - rm; ++r) {
            for (int c = cm; c < columns - cm; ++c) {
                const int ot = r + rm, ol = r - rm - 1, orc = c + cm, olc = c - cm - 1;
                float outer = AT(ot, orc);
                if (ol >= 0) outer -= AT(ol, orc);
                if (olc >= 0) outer -= AT(ot, olc);
                if (ol >= 0 && olc >= 0) outer += AT(ol, olc);
                const float inner = AT(r + gr, c + gc) - AT(r - gr - 1, c + gc) -
                                    AT(r + gr, c - gc - 1) + AT(r - gr - 1, c - gc - 1);
                threshold[(size_t)r * columns + c] = scale * (outer - inner);
            }
        }
#undef AT
    }
    for (size_t i = 0; i < count; ++i) {
        /* rt.cpp:222-236, float branch; NaN thresholds never detect */
        detections[i] = (!isnan(threshold[i]) && x[i] > threshold[i]) ? 1 : 0;
    }
    free(cum);
    return OR_OK;
}

int or_ca_cfar_f64(const float* x, int rows, int columns, int gr, int gc, int rr, int rc,
                   double pfa, double* threshold64, uint8_t* detections)
{
    if (!validate_cfar(2, rows, columns, gr, gc, rr, rc, pfa)) return OR_INVALID;
    const int count_ref = or_cfar_reference_count_2d(gr, gc, rr, rc);
    double alpha;
    or_cfar_alpha(pfa, count_ref, &alpha);
    const int rm = gr + rr, cm = gc + rc;
    for (int r = 0; r < rows; ++r) {
        for (int c = 0; c < columns; ++c) {
            const size_t i = (size_t)r * columns + c;
            double t = 0.0;
            if (r >= rm && r < rows - rm && c >= cm && c < columns - cm) {
                double sum = 0.0;
                for (int dr = -rm; dr <= rm; ++dr) {
                    for (int dc = -cm; dc <= cm; ++dc) {
                        if (abs(dr) <= gr && abs(dc) <= gc) continue;
                        sum += (double)x[(size_t)(r + dr) * columns + (c + dc)];
                    }
                }
                t = alpha / (double)count_ref * sum;
            }
            if (threshold64) threshold64[i] = t;
            detections[i] = ((double)x[i] > t) ? 1 : 0;
        }
    }
    return OR_OK;
}

int or_ca_cfar_f64_rows(const float* x, int rows, int columns, int gr, int gc, int rr, int rc,
                        double pfa, int row_begin, int row_end, double* threshold64,
                        uint8_t* detections)
{
    /* Same geometry, border rule and test as or_ca_cfar_f64 (rt.cpp:161-220,465-555). */
    if (!validate_cfar(2, rows, columns, gr, gc, rr, rc, pfa)) return OR_INVALID;
    if (row_begin < 0 || row_end > rows || row_begin > row_end) return OR_INVALID;
    const int count_ref = or_cfar_reference_count_2d(gr, gc, rr, rc);
    double alpha;
    or_cfar_alpha(pfa, count_ref, &alpha);
    const double scale = alpha / (double)count_ref;
    const int rm = gr + rr, cm = gc + rc;
    const int in_lo = row_begin - rm < 0 ? 0 : row_begin - rm;
    const int in_hi = row_end + rm > rows ? rows : row_end + rm;
    const int band = in_hi - in_lo;
    /* full[r][c]: sum over |dc| <= cm; side[r][c]: sum over gc < |dc| <= cm */
    double* full = (double*)calloc((size_t)band * columns, sizeof(double));
    double* side = (double*)calloc((size_t)band * columns, sizeof(double));
    if (band > 0 && (!full || !side)) { free(full); free(side); return OR_INVALID; }
    for (int r = in_lo; r < in_hi; ++r) {
        const float* xr = x + (size_t)r * columns;
        double* fr = full + (size_t)(r - in_lo) * columns;
        double* sr = side + (size_t)(r - in_lo) * columns;
        for (int c = cm; c < columns - cm; ++c) {
            double s = 0.0;
            for (int dc = -cm; dc < -gc; ++dc) s += (double)xr[c + dc];
            for (int dc = gc + 1; dc <= cm; ++dc) s += (double)xr[c + dc];
            double f = s;
            for (int dc = -gc; dc <= gc; ++dc) f += (double)xr[c + dc];
            fr[c] = f;
            sr[c] = s;
        }
    }
    for (int r = row_begin; r < row_end; ++r) {
        const size_t o = (size_t)(r - row_begin) * columns;
        const int interior_row = r >= rm && r < rows - rm;
        for (int c = 0; c < columns; ++c) {
            double t = 0.0;
            if (interior_row && c >= cm && c < columns - cm) {
                double sum = 0.0;
                for (int dr = -rm; dr <= rm; ++dr) {
                    const size_t k = (size_t)(r + dr - in_lo) * columns + c;
                    sum += (dr < -gr || dr > gr) ? full[k] : side[k];
                }
                t = scale * sum;
            }
            if (threshold64) threshold64[o + c] = t;
            detections[o + c] = ((double)x[(size_t)r * columns + c] > t) ? 1 : 0;
        }
    }
    free(full);
    free(side);
    return OR_OK;
}

/* ------------------------------------------------------------------ filters */

int or_firfilter(const float* b, int nb, const float* x, int rows, int n, const float* zi,
                 float* y, float* zf)
{
    /* ft.cpp:1536-1590 (last axis, optional zi/zf). */
    if (nb < 1 || rows < 1 || n < 1) return OR_INVALID;
    const int state = nb - 1;
    for (int line = 0; line < rows; ++line) {
        const float* xl = x + (size_t)line * n;
        for (int full = 0; full < n + (zf && zi ? state : 0); ++full) {
            double v = 0.0;
            for (int tap = 0; tap <= state; ++tap) {
                const int s = full - tap;
                if (s >= 0 && s < n) v += (double)b[tap] * (double)xl[s];
            }
            if (zi && full < state) v += (double)zi[(size_t)line * state + full];
            if (full < n) y[(size_t)line * n + full] = (float)v;
            else zf[(size_t)line * state + (full - n)] = (float)v;
        }
    }
    return OR_OK;
}

int64_t or_upfirdn_length(int n, int nh, int up, int down)
{
    /* ft.cpp:1091-1098: floor(((n-1)*up + nh - 1) / down) + 1 */
    const long long num = ((long long)n - 1) * up + nh - 1;
    long long q = num / down;
    if (num % down < 0) --q;
    return q + 1;
}

int or_upfirdn_f32(const float* h, int nh, const float* x, int rows, int n, int up, int down,
                   float* out)
{
    /* ft.cpp:2585-2612 */
    if (nh < 1 || up < 1 || down < 1) return OR_INVALID;
    const int64_t nout = or_upfirdn_length(n, nh, up, down);
    for (int line = 0; line < rows; ++line) {
        for (int64_t m = 0; m < nout; ++m) {
            const long long filtered = (long long)m * down;
            float sum = 0.0F;
            for (int tap = 0; tap < nh; ++tap) {
                const long long cand = filtered - tap;
                if (cand % up != 0) continue;
                const long long src = cand / up;
                if (src < 0 || src >= n) continue;
                sum += h[tap] * x[(size_t)line * n + (size_t)src];
            }
            out[(size_t)line * nout + (size_t)m] = sum;
        }
    }
    return OR_OK;
}

static int gcd_int(int a, int b)
{
    while (b) { const int t = a % b; a = b; b = t; }
    return a;
}

int or_resample_poly_layout(int n, int up, int down, int custom, int ncoeffs,
                            or_resample_layout* L)
{
    /* ft.cpp:933-1044 */
    if (up < 1 || down < 1 || n < 0) return OR_INVALID;
    memset(L, 0, sizeof(*L));
    const int g = gcd_int(up, down);
    L->up = up / g;
    L->down = down / g;
    L->identity = L->up == 1 && L->down == 1;
    if (L->identity) { L->output_samples = n; return OR_OK; }
    L->output_samples = (int)(((long long)n * L->up + L->down - 1) / L->down);
    if (custom) {
        L->coefficient_count = ncoeffs;
        L->half_length = ncoeffs == 0 ? -1 : (ncoeffs - 1) / 2;
    } else {
        const int mr = L->up > L->down ? L->up : L->down;
        L->half_length = 10 * mr;
        L->coefficient_count = 2 * L->half_length + 1;
    }
    const int rem = ((L->half_length % L->down) + L->down) % L->down;
    L->prefix_zeros = L->down - rem;
    L->output_start = (L->half_length + L->prefix_zeros) / L->down;
    return OR_OK;
}

static double bessel_i0_poly(double v)
{
    /* ft.cpp:159-174: Abramowitz-Stegun 9.8.1 / 9.8.2 polynomial approximations */
    const double a = fabs(v);
    if (a < 3.75) {
        const double r = v / 3.75;
        const double y = r * r;
        return 1.0 + y * (3.5156229 + y * (3.0899424 + y * (1.2067492 + y * (0.2659732 +
               y * (0.0360768 + y * 0.0045813)))));
    }
    const double y = 3.75 / a;
    return exp(a) / sqrt(a) * (0.39894228 + y * (0.01328592 + y * (0.00225319 + y *
           (-0.00157565 + y * (0.00916281 + y * (-0.02057706 + y * (0.02635537 + y *
           (-0.01647633 + y * 0.00392377))))))));
}

int or_resample_poly_design(const or_resample_layout* L, double beta, double* taps)
{
    /* ft.cpp:176-222, Kaiser branch */
    const int count = L->coefficient_count, half = L->half_length;
    if (count < 1 || half < 1) return OR_INVALID;
    const double denom = bessel_i0_poly(beta);
    const double cutoff = 1.0 / (L->up > L->down ? L->up : L->down);
    double scale = 0.0;
    for (int i = 0; i < count; ++i) {
        const double ratio = (double)(i - half) / half;
        const double bounded = 1.0 - ratio * ratio > 0.0 ? 1.0 - ratio * ratio : 0.0;
        const double w = bessel_i0_poly(beta * sqrt(bounded)) / denom;
        const int off = i - half;
        const double sinc = off == 0 ? cutoff
            : sin(3.1415926535897932384626433832795 * cutoff * off) /
              (3.1415926535897932384626433832795 * off);
        taps[i] = sinc * w;
        scale += taps[i];
    }
    for (int i = 0; i < count; ++i) taps[i] = taps[i] / scale * L->up;
    return OR_OK;
}

int or_resample_poly_f64(const double* taps, const or_resample_layout* L, const float* x,
                         int rows, int n, double* out)
{
    /* ft.cpp:2687-2712 */
    for (int line = 0; line < rows; ++line) {
        for (int m = 0; m < L->output_samples; ++m) {
            const long long filtered = ((long long)m + L->output_start) * L->down;
            double sum = 0.0;
            for (int tap = 0; tap < L->coefficient_count; ++tap) {
                const long long cand = filtered - L->prefix_zeros - tap;
                if (cand % L->up != 0) continue;
                const long long src = cand / L->up;
                if (src < 0 || src >= n) continue;
                sum += taps[tap] * (double)x[(size_t)line * n + (size_t)src];
            }
            out[(size_t)line * L->output_samples + m] = sum;
        }
    }
    return OR_OK;
}

int or_resample_poly_f32(const float* taps, const or_resample_layout* L, const float* x,
                         int rows, int n, float* out)
{
    /* ft.cpp:2656-2684 */
    for (int line = 0; line < rows; ++line) {
        for (int m = 0; m < L->output_samples; ++m) {
            const long long filtered = ((long long)m + L->output_start) * L->down;
            float sum = 0.0F;
            for (int tap = 0; tap < L->coefficient_count; ++tap) {
                const long long cand = filtered - L->prefix_zeros - tap;
                if (cand % L->up != 0) continue;
                const long long src = cand / L->up;
                if (src < 0 || src >= n) continue;
                sum += taps[tap] * x[(size_t)line * n + (size_t)src];
            }
            out[(size_t)line * L->output_samples + m] = sum;
        }
    }
    return OR_OK;
}

/* ---------------------------------------------------------------- ambgfun */

/* normalized_reference (rt.cpp:30-52): every value divided by the FP64 norm of the whole
 * array; a zero norm gives NaN values. */
static double complex* or_normalized(const float* v, int count)
{
    double sum = 0.0;
    for (int i = 0; i < count; ++i) {
        const double re = (double)v[2 * i], im = (double)v[2 * i + 1];
        sum += re * re + im * im;
    }
    const double norm = sqrt(sum);
    double complex* out = (double complex*)malloc(sizeof(double complex) * (size_t)(count > 0 ? count : 1));
    for (int i = 0; i < count; ++i) {
        if (norm == 0.0) out[i] = CMPLX(NAN, NAN);
        else out[i] = CMPLX((double)v[2 * i] / norm, (double)v[2 * i + 1] / norm);
    }
    return out;
}

/* direct_transform (rt.cpp:54-72): length-point DFT of the first min(n, length) inputs,
 * inverse with the positive exponent and 1/length. */
static double complex* or_direct_transform(const double complex* in, int n, int length, int inverse)
{
    double complex* out = (double complex*)malloc(sizeof(double complex) * (size_t)length);
    const double sign = inverse ? 1.0 : -1.0;
    const double scale = inverse ? 1.0 / (double)length : 1.0;
    for (int f = 0; f < length; ++f) {
        double complex sum = 0.0;
        for (int s = 0; s < n && s < length; ++s) {
            const double angle = sign * 2.0 * kPi * (double)f * (double)s / (double)length;
            sum += in[s] * CMPLX(cos(angle), sin(angle));
        }
        out[f] = sum * scale;
    }
    return out;
}

int or_ambgfun(const float* x, int x_count, int nx, const float* y, int y_count, int ny,
               int cut, double fs, double cut_value, double* out)
{
    if (!y) {
        y = x;
        y_count = x_count;
        ny = nx;
    }
    if (!x || !out || nx < 1 || ny < 1 || nx > x_count || ny > y_count || cut < 0 || cut > 2)
        return OR_INVALID;
    if (cut != 0 && fs == 0.0) return OR_INVALID;
    const int rows = nx + ny - 1;
    int nfreq = 1;
    while (nfreq < rows) nfreq <<= 1;
    double complex* xn = or_normalized(x, x_count);
    double complex* yn = or_normalized(y, y_count);
    if (cut == 0) {
        for (int row = 0; row < rows; ++row) {
            for (int shifted = 0; shifted < nfreq; ++shifted) {
                const int frequency = (shifted - nfreq / 2 + nfreq) % nfreq;
                double complex sum = 0.0;
                for (int column = 0; column < ny; ++column) {
                    const int xc = column - (nx - 1) + row;
                    if (xc < 0 || xc >= nx) continue;
                    const double angle = 2.0 * kPi * (double)frequency * (double)column / (double)nfreq;
                    sum += yn[column] * conj(xn[xc]) * CMPLX(cos(angle), sin(angle));
                }
                out[(size_t)row * nfreq + shifted] = cabs(sum);
            }
        }
    } else if (cut == 1) {
        double complex* xf = or_direct_transform(xn, x_count, nfreq, 0);
        for (int i = 0; i < nfreq; ++i) {
            const double frequency = -fs / 2.0 + fs * (double)i / (double)nfreq;
            const double angle = 2.0 * kPi * frequency * cut_value;
            xf[i] *= CMPLX(cos(angle), sin(angle));
        }
        double complex* xs = or_direct_transform(xf, nfreq, nfreq, 1);
        double complex* prod = (double complex*)calloc((size_t)nfreq, sizeof(double complex));
        for (int i = 0; i < ny && i < nfreq; ++i) prod[i] = yn[i] * conj(xs[i]);
        double complex* tr = or_direct_transform(prod, nfreq, nfreq, 1);
        for (int i = 0; i < nfreq; ++i) out[i] = (double)nfreq * cabs(tr[(i + nfreq / 2) % nfreq]);
        free(xf);
        free(xs);
        free(prod);
        free(tr);
    } else {
        double complex* mod = (double complex*)malloc(sizeof(double complex) * (size_t)x_count);
        for (int i = 0; i < x_count; ++i) mod[i] = xn[i];
        for (int i = 0; i < nx; ++i) {
            const double time = (double)i / fs;
            const double angle = 2.0 * kPi * cut_value * time;
            mod[i] *= CMPLX(cos(angle), sin(angle));
        }
        double complex* yf = or_direct_transform(yn, y_count, rows, 0);
        double complex* xf = or_direct_transform(mod, x_count, rows, 0);
        double complex* prod = (double complex*)malloc(sizeof(double complex) * (size_t)rows);
        for (int i = 0; i < rows; ++i) prod[i] = yf[i] * conj(xf[i]);
        double complex* tr = or_direct_transform(prod, rows, rows, 1);
        for (int i = 0; i < rows; ++i) out[i] = cabs(tr[(i - rows / 2 + rows) % rows]);
        free(mod);
        free(yf);
        free(xf);
        free(prod);
        free(tr);
    }
    free(xn);
    free(yn);
    return OR_OK;
}

/* ------------------------------------------------------------ Task1 echo */

static uint32_t or_task1_hash(uint32_t index, uint32_t seed)
{
    uint32_t v = seed ^ (index * 747796405U + 2891336453U);
    v ^= v >> 16;
    v *= 2246822519U;
    v ^= v >> 13;
    v *= 3266489917U;
    return v ^ (v >> 16);
}

int or_task1_echo(const float* waveform, int L, int P, int N, int delay, double fd, uint32_t seed,
                  double prf, double fs, double amplitude, float noise_std, double* noiseless,
                  float* noise)
{
    if (!waveform || P < 1 || N < 1 || L < 1 || delay < 0 || delay + L > N) return OR_INVALID;
    for (long long e = 0; e < (long long)P * N; ++e) {
        const int p = (int)(e / N), n = (int)(e % N);
        double re = 0.0, im = 0.0;
        const int src = n - delay;
        if (src >= 0 && src < L) {
            const double t = (double)p / prf + (double)n / fs;
            const double ph = 2.0 * kPi * fd * t;
            const double c = cos(ph), s = sin(ph);
            const double wr = waveform[2 * src], wi = waveform[2 * src + 1];
            re = amplitude * (wr * c - wi * s);
            im = amplitude * (wr * s + wi * c);
        }
        if (noiseless) {
            noiseless[2 * e] = re;
            noiseless[2 * e + 1] = im;
        }
        if (noise) {
            const uint32_t k = (uint32_t)(2 * e);
            noise[2 * e] = ((float)(or_task1_hash(k, seed) & 0xffffU) / 32767.5F - 1.0F) * noise_std;
            noise[2 * e + 1] = ((float)(or_task1_hash(k + 1U, seed) & 0xffffU) / 32767.5F - 1.0F) * noise_std;
        }
    }
    return OR_OK;
}

/* ---------------------------------------------------------------- firfilter2 */

/* f rounded to the nearest binary16 value (ties to even; infinity past 65520), as a float. */
static float or_round_half(float f)
{
    if (isnan(f)) return f;
    const float a = fabsf(f);
    if (a >= 65520.0f) return copysignf(INFINITY, f);
    double quantum;
    if (a < 6.103515625e-05f) {
        quantum = ldexp(1.0, -24);            /* subnormal spacing */
    } else {
        int e;
        frexpf(a, &e);                        /* a in [2^(e-1), 2^e): 11 significant bits */
        quantum = ldexp(1.0, e - 11);
    }
    return copysignf((float)(nearbyint((double)a / quantum) * quantum), f);
}

/* filtering_typed.cpp:1597-1620: 2 * endpoint - reflected in the element type. */
static float or_odd_reflect(float endpoint, float reflected, int rounding)
{
    if (rounding == 1) {
        const float doubled = or_round_half(2.0f * endpoint);
        return or_round_half(doubled - reflected);
    }
    if (rounding >= 2 && rounding <= 4) {
        const int bits = rounding == 2 ? 8 : rounding == 3 ? 16 : 32;
        const long long modulus = 1LL << bits, sign = modulus / 2;
        long long v = 2LL * (long long)endpoint - (long long)reflected;
        v %= modulus;
        if (v < 0) v += modulus;
        if (v >= sign) v -= modulus;
        return (float)v;
    }
    const float doubled = 2.0f * endpoint;
    return doubled - reflected;
}

/* One causal pass with the steady-state initial state: out[i] = state[i] * scale (i < nb-1)
 * + sum_k b[k] in[i-k], state[s] = b[s+1] + ... + b[nb-1] (filtering_typed.cpp:1645-1664). */
static void or_fir_steady(const double* b, int nb, const double* state, const double* in, int count,
                          double scale, double* out)
{
    for (int i = 0; i < count; ++i) {
        double v = i < nb - 1 ? state[i] * scale : 0.0;
        for (int k = 0; k < nb; ++k)
            if (i - k >= 0) v += b[k] * in[i - k];
        out[i] = v;
    }
}

int or_firfilter2(const float* b, int nb, const float* x, int lines, int n, int padtype, int has_padlen,
                  int padlen, int rounding, double* out)
{
    if (nb < 1 || padtype < 0 || padtype > 3 || lines < 0 || n < 1) return OR_INVALID;
    int requested = 0;
    if (padtype != 3) requested = has_padlen ? padlen : 3 * nb;
    if (n <= requested) return OR_INVALID;
    const int edge = requested > 0 ? requested : 0;
    const int ne = n + 2 * edge;
    double* bd = malloc(sizeof(double) * nb);
    double* state = malloc(sizeof(double) * (nb > 1 ? nb - 1 : 1));
    double* e = malloc(sizeof(double) * ne);
    double* f = malloc(sizeof(double) * ne);
    double* g = malloc(sizeof(double) * ne);
    if (!bd || !state || !e || !f || !g) {
        free(bd); free(state); free(e); free(f); free(g);
        return OR_INVALID;
    }
    for (int k = 0; k < nb; ++k) bd[k] = b[k];
    double suffix = 0.0;
    for (int s = nb - 2; s >= 0; --s) {
        suffix += bd[s + 1];
        state[s] = suffix;
    }
    for (int line = 0; line < lines; ++line) {
        const float* xl = x + (size_t)line * n;
        for (int i = 0; i < ne; ++i) {
            float v;
            if (i < edge) {
                const float r = xl[edge - i];
                v = padtype == 0 ? or_odd_reflect(xl[0], r, rounding) : padtype == 1 ? r : xl[0];
            } else if (i < edge + n) {
                v = xl[i - edge];
            } else {
                const float r = xl[n - 2 - (i - edge - n)];
                v = padtype == 0 ? or_odd_reflect(xl[n - 1], r, rounding) : padtype == 1 ? r : xl[n - 1];
            }
            e[i] = v;
        }
        or_fir_steady(bd, nb, state, e, ne, e[0], f);
        /* backward pass on the reversed forward output, scaled by its first (= last) value */
        for (int i = 0; i < ne; ++i) e[i] = f[ne - 1 - i];
        or_fir_steady(bd, nb, state, e, ne, e[0], g);
        for (int m = 0; m < n; ++m) out[(size_t)line * n + m] = g[ne - 1 - (edge + m)];
    }
    free(bd); free(state); free(e); free(f); free(g);
    return OR_OK;
}

/* ---------------------------------------------------------------- hilbert */

int or_hilbert(const float* x, int lines, int n, int nfft, double* out)
{
    /* the reference's direct double sums, phase evaluated per term as in
       filtering_typed.cpp:1838-1870 */
    if (lines < 0 || n < 0 || nfft < 1) return OR_INVALID;
    const double two_pi = 6.283185307179586476925286766559;
    double* spec = malloc(sizeof(double) * 2 * nfft);
    if (!spec) return OR_INVALID;
    for (int line = 0; line < lines; ++line) {
        const float* xl = x + (size_t)line * n;
        for (int k = 0; k < nfft; ++k) {
            double re = 0.0, im = 0.0;
            for (int j = 0; j < nfft; ++j) {
                const double value = j < n ? (double)xl[j] : 0.0;
                const double angle = -two_pi * k * j / nfft;
                re += value * cos(angle);
                im += value * sin(angle);
            }
            const double w = (k == 0 || ((nfft % 2) == 0 && k == nfft / 2)) ? 1.0
                           : (k < (nfft + 1) / 2 ? 2.0 : 0.0);
            spec[2 * k] = re * w;
            spec[2 * k + 1] = im * w;
        }
        double* ol = out + (size_t)2 * line * nfft;
        for (int m = 0; m < nfft; ++m) {
            double re = 0.0, im = 0.0;
            for (int k = 0; k < nfft; ++k) {
                const double angle = two_pi * k * m / nfft;
                re += spec[2 * k] * cos(angle) - spec[2 * k + 1] * sin(angle);
                im += spec[2 * k] * sin(angle) + spec[2 * k + 1] * cos(angle);
            }
            ol[2 * m] = re / nfft;
            ol[2 * m + 1] = im / nfft;
        }
    }
    free(spec);
    return OR_OK;
}
