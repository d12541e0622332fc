// Shared-memory FFT machinery for sm_100a.
//
// One transform of length N (a power of two, N <= 16384) is carried by T = N / E
// threads that each hold E complex64 values in registers.  The transform is a
// sequence of Stockham-ordered radix passes: every pass is an in-register radix-E
// DFT (the last pass may use a smaller radix) followed by a twiddle multiply and an
// exchange through shared memory.  Register r of thread t always holds element
// t + T*r both before the first pass and after the last one, so
//   * global loads and stores are coalesced (for fixed r, consecutive t), and
//   * a forward transform can be followed directly by an elementwise product and an
//     inverse transform with no reordering in between (the matched filter).
//
// Shared-memory exchange buffers are padded per pass so that every warp access is
// free of bank conflicts: buffer i (written by pass i, read by pass i+1) inserts
// M_{i+1} pad slots after every M_i elements, where M_i is the sub-transform length
// after pass i.  Callers interleave C independent transforms in one buffer with
// element stride C (C = 1 for row transforms, C = 16 for column transforms).
//
// Twiddles W_M^{n k} come from a device table of exp(-2 pi i j / 65536) generated in
// FP64; per pass a thread loads W^{n}, W^{2n}, W^{4n}, ... and forms the other powers
// by at most four products.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <type_traits>

namespace zkx {

constexpr int kTwiddleLog = 16;
constexpr int kTwiddleSize = 1 << kTwiddleLog;  // exp(-2 pi i j / 65536), j < 65536
constexpr int kMaxSmemFftLog = 14;              // one CTA holds up to 16384 points

// ------------------------------------------------------------------ helpers

template <int I, int N, class F>
__device__ __forceinline__ void static_for(F&& f)
{
    if constexpr (I < N) {
        f(std::integral_constant<int, I>{});
        static_for<I + 1, N>(f);
    }
}

constexpr int ilog2(int n) { return n <= 1 ? 0 : 1 + ilog2(n >> 1); }

constexpr int bit_reverse(int v, int bits)
{
    int r = 0;
    for (int i = 0; i < bits; ++i) r |= ((v >> i) & 1) << (bits - 1 - i);
    return r;
}

#ifndef ZKX_F32X2
#define ZKX_F32X2 1
#endif

#if ZKX_F32X2
// Complex add/sub as one packed FP32x2 instruction (sm_100a add/sub.rn.f32x2): the same
// IEEE round-to-nearest results as two scalar adds, half the issue slots.
__device__ __forceinline__ unsigned long long pack2(float2 a)
{
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
    return r;
}
__device__ __forceinline__ float2 unpack2(unsigned long long r)
{
    float2 a;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(r));
    return a;
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b)
{
    unsigned long long d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pack2(a)), "l"(pack2(b)));
    return unpack2(d);
}
__device__ __forceinline__ float2 csub(float2 a, float2 b)
{
    unsigned long long d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pack2(a)), "l"(pack2(b)));
    return unpack2(d);
}
#else
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
#endif
__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
// a * conj(b)
__device__ __forceinline__ float2 cmulc(float2 a, float2 b)
{
    return make_float2(fmaf(a.x, b.x, a.y * b.y), fmaf(a.y, b.x, -a.x * b.y));
}
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }

// cos(2 pi j / 32) for j = 0..8 (first quadrant of the 32-point circle).
constexpr double kQuarterCos32[9] = {
    1.0,
    0.98078528040323044912618223613424,
    0.92387953251128675612818318939679,
    0.83146961230254523707878837761791,
    0.70710678118654752440084436210485,
    0.55557023301960222474283081394853,
    0.38268343236508977172845998403040,
    0.19509032201612826784828486847702,
    0.0};

constexpr double root_cos32(int j)
{
    j = ((j % 32) + 32) % 32;
    if (j <= 8) return kQuarterCos32[j];
    if (j <= 16) return -kQuarterCos32[16 - j];
    if (j <= 24) return -kQuarterCos32[j - 16];
    return kQuarterCos32[32 - j];
}
constexpr double root_sin32(int j) { return root_cos32(j - 8); }

// a * exp(DIR * 2 pi i * J / 32), DIR = -1 forward, +1 inverse; special angles cost
// no multiplies (multiples of pi/2) or two (odd multiples of pi/4).
template <int J, int DIR>
__device__ __forceinline__ float2 rot32(float2 a)
{
    constexpr int j = ((J % 32) + 32) % 32;
    if constexpr (j == 0) {
        return a;
    } else if constexpr (j == 16) {
        return make_float2(-a.x, -a.y);
    } else if constexpr (j == 8 || j == 24) {
        // exp(+-i pi/2) = sign * i
        constexpr int sgn = (j == 8 ? 1 : -1) * DIR;
        return sgn > 0 ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
    } else if constexpr (j % 8 == 4) {
        constexpr float c = (float)root_cos32(j);
        constexpr float s = (float)(DIR * root_sin32(j));
        constexpr float h = 0.70710678118654752440f;
        constexpr float sc = c > 0 ? 1.0f : -1.0f;
        constexpr float ss = s > 0 ? 1.0f : -1.0f;
        return make_float2((sc * a.x - ss * a.y) * h, (ss * a.x + sc * a.y) * h);
    } else {
        constexpr float c = (float)root_cos32(j);
        constexpr float s = (float)(DIR * root_sin32(j));
        return make_float2(fmaf(a.x, c, -a.y * s), fmaf(a.x, s, a.y * c));
    }
}

// Complex add/sub as two scalar FP32 adds, whatever ZKX_F32X2 says (the same IEEE results).
__device__ __forceinline__ float2 cadd_scalar(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub_scalar(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

// In-register DFT of R points (R | 32): radix-2 decimation in frequency with
// compile-time twiddles, then a static bit-reversal so v[k] = X[k] on return.
// PACKED picks the butterflies' add/sub form: packed f32x2 (cadd/csub) or scalar.  The
// results are identical; which one issues faster depends on the kernel's instruction mix
// (measured: scalar adds make the four-step compression kernel 2.4% faster and the Doppler
// kernel 38% slower).
template <int R, int DIR, bool PACKED = true>
__device__ __forceinline__ void dft(float2* v)
{
    static_assert(R >= 1 && R <= 32 && (R & (R - 1)) == 0, "radix must be a power of two <= 32");
    constexpr int L = ilog2(R);
    static_for<0, L>([&](auto S) {
        constexpr int span = R >> (decltype(S)::value + 1);
        static_for<0, R / (2 * span)>([&](auto B) {
            static_for<0, span>([&](auto J) {
                constexpr int i0 = decltype(B)::value * 2 * span + decltype(J)::value;
                constexpr int i1 = i0 + span;
                const float2 a = v[i0];
                const float2 b = v[i1];
                v[i0] = PACKED ? cadd(a, b) : cadd_scalar(a, b);
                v[i1] = rot32<decltype(J)::value * (32 / (2 * span)), DIR>(PACKED ? csub(a, b) : csub_scalar(a, b));
            });
        });
    });
    if constexpr (R > 2) {
        float2 t[R];
        static_for<0, R>([&](auto K) { t[decltype(K)::value] = v[bit_reverse(decltype(K)::value, L)]; });
        static_for<0, R>([&](auto K) { v[decltype(K)::value] = t[decltype(K)::value]; });
    }
}

// ----------------------------------------------------------------- the plan

// Compile-time description of a length-N transform with E values per thread.
template <int N_, int E_>
struct FftPlan {
    static constexpr int N = N_;
    static constexpr int E = E_ < N_ ? E_ : N_;
    static constexpr int LOGN = ilog2(N);
    static constexpr int LOGE = ilog2(E);
    static constexpr int T = N / E;                            // threads per transform
    static constexpr int PASSES = LOGN == 0 ? 1 : (LOGN + LOGE - 1) / LOGE;
    static constexpr int LAST_LOG = LOGN - (PASSES - 1) * LOGE;  // radix of the last pass
    static constexpr int RLAST = 1 << LAST_LOG;
    // sub-transform length after pass i (i = 0..PASSES); M(0) = N, M(PASSES) = 1
    static constexpr int M(int i) { return i >= PASSES ? 1 : (N >> (LOGE * i)); }
    static constexpr int LOGM(int i) { return i >= PASSES ? 0 : LOGN - LOGE * i; }
    // padded size of exchange buffer i (1 <= i < PASSES)
    static constexpr int buffer_elems(int i) { return N + (N >> LOGM(i)) * M(i + 1); }
    static constexpr int smem_elems(bool pad = true)
    {
        int m = PASSES > 1 ? N : 0;
        for (int i = 1; i < PASSES && pad; ++i) m = buffer_elems(i) > m ? buffer_elems(i) : m;
        return m;
    }
    static_assert((N & (N - 1)) == 0 && N >= 1 && N <= (1 << kMaxSmemFftLog), "N");
    static_assert((E & (E - 1)) == 0 && E >= 1 && E <= 32, "E");
};

// Values per thread for a transform of length N (a plan table chosen so that every
// pass but the last uses the full radix and the thread count stays in 8..512).
#ifndef ZKX_E16384
#define ZKX_E16384 32
#endif
constexpr int elems_for(int n)
{
    return n <= 32 ? n : n == 64 ? 8 : n == 128 ? 16 : n == 256 ? 16 : n == 512 ? 32
         : n == 1024 ? 32 : n == 2048 ? 16 : n == 4096 ? 16 : n == 8192 ? 32 : ZKX_E16384;
}

// Transforms per CTA for row kernels: aim for >= 128 threads per CTA.
constexpr int rows_per_cta(int n)
{
    constexpr int kTarget = 128;
    const int t = n / elems_for(n);
    return t >= kTarget ? 1 : kTarget / t;
}

// Padded position of element addr of exchange buffer I (identity when PAD is false,
// which callers use when the C interleaved transforms already spread every warp
// access over all banks).
template <class PL, int I, bool PAD>
__device__ __forceinline__ int padded(int addr)
{
    if constexpr (PAD) {
        constexpr int lm = PL::LOGM(I);
        constexpr int w = PL::M(I + 1);
        return addr + ((addr >> lm) * w);
    } else {
        return addr;
    }
}

// Multiply v[k] (k = 1..R-1) by W_Mprev^(n k) (conjugated for DIR = +1) using the
// global twiddle table.  Mprev = 1 << LOGMPREV.
template <int R, int DIR, int LOGMPREV>
__device__ __forceinline__ void apply_twiddles(float2* v, int n, const float2* __restrict__ tw)
{
    if constexpr (R > 1) {
        constexpr int LOGR = ilog2(R);
        const unsigned base = (unsigned)n << (kTwiddleLog - LOGMPREV);
        float2 w[R];
        static_for<0, LOGR>([&](auto B) {
            constexpr int p = 1 << decltype(B)::value;
            float2 t = __ldg(&tw[(base * p) & (kTwiddleSize - 1)]);
            w[p] = DIR > 0 ? cconj(t) : t;
        });
        static_for<3, R>([&](auto K) {
            constexpr int k = decltype(K)::value;
            if constexpr ((k & (k - 1)) != 0) {
                constexpr int hi = 1 << ilog2(k);
                w[k] = cmul(w[hi], w[k - hi]);
            }
        });
        static_for<1, R>([&](auto K) { v[decltype(K)::value] = cmul(v[decltype(K)::value], w[decltype(K)::value]); });
    }
}

// The LOGR table entries apply_twiddles reads (W_Mprev^(n p), p = 1, 2, 4, ...), for
// callers that issue these loads early, e.g. while a tile copy is still in flight.
template <int R, int LOGMPREV>
__device__ __forceinline__ void load_twiddle_bases(float2 (&wb)[ilog2(R) > 0 ? ilog2(R) : 1], int n,
                                                   const float2* __restrict__ tw)
{
    const unsigned base = (unsigned)n << (kTwiddleLog - LOGMPREV);
    static_for<0, ilog2(R)>([&](auto B) {
        constexpr int b = decltype(B)::value;
        wb[b] = __ldg(&tw[(base << b) & (kTwiddleSize - 1)]);
    });
}

// apply_twiddles from bases loaded by load_twiddle_bases (the same products, in the
// same order, so the results are bit-identical).
template <int R, int DIR>
__device__ __forceinline__ void apply_twiddles_from(float2* v, const float2* wb)
{
    if constexpr (R > 1) {
        constexpr int LOGR = ilog2(R);
        float2 w[R];
        static_for<0, LOGR>([&](auto B) {
            constexpr int b = decltype(B)::value;
            w[1 << b] = DIR > 0 ? cconj(wb[b]) : wb[b];
        });
        static_for<3, R>([&](auto K) {
            constexpr int k = decltype(K)::value;
            if constexpr ((k & (k - 1)) != 0) {
                constexpr int hi = 1 << ilog2(k);
                w[k] = cmul(w[hi], w[k - hi]);
            }
        });
        static_for<1, R>([&](auto K) { v[decltype(K)::value] = cmul(v[decltype(K)::value], w[decltype(K)::value]); });
    }
}

// The same product with W_Mprev^(n k) read from a per-CTA shared table tab[n (R + 1) + k]
// (n < M of the pass; the odd row pitch keeps the lanes' reads on distinct banks).
template <int R, int DIR>
__device__ __forceinline__ void apply_twiddles_table(float2* v, int n, const float2* tab)
{
    const float2* row = tab + n * (R + 1);
    static_for<1, R>([&](auto K) {
        constexpr int k = decltype(K)::value;
        float2 w = row[k];
        if constexpr (DIR > 0) w = cconj(w);
        v[k] = cmul(v[k], w);
    });
}

// Rows n < PL::M(2) of the table apply_twiddles_table reads in the second pass of a
// three-pass plan: tab[n (E + 1) + k] = W_M(1)^(n k).  Callers size it mid_table_elems().
template <class PL>
constexpr int mid_table_elems() { return PL::PASSES == 3 ? PL::M(2) * (PL::E + 1) : 0; }

template <class PL>
__device__ __forceinline__ void fill_mid_table(float2* tab, int t, int nthreads, const float2* __restrict__ tw)
{
    constexpr int P = PL::E + 1;
    for (int i = t; i < mid_table_elems<PL>(); i += nthreads) {
        const int n = i / P, k = i - n * P;
        const unsigned idx = ((unsigned)(n * k) << (kTwiddleLog - PL::LOGM(1))) & (kTwiddleSize - 1);
        tab[i] = k < PL::E ? tw[idx] : make_float2(0.f, 0.f);
    }
}

// One transform of length PL::N.  On entry v[r] holds element t + T*r, on exit
// v[r] holds output bin t + T*r.  sm points at this transform's exchange buffer;
// element a of the buffer lives at sm[a * C].  The caller must __syncthreads()
// between two consecutive transforms that share sm.  All threads of the block
// must call this (it synchronises the block).
template <class PL, int DIR, int C, bool PAD = true>
__device__ __forceinline__ void fft_block(float2 (&v)[PL::E], float2* sm, int t,
                                          const float2* __restrict__ tw, const float2* mid = nullptr,
                                          const float2* first = nullptr)
{
    constexpr int E = PL::E;
    constexpr int T = PL::T;
    if constexpr (PL::PASSES == 1) {
        dft<E, DIR>(v);
        return;
    } else {
        // pass 1: n = t, s = 0, radix E, twiddle W_N^(t k) (bases preloaded in `first`
        // by load_twiddle_bases<E, PL::LOGN>(first, t, tw) when the caller has them)
        dft<E, DIR>(v);
        if (first != nullptr)
            apply_twiddles_from<E, DIR>(v, first);
        else
            apply_twiddles<E, DIR, PL::LOGN>(v, t, tw);
        static_for<0, E>([&](auto K) {
            constexpr int k = decltype(K)::value;
            sm[padded<PL, 1, PAD>(k * PL::M(1) + t) * C] = v[k];
        });
        __syncthreads();
        // middle passes 2 .. PASSES-1 (radix E)
        static_for<2, PL::PASSES>([&](auto IP) {
            constexpr int i = decltype(IP)::value;
            constexpr int Mi = PL::M(i);
            constexpr int Mprev = PL::M(i - 1);
            constexpr int Pprev = PL::N / Mprev;
            const int s = t >> PL::LOGM(i);
            const int n = t & (Mi - 1);
            static_for<0, E>([&](auto K) {
                constexpr int k = decltype(K)::value;
                v[k] = sm[padded<PL, i - 1, PAD>(s * Mprev + k * Mi + n) * C];
            });
            __syncthreads();
            dft<E, DIR>(v);
            if (i == 2 && mid != nullptr)
                apply_twiddles_table<E, DIR>(v, n, mid);
            else
                apply_twiddles<E, DIR, PL::LOGM(i - 1)>(v, n, tw);
            static_for<0, E>([&](auto K) {
                constexpr int k = decltype(K)::value;
                sm[padded<PL, i, PAD>((s + Pprev * k) * Mi + n) * C] = v[k];
            });
            __syncthreads();
        });
        // last pass: radix RLAST, each thread owns J = E / RLAST sub-transforms
        constexpr int R = PL::RLAST;
        constexpr int J = E / R;
        constexpr int LP = PL::PASSES - 1;  // buffer index read by the last pass
        float2 u[J][R];
        static_for<0, J>([&](auto JJ) {
            constexpr int j = decltype(JJ)::value;
            const int sj = t + j * T;
            static_for<0, R>([&](auto K) {
                constexpr int k = decltype(K)::value;
                u[j][k] = sm[padded<PL, LP, PAD>(sj * R + k) * C];
            });
        });
        static_for<0, J>([&](auto JJ) { dft<R, DIR>(u[decltype(JJ)::value]); });
        static_for<0, J>([&](auto JJ) {
            static_for<0, R>([&](auto K) {
                v[decltype(JJ)::value + J * decltype(K)::value] = u[decltype(JJ)::value][decltype(K)::value];
            });
        });
    }
}

}  // namespace zkx
