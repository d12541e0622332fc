// Four-step FFT ordering for the fused range-compression kernels (N = 4096, 8192, 16384).
//
// The Stockham plan of fft_core.cuh redistributes the whole transform through shared
// memory between every pair of passes, so each exchange is a block-wide all-to-all with
// two __syncthreads.  Here only the first exchange is block-wide:
//
//   pass 1   thread t holds x[t + T r] (r < E): radix-E DFT over r, times W_N^(t k1);
//            the E outputs k1 go to E groups (one per k1) through shared memory
//            (__syncthreads) -- the remaining work is E independent T-point DFTs;
//   pass 2   group g = k1 is P = T / E consecutive threads of one warp; thread (g, u)
//            holds X1_g[u + P r'] (r' < E): radix-E DFT over r', times W_T^(u k2);
//   pass 3   inside the group (shared memory, __syncwarp only): thread (g, u') takes the
//            E / P sub-transforms k2 = u' + P j and does the radix-P DFT over u.
//
// Register q = j P + k3 of thread (g, u') then holds bin g + E (u' + P j) + E^2 k3
// (digit-reversed order), where the matched filter multiplies by the spectrum, and the
// inverse runs the same steps backwards (conjugate roots), ending with output element
// t + T r in register r -- the natural layout of the load, so stores are coalesced.
// Per pulse the CTA synchronises twice per direction instead of three to four times,
// and the local exchanges of one warp overlap the arithmetic of the others.
//
// The butterflies use scalar complex adds (dft<.., false>), faster here than the packed form.
//
// Shared layout: group g owns E * Q words at g * PITCH (Q = P + 1 words per row of the
// local exchange, an odd pitch that spreads a half-warp's column reads over all banks;
// PITCH keeps the two groups of a half-warp on disjoint banks when P = 8).  The global
// exchange stores element t of group g at g * PITCH + t.  Every access of every phase
// is free of bank conflicts for 64-bit words.
#pragma once

#include "fft_core.cuh"
#include "tcgen05.cuh"

namespace zkx {

template <int N_>
struct LocalPlan {
    static constexpr int N = N_;
    static constexpr int E = elems_for(N);   // radix of passes 1 and 2, values per thread
    static constexpr int T = N / E;          // threads per transform
    static constexpr int P = T / E;          // threads per group = radix of pass 3
    static constexpr int J = E / P;          // pass-3 sub-transforms per thread
    static constexpr int LOGN = ilog2(N);
    static constexpr int LOGT = ilog2(T);
    static constexpr int Q = P + 1;
    static constexpr int PITCH = P == 16 ? E * Q : (E * Q % 16 == 8 ? E * Q : (E * Q / 16) * 16 + 24);
    static constexpr int EXCHANGE = E * PITCH;             // words of the exchange area
    static constexpr int TABLE = P * (E + 1);               // W_T^(u k2), row u at pitch E + 1
    static_assert(P == 8 || P == 16, "three passes with a group of 8 or 16 threads");
    static_assert(E * P * E == N && EXCHANGE >= N, "plan");
};

// True for the lengths the compression kernels run with this ordering.
constexpr bool local_fft_for(int n) { return n == 4096 || n == 8192 || n == 16384; }

// Fill the pass-2 twiddle table: tab[u (E + 1) + k] = W_T^(u k).
template <class LP>
__device__ __forceinline__ void fill_local_table(float2* tab, int t, int nthreads, const float2* __restrict__ tw)
{
    for (int i = t; i < LP::TABLE; i += nthreads) {
        const int u = i / (LP::E + 1), k = i - u * (LP::E + 1);
        const unsigned idx = ((unsigned)(u * k) << (kTwiddleLog - LP::LOGT)) & (kTwiddleSize - 1);
        tab[i] = k < LP::E ? tw[idx] : make_float2(0.f, 0.f);
    }
}

// Forward transform.  In: v[r] = x[t + T r].  Out: v[j P + k3] = X[g + E (u + P j) + E^2 k3]
// with g = t / P, u = t % P.  `twiddle(v)` multiplies v[k] by W_N^(t k) (pass 1), `tab` is the
// pass-2 table.  The caller must __syncthreads before the call if the exchange area was
// read since its last write.
template <class LP, class Twiddle>
__device__ __forceinline__ void local_fft_forward(float2 (&v)[LP::E], float2* sm, int t, Twiddle&& twiddle,
                                                  const float2* tab)
{
    constexpr int E = LP::E, P = LP::P, Q = LP::Q, J = LP::J;
    const int g = t / P, u = t - (t / P) * P;
    float2* region = sm + g * LP::PITCH;
    // pass 1
    dft<E, -1, false>(v);
    twiddle(v);
    static_for<0, E>([&](auto K) {
        constexpr int k = decltype(K)::value;
        sm[k * LP::PITCH + t] = v[k];
    });
    __syncthreads();
    // pass 2
    static_for<0, E>([&](auto R) {
        constexpr int r = decltype(R)::value;
        v[r] = region[u + P * r];
    });
    dft<E, -1, false>(v);
    apply_twiddles_table<E, -1>(v, u, tab);
    __syncwarp();
    static_for<0, E>([&](auto K) {
        constexpr int k = decltype(K)::value;
        region[k * Q + u] = v[k];
    });
    __syncwarp();
    // pass 3
    static_for<0, J>([&](auto JJ) {
        constexpr int j = decltype(JJ)::value;
        float2 z[P];
        static_for<0, P>([&](auto U) { z[decltype(U)::value] = region[(u + P * j) * Q + decltype(U)::value]; });
        dft<P, -1, false>(z);
        static_for<0, P>([&](auto K3) { v[j * P + decltype(K3)::value] = z[decltype(K3)::value]; });
    });
}

// Inverse of local_fft_forward (unnormalised): in the digit-reversed layout, out v[r] at
// element t + T r.  Its first writes go to the rows this thread alone read at the end of
// the forward transform, so none of the group's reads can be overtaken; it ends after the
// block-wide reads of the last exchange, so the caller must __syncthreads before anything
// overwrites the area.  `twiddle_conj(v)` multiplies v[k] by conj(W_N^(t k)).
template <class LP, class Twiddle>
__device__ __forceinline__ void local_fft_inverse(float2 (&v)[LP::E], float2* sm, int t, Twiddle&& twiddle_conj,
                                                  const float2* tab)
{
    constexpr int E = LP::E, P = LP::P, Q = LP::Q, J = LP::J;
    const int g = t / P, u = t - (t / P) * P;
    float2* region = sm + g * LP::PITCH;
    // pass 3 inverse: radix-P over k3, back to the (k2, u) rows
    static_for<0, J>([&](auto JJ) {
        constexpr int j = decltype(JJ)::value;
        float2 z[P];
        static_for<0, P>([&](auto K3) { z[decltype(K3)::value] = v[j * P + decltype(K3)::value]; });
        dft<P, 1, false>(z);
        static_for<0, P>([&](auto U) { region[(u + P * j) * Q + decltype(U)::value] = z[decltype(U)::value]; });
    });
    __syncwarp();
    // pass 2 inverse
    static_for<0, E>([&](auto K) {
        constexpr int k = decltype(K)::value;
        v[k] = region[k * Q + u];
    });
    apply_twiddles_table<E, 1>(v, u, tab);
    dft<E, 1, false>(v);
    __syncwarp();
    static_for<0, E>([&](auto R) {
        constexpr int r = decltype(R)::value;
        region[u + P * r] = v[r];
    });
    __syncthreads();
    // pass 1 inverse
    static_for<0, E>([&](auto K) {
        constexpr int k = decltype(K)::value;
        v[k] = sm[k * LP::PITCH + t];
    });
    twiddle_conj(v);
    dft<E, 1, false>(v);
}

// Spectrum index of register q = j P + k3 of thread t after local_fft_forward.
template <class LP>
__device__ __forceinline__ int local_bin(int t, int q)
{
    const int g = t / LP::P, u = t - g * LP::P;
    const int j = q / LP::P, k3 = q - j * LP::P;
    return g + LP::E * (u + LP::P * j) + LP::E * LP::E * k3;
}

// The spectrum bins a thread's registers hold after local_fft_forward, in register order,
// into its own tensor-memory lane at `cols` (2E consecutive FP32 columns), read once from
// the natural-order spectrum; then tmem_multiply applies them per transform.
template <class LP>
__device__ __forceinline__ void spectrum_to_tmem(const float2* __restrict__ spectrum, int t, uint32_t cols)
{
#pragma unroll
    for (int c = 0; c < 2 * LP::E; c += 16) {
        float sv[16];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const float2 b = __ldg(&spectrum[local_bin<LP>(t, c / 2 + i)]);
            sv[2 * i] = b.x;
            sv[2 * i + 1] = b.y;
        }
        tmem_store16(cols + c, sv);
    }
    tmem_wait_store();
}

// v[k] *= s_k (CONJ: conj(s_k)) with s_k the complex word pair at columns 2k, 2k+1.
template <int E, bool CONJ>
__device__ __forceinline__ void tmem_multiply(float2 (&v)[E], uint32_t cols)
{
#pragma unroll
    for (int c = 0; c < 2 * E; c += 16) {
        float w[16];
        tmem_load16(cols + c, w);
        tmem_wait_load();
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const float2 m = make_float2(w[2 * i], w[2 * i + 1]);
            v[c / 2 + i] = CONJ ? cmulc(v[c / 2 + i], m) : cmul(v[c / 2 + i], m);
        }
    }
}

}  // namespace zkx
