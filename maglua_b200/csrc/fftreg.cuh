// fftreg.cuh -- register-resident FFTs for power-of-two lengths.
//
//  * RegFFT<E, SIGN>: an E-point DFT (E <= 64) held in one thread's registers,
//    natural order in and out, radix-2 decimation in time with compile-time
//    indices; twiddles w_64^k from a constant-memory table.
//  * Four-step line FFT over N = T * E points held by T cooperating lanes of
//    one warp (T a power of two <= 16): lane t holds x[t + T j] (j < E); an
//    E-point DFT per lane, twiddle w_N^{t k1}, an exchange through shared
//    memory, a T-point DFT per (k1) -> lane-owned outputs.
#pragma once
#include "device.cuh"

namespace fr {

// w_64^k = exp(-2 pi i k / 64); one copy per translation unit that includes
// this header, filled by that unit's fftreg_init().
static __constant__ float2 c_w64[64];
static __constant__ double2 c_w64d[64];   // the same in FP64, for double2 lines

template <typename C>
__device__ __forceinline__ C w64(int k, int sign)
{
    const float2 w = c_w64[k & 63];
    C c;
    c.x = w.x;
    c.y = sign > 0 ? -w.y : w.y;
    return c;
}
template <>
__device__ __forceinline__ double2 w64<double2>(int k, int sign)
{
    const double2 w = c_w64d[k & 63];
    return make_double2(w.x, sign > 0 ? -w.y : w.y);
}

template <int E, int SIGN, typename C>
struct RegFFT {
    __device__ __forceinline__ static void run(C* v)
    {
        C ev[E / 2], od[E / 2];
#pragma unroll
        for (int i = 0; i < E / 2; i++) { ev[i] = v[2 * i]; od[i] = v[2 * i + 1]; }
        RegFFT<E / 2, SIGN, C>::run(ev);
        RegFFT<E / 2, SIGN, C>::run(od);
#pragma unroll
        for (int k = 0; k < E / 2; k++) {
            const C t = cmul(od[k], w64<C>(k * (64 / E), SIGN));
            v[k] = cadd(ev[k], t);
            v[k + E / 2] = csub(ev[k], t);
        }
    }
};
template <int SIGN, typename C>
struct RegFFT<1, SIGN, C> {
    __device__ __forceinline__ static void run(C*) {}
};
template <int SIGN, typename C>
struct RegFFT<2, SIGN, C> {
    __device__ __forceinline__ static void run(C* v)
    {
        const C a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    }
};
template <int SIGN, typename C>
struct RegFFT<4, SIGN, C> {
    __device__ __forceinline__ static void run(C* v)
    {
        const C a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
        const C b0 = cadd(v[1], v[3]), b1 = cmul_i(csub(v[1], v[3]), SIGN);
        v[0] = cadd(a0, b0);
        v[2] = csub(a0, b0);
        v[1] = cadd(a1, b1);
        v[3] = csub(a1, b1);
    }
};

// Lane layout of a four-step FFT of N = T * E points.
template <int N>
struct Split {
    // T lanes x E elements; T <= E, both powers of two.
    static constexpr int T = N <= 4 ? 1 : (N <= 32 ? (N <= 8 ? 2 : 4) : (N <= 128 ? 8 : 16));
    static constexpr int E = N / T;
};

// One line of N points in a warp-aligned group of T lanes.
//   in:  v[j] = x[t + T j]
//   out: lane t holds X[k1 + E k2] for k1 in {t, t + T, ...} (E/T values of k1)
//        and k2 < T, in out[q * T + k2] with k1 = t + q T.
// ex is this line's shared-memory exchange buffer of E*(T+1) elements; the lanes
// of the group synchronise with __syncwarp(mask).
template <int N, int SIGN, typename C>
__device__ __forceinline__ void line_fft(C* v, C* ex, int t, unsigned mask, const C* twN)
{
    constexpr int T = Split<N>::T, E = Split<N>::E;
    RegFFT<E, SIGN, C>::run(v);
    if (T > 1) {
#pragma unroll
        for (int k1 = 1; k1 < E; k1++) {
            if (t == 0) continue;
            const int e = (t * k1) & (N - 1);
            C w = twN[e];
            if (SIGN > 0) w.y = -w.y;
            v[k1] = cmul(v[k1], w);
        }
        // exchange: ex[k1 * (T+1) + t] = Y_t[k1] (rows padded against bank conflicts)
#pragma unroll
        for (int k1 = 0; k1 < E; k1++) ex[k1 * (T + 1) + t] = v[k1];
        __syncwarp(mask);
        // lane t takes k1 = t + q T for q < E/T: T-point DFT over the T lanes
#pragma unroll
        for (int q = 0; q < E / T; q++) {
            C u[T];
            const int k1 = t + q * T;
#pragma unroll
            for (int s = 0; s < T; s++) u[s] = ex[k1 * (T + 1) + s];
            RegFFT<T, SIGN, C>::run(u);
#pragma unroll
            for (int k2 = 0; k2 < T; k2++) v[q * T + k2] = u[k2];
        }
        __syncwarp(mask);
    }
}

// Output index of element r of lane t after line_fft: X[k1 + E k2],
// r = q T + k2, k1 = t + q T.
template <int N>
__device__ __forceinline__ int out_index(int t, int r)
{
    constexpr int T = Split<N>::T, E = Split<N>::E;
    if (T == 1) return r;
    const int q = r / T, k2 = r % T;
    return (t + q * T) + E * k2;
}

} // namespace fr

namespace fr {

// ------------------------------------------------------------------ shared-memory Stockham
// Threads per line for a power-of-two length N: N/8 (at most 32), so each
// thread owns two radix-4 butterflies per stage (four at N = 512).
template <int N>
struct Tpl {
    static constexpr int V = N / 8 < 1 ? 1 : (N / 8 > 32 ? 32 : N / 8);
};

// One radix-R Stockham stage (R = 2 or 4) of a line of N points: thread tl
// of the line's TPL threads handles butterflies j = tl + TPL m.  tw is the
// N-entry table exp(-2 pi i k / N) (conjugated for SIGN = +1).  C is float2
// or double2.
template <int N, int R, int NS, int SIGN, int TPL, typename C>
__device__ __forceinline__ void sm_stage(const C* src, C* dst, int tl, const C* tw)
{
    constexpr int NB = N / R;
    constexpr int TWS = N / (NS * R);
#pragma unroll
    for (int m = 0; m < (NB + TPL - 1) / TPL; m++) {
        const int j = tl + TPL * m;
        if (NB % TPL != 0 && j >= NB) break;
        const int jm = j & (NS - 1);
        C v[R];
#pragma unroll
        for (int r = 0; r < R; r++) {
            C x = src[j + r * NB];
            if (NS > 1 && r > 0) {
                C w = tw[(r * jm * TWS) & (N - 1)];
                if (SIGN > 0) w.y = -w.y;
                x = cmul(x, w);
            }
            v[r] = x;
        }
        if (R == 4) RegFFT<4, SIGN, C>::run(v);
        else RegFFT<2, SIGN, C>::run(v);
        const int idxD = (j - jm) * R + jm;
#pragma unroll
        for (int r = 0; r < R; r++) dst[idxD + r * NS] = v[r];
    }
}

// A line's TPL threads are consecutive and TPL divides 32, so every line
// lies inside one warp: a stage only has to synchronise the warp.
template <int N, int SIGN, int TPL, int NS, typename C>
struct SmStages {
    static_assert(TPL <= 32 && 32 % TPL == 0, "a line's threads must lie in one warp");
    // radix-4 while four more points fit, a final radix-2 when log2(N) is odd
    __device__ __forceinline__ static C* run(C* a, C* b, int tl, const C* tw, bool act)
    {
        if (NS * 4 <= N) {
            if (act) sm_stage<N, 4, NS, SIGN, TPL, C>(a, b, tl, tw);
            __syncwarp();
            return SmStages<N, SIGN, TPL, (NS * 4 <= N ? NS * 4 : N), C>::run(b, a, tl, tw, act);
        } else if (NS * 2 <= N) {
            if (act) sm_stage<N, 2, NS, SIGN, TPL, C>(a, b, tl, tw);
            __syncwarp();
            return b;
        }
        return a;
    }
};
template <int N, int SIGN, int TPL, typename C>
struct SmStages<N, SIGN, TPL, N, C> {
    __device__ __forceinline__ static C* run(C* a, C*, int, const C*, bool) { return a; }
};

// Transform line l (data at a + l*LS, scratch at b + l*LS; LS = N or a
// padded line stride) by its TPL threads (tl = thread index within the
// line).  Every thread of the CTA must call this (act = false for threads
// without a line): the stages synchronise the warp, and the CTA is
// synchronised once after the last stage, so the caller may read any line.
// Returns the base (a or b) that holds the result.
template <int N, int SIGN, int TPL, typename C, int LS = N>
__device__ __forceinline__ C* sm_fft(C* a, C* b, int l, int tl, const C* tw, bool act)
{
    C* r = SmStages<N, SIGN, TPL, 1, C>::run(a + (size_t)l * LS, b + (size_t)l * LS, tl, tw, act);
    __syncthreads();
    return r == a + (size_t)l * LS ? a : b;
}

} // namespace fr
