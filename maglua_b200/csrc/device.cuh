// device.cuh -- device-side building blocks shared by every kernel:
//   * Philox4x32-10 counter-based RNG (Salmon, Moraes, Dror, Shaw, SC'11)
//     and a Box-Muller transform to normals;
//   * a CTA-cooperative mixed-radix Stockham FFT over lines held in shared
//     memory (any length whose factors are small; radix 2/3/4/5/8 fast
//     paths, direct DFT for other primes);
//   * small complex helpers.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

// Programmatic dependent launch (kernels launched with launch_pdl): a kernel
// may be scheduled while the previous kernel of its stream finishes.
// pdl_wait() returns once that kernel has completed and its writes are
// visible; nothing a predecessor writes may be read before it.
// pdl_trigger() lets the next kernel be scheduled.  Both are no-ops for a
// kernel launched without the attribute.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Device timeline stamps (%globaltimer, ns): slot t[0] takes the earliest
// start over the CTAs that call tl_start, t[1] the latest end over those
// that call tl_end (after the CTA's last store).  No-ops for a null t.
__device__ __forceinline__ unsigned long long gtimer_ns()
{
    unsigned long long v;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(v));
    return v;
}
__device__ __forceinline__ void tl_start(unsigned long long* t)
{
    if (t && threadIdx.x == 0) atomicMin(t, gtimer_ns());
}
__device__ __forceinline__ void tl_end(unsigned long long* t)
{
    if (t) {
        __syncthreads();
        if (threadIdx.x == 0) atomicMax(t + 1, gtimer_ns());
    }
}

#ifndef MLB_HD
#define MLB_HD __host__ __device__ __forceinline__
#endif

// --------------------------------------------------------------- Philox
// Philox4x32 with 10 rounds.  Multipliers and Weyl key increments are the
// published ones (Salmon et al. 2011, Table 2).
struct Philox4 { uint32_t v[4]; };

MLB_HD uint32_t mlb_mulhi32(uint32_t a, uint32_t b)
{
#ifdef __CUDA_ARCH__
    return __umulhi(a, b);
#else
    return (uint32_t)(((uint64_t)a * (uint64_t)b) >> 32);
#endif
}

MLB_HD Philox4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                             uint32_t k0, uint32_t k1)
{
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; r++) {
        if (r > 0) { k0 += W0; k1 += W1; }
        const uint32_t hi0 = mlb_mulhi32(M0, c0), lo0 = M0 * c0;
        const uint32_t hi1 = mlb_mulhi32(M1, c2), lo1 = M1 * c2;
        const uint32_t n0 = hi1 ^ c1 ^ k0;
        const uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    }
    Philox4 o;
    o.v[0] = c0; o.v[1] = c1; o.v[2] = c2; o.v[3] = c3;
    return o;
}

// Three standard normals for (site, counter) under a 64-bit seed.
// Counter words: (site, counter lo, counter hi, stream tag).
__device__ __forceinline__ float3 philox_normal3(uint64_t seed, uint64_t counter, uint32_t site,
                                                 uint32_t tag)
{
    Philox4 r = philox4x32_10(site, (uint32_t)counter, (uint32_t)(counter >> 32), tag,
                              (uint32_t)seed, (uint32_t)(seed >> 32));
    // uniforms in (0,1): 24 high bits plus half an ulp
    const float s24 = 5.9604644775390625e-08f; // 2^-24
    const float u0 = ((float)(r.v[0] >> 8) + 0.5f) * s24;
    const float u1 = ((float)(r.v[1] >> 8) + 0.5f) * s24;
    const float u2 = ((float)(r.v[2] >> 8) + 0.5f) * s24;
    const float u3 = ((float)(r.v[3] >> 8) + 0.5f) * s24;
    // Box-Muller with the hardware log/sin/cos approximations (absolute
    // error ~1e-6 of the unit-variance normal; the noise is statistical)
    const float ra = sqrtf(-2.0f * __logf(u0));
    const float rb = sqrtf(-2.0f * __logf(u2));
    float sa, ca;
    __sincosf(6.283185307179586f * u1, &sa, &ca);
    const float cb = __cosf(6.283185307179586f * u3);
    return make_float3(ra * ca, ra * sa, rb * cb);
}

// --------------------------------------------------------------- complex
template <typename R> struct CT;
template <> struct CT<float> { typedef float2 T; };
template <> struct CT<double> { typedef double2 T; };

template <typename C> __device__ __forceinline__ C cmk(decltype(C().x) a, decltype(C().x) b)
{
    C c; c.x = a; c.y = b; return c;
}
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return cmk<C>(a.x + b.x, a.y + b.y); }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return cmk<C>(a.x - b.x, a.y - b.y); }
template <typename C> __device__ __forceinline__ C cmul(C a, C b)
{
    return cmk<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename C> __device__ __forceinline__ C cconj(C a) { return cmk<C>(a.x, -a.y); }
// multiply by -i*sign... : returns a * (sign * i) for sign in {+1,-1}
template <typename C> __device__ __forceinline__ C cmul_i(C a, int sign)
{
    return sign > 0 ? cmk<C>(-a.y, a.x) : cmk<C>(a.y, -a.x);
}

// --------------------------------------------------------------- FFT plan
// A length-N plan: radices in stage order and the offset of its N-entry
// twiddle table tw[k] = exp(-2 pi i k / N) inside a shared pool.
#define MLB_FFT_MAX_STAGES 16
struct FftLen {
    int n;
    int nst;
    int radix[MLB_FFT_MAX_STAGES];
    int tw_off;
};

// Line geometry inside a shared-memory buffer: line l starts at
// (l / lpg) * gstride + (l % lpg) * ls and its elements are es apart.
struct LineGeo {
    int nlines, lpg, gstride, ls, es;
    int line_fast; // 1: consecutive threads take consecutive lines
};

__device__ __forceinline__ int geo_base(const LineGeo& g, int l)
{
    return (l / g.lpg) * g.gstride + (l % g.lpg) * g.ls;
}

template <typename C>
__device__ __forceinline__ C tw_get(const C* tw, int e, int sign)
{
    C w = tw[e];
    return sign > 0 ? cconj(w) : w;
}

// In-register DFT of R points, w_R = exp(sign*2 pi i/R).
template <typename C, int R>
__device__ __forceinline__ void dft_small(C* v, int sign, const C* tw, int N)
{
    if (R == 2) {
        C a = v[0], b = v[1];
        v[0] = cadd(a, b); v[1] = csub(a, b);
    } else if (R == 4) {
        C a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
        C b0 = cadd(v[1], v[3]), b1 = cmul_i(csub(v[1], v[3]), sign);
        v[0] = cadd(a0, b0); v[2] = csub(a0, b0);
        v[1] = cadd(a1, b1); v[3] = csub(a1, b1);
    } else if (R == 8) {
        typedef decltype(C().x) Rl;
        const Rl h = (Rl)0.70710678118654752440;
        // radix-2 on pairs (0,4),(1,5),(2,6),(3,7), twiddle, then radix-4 on each half
        C e[4], o[4];
#pragma unroll
        for (int k = 0; k < 4; k++) { e[k] = cadd(v[k], v[k + 4]); o[k] = csub(v[k], v[k + 4]); }
        // o[k] *= w8^k
        o[1] = cmk<C>((o[1].x - (Rl)sign * o[1].y) * h, (o[1].y + (Rl)sign * o[1].x) * h);
        o[2] = cmul_i(o[2], sign);
        o[3] = cmk<C>((-o[3].x - (Rl)sign * o[3].y) * h, (-o[3].y + (Rl)sign * o[3].x) * h);
        dft_small<C, 4>(e, sign, tw, N);
        dft_small<C, 4>(o, sign, tw, N);
        v[0] = e[0]; v[2] = e[1]; v[4] = e[2]; v[6] = e[3];
        v[1] = o[0]; v[3] = o[1]; v[5] = o[2]; v[7] = o[3];
    } else if (R == 3) {
        typedef decltype(C().x) Rl;
        const Rl c1 = (Rl)-0.5, s1 = (Rl)0.86602540378443864676 * (Rl)sign;
        C t = cadd(v[1], v[2]);
        C d = csub(v[1], v[2]);
        C m = cmk<C>(v[0].x + c1 * t.x, v[0].y + c1 * t.y);
        C r = cmk<C>(-s1 * d.y, s1 * d.x);
        v[0] = cadd(v[0], t);
        v[1] = cadd(m, r);
        v[2] = csub(m, r);
    } else {
        // generic direct DFT using the plan's twiddle table (w_R^m = tw[m*N/R])
        C o[R];
#pragma unroll
        for (int k = 0; k < R; k++) {
            C acc = v[0];
#pragma unroll
            for (int r = 1; r < R; r++) {
                const int m = (r * k) % R;
                acc = cadd(acc, cmul(v[r], tw_get(tw, m * (N / R), sign)));
            }
            o[k] = acc;
        }
#pragma unroll
        for (int k = 0; k < R; k++) v[k] = o[k];
    }
}

template <typename C, int R>
__device__ __forceinline__ void stockham_stage(const C* src, C* dst, const LineGeo& g, int N,
                                               int Ns, int sign, const C* tw)
{
    const int nb = N / R;               // butterflies per line
    const int total = g.nlines * nb;
    const int stride_tw = N / (Ns * R);
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
        int l, j;
        if (g.line_fast) { l = t % g.nlines; j = t / g.nlines; }
        else { j = t % nb; l = t / nb; }
        const int base = geo_base(g, l);
        const int jm = j % Ns;
        C v[R];
#pragma unroll
        for (int r = 0; r < R; r++) {
            C x = src[base + (j + r * nb) * g.es];
            if (r > 0 && jm > 0) x = cmul(x, tw_get(tw, (r * jm * stride_tw) % N, sign));
            v[r] = x;
        }
        dft_small<C, R>(v, sign, tw, N);
        const int idxD = (j / Ns) * Ns * R + jm;
#pragma unroll
        for (int r = 0; r < R; r++) dst[base + (idxD + r * Ns) * g.es] = v[r];
    }
}

// Generic-radix stage for primes without a fast path (R <= 32).
template <typename C>
__device__ void stockham_stage_gen(const C* src, C* dst, const LineGeo& g, int N, int R, int Ns,
                                   int sign, const C* tw)
{
    const int nb = N / R;
    const int total = g.nlines * nb;
    const int stride_tw = N / (Ns * R);
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
        int l, j;
        if (g.line_fast) { l = t % g.nlines; j = t / g.nlines; }
        else { j = t % nb; l = t / nb; }
        const int base = geo_base(g, l);
        const int jm = j % Ns;
        const int idxD = (j / Ns) * Ns * R + jm;
        for (int k = 0; k < R; k++) {
            C acc = cmk<C>(0, 0);
            for (int r = 0; r < R; r++) {
                C x = src[base + (j + r * nb) * g.es];
                const long long e = (long long)r * jm * stride_tw + (long long)((r * k) % R) * (N / R);
                acc = cadd(acc, cmul(x, tw_get(tw, (int)(e % N), sign)));
            }
            dst[base + (idxD + k * Ns) * g.es] = acc;
        }
    }
}

// Transform every line described by g.  Data starts in a; b is scratch with
// the same layout.  Returns the buffer that holds the result.  All threads
// of the CTA must call it; it synchronises internally and on return.
template <typename C>
__device__ C* cta_fft(C* a, C* b, const LineGeo& g, const FftLen& L, const C* tw_pool, int sign)
{
    const C* tw = tw_pool + L.tw_off;
    C* src = a;
    C* dst = b;
    int Ns = 1;
    for (int s = 0; s < L.nst; s++) {
        const int R = L.radix[s];
        switch (R) {
        case 2: stockham_stage<C, 2>(src, dst, g, L.n, Ns, sign, tw); break;
        case 3: stockham_stage<C, 3>(src, dst, g, L.n, Ns, sign, tw); break;
        case 4: stockham_stage<C, 4>(src, dst, g, L.n, Ns, sign, tw); break;
        case 5: stockham_stage<C, 5>(src, dst, g, L.n, Ns, sign, tw); break;
        case 7: stockham_stage<C, 7>(src, dst, g, L.n, Ns, sign, tw); break;
        case 8: stockham_stage<C, 8>(src, dst, g, L.n, Ns, sign, tw); break;
        default: stockham_stage_gen<C>(src, dst, g, L.n, R, Ns, sign, tw); break;
        }
        __syncthreads();
        Ns *= R;
        C* t = const_cast<C*>(src);
        src = dst;
        dst = t;
    }
    return const_cast<C*>(src);
}
