// conv_fast.cu -- fast path of the dipole convolution and of the fused step
// for power-of-two padded grids (16..512 in x and y, 1..32 in z).
//
//   k_fx_fast<PX>      R2C along x: two real rows packed into one complex
//                      line, register four-step FFT, split, coalesced store
//                      to SPEC[kx][c][z][y].
//   k_yz_fast<PY,PZ>   per kx: y FFT (register four-step) of the data rows,
//                      z FFT + real-symmetric tensor multiply + inverse z FFT
//                      in one thread's registers per ky, inverse y FFT.
//   k_ix_fast<PX>      C2R along x: two rows per complex line.
//   k_fused_fast<...>  field terms + LLG for uniform-parameter systems with
//                      a six-neighbour stencil, no integer division and
//                      host-folded constants.
#include "device.cuh"
#include "fftreg.cuh"
#include "fused.cuh"
#include "kparams.h"
#include "launch.h"

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>

namespace mlb {

cudaError_t fftreg_init()
{
    float2 h[64];
    double2 hd[64];
    for (int k = 0; k < 64; k++) {
        const double a = 2.0 * M_PI * k / 64.0;
        h[k] = make_float2((float)cos(a), (float)(-sin(a)));
        hd[k] = make_double2(cos(a), -sin(a));
    }
    cudaError_t e = cudaMemcpyToSymbol(fr::c_w64, h, sizeof(h));
    if (e != cudaSuccess) return e;
    return cudaMemcpyToSymbol(fr::c_w64d, hd, sizeof(hd));
}

} // namespace mlb

using fr::Split;

// ------------------------------------------------------------------ x passes
// A CTA of 256 threads transforms L = 256/TPL complex lines; line l packs
// rows (row0 + 2l, row0 + 2l + 1) of one component as real and imaginary
// parts, rows counted over the flattened (z, y) index r = z ny + y (SPEC is
// contiguous in r), so small layers fill a CTA.  Global loads are gathered into registers in unrolled
// batches before they are written to shared memory, so each thread has all
// its loads in flight at once.
template <int PX>
struct XCfg {
    static constexpr int NT = 256;
    static constexpr int TPL = fr::Tpl<PX>::V;
    static constexpr int L = NT / TPL;
    static constexpr int ROWS = 2 * L;
    static constexpr int KX = PX / 2 + 1;
    static constexpr int LINE = L * PX;                        // line buffer
    static constexpr int SPEC = ROWS * KX;                     // [ROWS][KX] staging
    static constexpr int BUF = LINE > SPEC ? LINE : SPEC;      // each of A, B
    // FP32 lines of 32 to 256 points use the register four-step
    // transform, with one exchange buffer per line after the two line buffers
    static constexpr int EX = (PX >= 32 && PX <= 256) ? L * fr::Split<PX>::E * (fr::Split<PX>::T + 1) : 0;
    static constexpr int SMEM = (PX + 2 * BUF + EX) * 8;       // bytes (FP32)
    static constexpr int SMEM_D = (PX + 2 * BUF) * 16;         // bytes (FP64)
};

// FP32 x lines of 32 to 256 points: the four-step register FFT of
// fr::line_fft (Split<N>::T lanes x Split<N>::E points, one warp-synchronous
// exchange through ex, E (T + 1) elements per line), in place on a
// natural-order line: the lanes have read the whole line before any of them
// writes it back.
template <int N>
struct XReg {
    static constexpr bool OK = N >= 32 && N <= 256;
    static constexpr int T = fr::Split<N>::T, E = fr::Split<N>::E, EX = E * (T + 1);
};
template <int N, int SIGN>
__device__ __forceinline__ void xreg_line(float2* line, float2* ex, int t, unsigned mask, const float2* tw)
{
    constexpr int T = XReg<N>::T, E = XReg<N>::E;
    float2 v[E];
#pragma unroll
    for (int j = 0; j < E; j++) v[j] = line[t + T * j];
    fr::line_fft<N, SIGN, float2>(v, ex, t, mask, tw);
#pragma unroll
    for (int r = 0; r < E; r++) line[fr::out_index<N>(t, r)] = v[r];
}

// The CTA's nl lines (line l at base + l ls) in place, line l by threads
// T l .. T l + T - 1.  Every thread of the CTA calls this; the CTA is
// synchronised after the transforms.
template <int N, int SIGN>
__device__ __forceinline__ void xreg_lines(float2* base, int ls, int nl, float2* ex, const float2* tw)
{
    constexpr int T = XReg<N>::T;
    const int l = threadIdx.x / T, t = threadIdx.x % T;
    if (l < nl) {
        const unsigned mask = ((1u << T) - 1u) << ((threadIdx.x & 31) & ~(T - 1));
        xreg_line<N, SIGN>(base + (size_t)l * ls, ex + (size_t)l * XReg<N>::EX, t, mask, tw);
    }
    __syncthreads();
}

// R = float or double (state precision), C the matching complex type.
template <int PX, typename R = float>
__global__ void __launch_bounds__(256) k_fx_fast(ConvK c, const typename CT<R>::T* __restrict__ tw,
                                                 const R* __restrict__ sx, const R* __restrict__ sy,
                                                 const R* __restrict__ sz, typename CT<R>::T* __restrict__ spec)
{
    typedef typename CT<R>::T C;
    pdl_trigger();
    pdl_wait();
    if (c.run_if && *c.run_if == 0) return;
    using X = XCfg<PX>;
    constexpr int NT = X::NT;
    extern __shared__ __align__(16) unsigned char smraw_fx[];
    C* twl = reinterpret_cast<C*>(smraw_fx);   // [PX]
    C* A = twl + PX;                           // [L][PX]
    C* B = A + X::BUF;                         // [L][PX]
    const int comp = blockIdx.z % 3, rep = blockIdx.z / 3;
    const int nr = c.nz * c.ny;                 // rows (z, y) of one component, flattened
    const int row0 = blockIdx.x * X::ROWS;
    const size_t nsite = (size_t)c.nx * c.ny * c.nz;
    spec += (size_t)rep * c.Kx * 3 * nr;
    const R* src = (comp == 0 ? sx : (comp == 1 ? sy : sz)) + rep * nsite;
    for (int k = threadIdx.x; k < PX; k += NT) twl[k] = tw[k];
    constexpr int IT = (X::LINE + NT - 1) / NT;
    C v[IT];
#pragma unroll
    for (int it = 0; it < IT; it++) {
        const int idx = threadIdx.x + it * NT;
        const int l = idx / PX, x = idx % PX;
        const int ya = row0 + 2 * l, yb = ya + 1;
        R a = 0, b = 0;
        if (idx < X::LINE && x < c.nx) {
            if (ya < nr) a = __ldg(src + (size_t)ya * c.nx + x);
            if (yb < nr) b = __ldg(src + (size_t)yb * c.nx + x);
        }
        v[it] = cmk<C>(a, b);
    }
#pragma unroll
    for (int it = 0; it < IT; it++) {
        const int idx = threadIdx.x + it * NT;
        if (idx < X::LINE) A[idx] = v[it];
    }
    __syncthreads();
    const C* Rl;
    if constexpr (XReg<PX>::OK && sizeof(R) == 4) {
        xreg_lines<PX, -1>(A, PX, X::L, B + X::BUF, twl);
        Rl = A;
    } else {
        const int l = threadIdx.x / X::TPL, tl = threadIdx.x % X::TPL;
        Rl = fr::sm_fft<PX, -1, X::TPL>(A, B, l, tl, twl, true);
    }
    // split the two real rows and store SPEC[kx][comp][row] (row = z ny + y)
    const int rows_here = min(X::ROWS, nr - row0);
    constexpr int IS = (X::SPEC + NT - 1) / NT;
#pragma unroll
    for (int it = 0; it < IS; it++) {
        const int idx = threadIdx.x + it * NT;
        const int kx = idx / X::ROWS, row = idx % X::ROWS;
        if (idx >= X::SPEC || row >= rows_here) continue;
        const C* Z = Rl + (row >> 1) * PX;
        const C zk = Z[kx], zn = Z[(PX - kx) & (PX - 1)];
        C o;
        if ((row & 1) == 0) o = cmk<C>((R)0.5 * (zk.x + zn.x), (R)0.5 * (zk.y - zn.y));
        else o = cmk<C>((R)0.5 * (zk.y + zn.y), (R)0.5 * (zn.x - zk.x));
        spec[((size_t)kx * 3 + comp) * nr + row0 + row] = o;
    }
}

template <int PX, typename R = float>
__global__ void __launch_bounds__(256) k_ix_fast(ConvK c, const typename CT<R>::T* __restrict__ tw,
                                                 const typename CT<R>::T* __restrict__ spec, R* __restrict__ hx,
                                                 R* __restrict__ hy, R* __restrict__ hz)
{
    typedef typename CT<R>::T C;
    pdl_trigger();
    pdl_wait();
    if (c.run_if && *c.run_if == 0) return;
    using X = XCfg<PX>;
    constexpr int KX = X::KX, NT = X::NT;
    extern __shared__ __align__(16) unsigned char smraw_ix[];
    C* twl = reinterpret_cast<C*>(smraw_ix);   // [PX]
    C* A = twl + PX;                           // [L][PX] lines
    C* B = A + X::BUF;                         // [ROWS][KX] spectra, then scratch
    const int comp = blockIdx.z % 3, rep = blockIdx.z / 3;
    const int nr = c.nz * c.ny;                 // rows (z, y) of one component, flattened
    const int row0 = blockIdx.x * X::ROWS;
    const int rows_here = min(X::ROWS, nr - row0);
    const size_t nsite = (size_t)c.nx * c.ny * c.nz;
    spec += (size_t)rep * c.Kx * 3 * nr;
    R* dst = (comp == 0 ? hx : (comp == 1 ? hy : hz)) + rep * nsite;
    for (int k = threadIdx.x; k < PX; k += NT) twl[k] = tw[k];
    constexpr int IS = (X::SPEC + NT - 1) / NT;
    {
        C v[IS];
#pragma unroll
        for (int it = 0; it < IS; it++) {
            const int idx = threadIdx.x + it * NT;
            const int kx = idx / X::ROWS, row = idx % X::ROWS;
            v[it] = cmk<C>(0, 0);
            if (idx < X::SPEC && row < rows_here)
                v[it] = spec[((size_t)kx * 3 + comp) * nr + row0 + row];
        }
#pragma unroll
        for (int it = 0; it < IS; it++) {
            const int idx = threadIdx.x + it * NT;
            const int kx = idx / X::ROWS, row = idx % X::ROWS;
            if (idx < X::SPEC) B[row * KX + kx] = v[it];
        }
    }
    __syncthreads();
    // line l: Z[k] = S_row(2l)[k] + i S_row(2l+1)[k] with Hermitian completion
    constexpr int IL = (X::LINE + NT - 1) / NT;
#pragma unroll
    for (int it = 0; it < IL; it++) {
        const int idx = threadIdx.x + it * NT;
        if (idx >= X::LINE) continue;
        const int l = idx / PX, k = idx % PX;
        const C* Sa = B + (2 * l) * KX;
        const C* Sb = B + (2 * l + 1) * KX;
        C a, b;
        if (k < KX) { a = Sa[k]; b = Sb[k]; }
        else { a = cconj(Sa[PX - k]); b = cconj(Sb[PX - k]); }
        A[idx] = cmk<C>(a.x - b.y, a.y + b.x);
    }
    __syncthreads();
    const C* Rl;
    if constexpr (XReg<PX>::OK && sizeof(R) == 4) {
        xreg_lines<PX, +1>(A, PX, X::L, B + X::BUF, twl);
        Rl = A;
    } else {
        const int l = threadIdx.x / X::TPL, tl = threadIdx.x % X::TPL;
        Rl = fr::sm_fft<PX, +1, X::TPL>(A, B, l, tl, twl, true);
    }
    constexpr int IO = (X::ROWS * PX + NT - 1) / NT;
#pragma unroll
    for (int it = 0; it < IO; it++) {
        const int idx = threadIdx.x + it * NT;
        const int row = idx / PX, x = idx % PX;
        if (idx >= X::ROWS * PX || row >= rows_here || x >= c.nx) continue;
        const C z = Rl[(row >> 1) * PX + x];
        dst[(size_t)(row0 + row) * c.nx + x] = (row & 1) ? z.y : z.x;
    }
}

// ------------------------------------------------------------------ (y,z) pass
// One CTA per kx.  y transforms of the 3*nz data lines by TPL threads each
// (in rounds), z transforms + tensor multiply with one thread per
// (component, ky) column, inverse y transforms.
// threads per CTA: 768 for the planes of a large film (one CTA per SM), 384
// when the z columns are 32 long (registers), 256 for planes up to 128 wide
// (many small replicas: several CTAs per SM)
template <int PY, int PZ>
struct YZT {
    static constexpr int N = PY <= 128 ? 256 : (PZ >= 32 ? 384 : 768);
    static constexpr int MINB = PY <= 128 ? 3 : 1;
};

template <int PY, int PZ>
__global__ void __launch_bounds__(YZT<PY, PZ>::N, YZT<PY, PZ>::MINB) k_yz_fast(ConvK c, const float2* __restrict__ twy,
                                                               float2* __restrict__ spec, const float* __restrict__ ten6)
{
    constexpr int NT = YZT<PY, PZ>::N;
    constexpr int TPL = fr::Tpl<PY>::V;
    constexpr int LPR = NT / TPL;    // lines per round
    extern __shared__ float2 sm[];
    const int kx = blockIdx.x;
    const int nz = c.nz, ny = c.ny;
    const int nlines = 3 * nz;
    spec += (size_t)blockIdx.y * c.Kx * 3 * nz * ny;
    float2* P = sm;                          // [3][nz][PY]
    float2* Pb = P + (size_t)nlines * PY;    // scratch [3][nz][PY]
    float2* Q = Pb + (size_t)nlines * PY;    // [3][PZ][PY]
    float2* twl = Q + (size_t)3 * PZ * PY;   // [PY]
    const float* Tk = ten6 + (size_t)kx * PZ * PY * 6;
    // the tensor and twiddles are constants of the plan: fetch them while
    // the previous kernel finishes
    if (threadIdx.x == 0) {
        // pull this kx's tensor chunk into L2 while the y transforms run
        const unsigned bytes = (unsigned)(PZ * PY * 6 * sizeof(float));
        if ((((uintptr_t)Tk) & 15) == 0 && (bytes & 15) == 0)
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(Tk), "r"(bytes) : "memory");
    }
    for (int k = threadIdx.x; k < PY; k += blockDim.x) twl[k] = twy[k];
    pdl_trigger();
    pdl_wait();
    tl_start(c.tl);
    if (c.run_if && *c.run_if == 0) return;
    float2* sp = spec + (size_t)kx * nlines * ny;
    {
        // at most 3*PZ*PY elements (nz <= PZ): unrolled gather, then store
        constexpr int IG = (3 * PZ * PY + NT - 1) / NT;
        float2 v[IG];
#pragma unroll
        for (int it = 0; it < IG; it++) {
            const int idx = threadIdx.x + it * NT;
            const int l = idx / PY, y = idx % PY;
            v[it] = (l < nlines && y < ny) ? sp[(size_t)l * ny + y] : make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int it = 0; it < IG; it++) {
            const int idx = threadIdx.x + it * NT;
            if (idx < nlines * PY) P[idx] = v[it];
        }
    }
    __syncthreads();
    const int lr = threadIdx.x / TPL, tl = threadIdx.x % TPL;
    float2* Y = P;
    for (int l0 = 0; l0 < nlines; l0 += LPR) {
        const int l = l0 + lr;
        Y = fr::sm_fft<PY, -1, TPL>(P, Pb, l < nlines ? l : 0, tl, twl, l < nlines);
    }
    // forward z FFT: one (component, ky) column per thread
    for (int w = threadIdx.x; w < 3 * PY; w += blockDim.x) {
        const int a = w / PY, ky = w % PY;
        float2 s[PZ];
#pragma unroll
        for (int z = 0; z < PZ; z++) s[z] = z < nz ? Y[((size_t)a * nz + z) * PY + ky] : make_float2(0.f, 0.f);
        fr::RegFFT<PZ, -1, float2>::run(s);
#pragma unroll
        for (int z = 0; z < PZ; z++) Q[((size_t)a * PZ + z) * PY + ky] = s[z];
    }
    __syncthreads();
    // tensor multiply (row a of the symmetric tensor) and inverse z FFT into P
    const float gg = c.g;
    for (int w = threadIdx.x; w < 3 * PY; w += blockDim.x) {
        const int a = w / PY, ky = w % PY;
        const int i0 = a == 0 ? 0 : (a == 1 ? 1 : 2);
        const int i1 = a == 0 ? 1 : (a == 1 ? 3 : 4);
        const int i2 = a == 0 ? 2 : (a == 1 ? 4 : 5);
        float2 h[PZ];
#pragma unroll
        for (int kz = 0; kz < PZ; kz++) {
            const float* Tp = Tk + ((size_t)kz * PY + ky) * 6;
            const float q0 = __ldg(Tp + i0) * gg, q1 = __ldg(Tp + i1) * gg, q2 = __ldg(Tp + i2) * gg;
            const float2 s0 = Q[(0 * PZ + kz) * PY + ky], s1 = Q[(1 * PZ + kz) * PY + ky], s2 = Q[(2 * PZ + kz) * PY + ky];
            h[kz] = make_float2(q0 * s0.x + q1 * s1.x + q2 * s2.x, q0 * s0.y + q1 * s1.y + q2 * s2.y);
        }
        fr::RegFFT<PZ, +1, float2>::run(h);
#pragma unroll
        for (int z = 0; z < PZ; z++)
            if (z < nz) P[((size_t)a * nz + z) * PY + ky] = h[z];
    }
    __syncthreads();
    // inverse y FFT
    for (int l0 = 0; l0 < nlines; l0 += LPR) {
        const int l = l0 + lr;
        Y = fr::sm_fft<PY, +1, TPL>(P, Pb, l < nlines ? l : 0, tl, twl, l < nlines);
    }
    {
        constexpr int IG = (3 * PZ * PY + NT - 1) / NT;
#pragma unroll
        for (int it = 0; it < IG; it++) {
            const int idx = threadIdx.x + it * NT;
            const int l = idx / PY, y = idx % PY;
            if (l < nlines && y < ny) sp[(size_t)l * ny + y] = Y[idx];
        }
    }
    tl_end(c.tl);
}

// ------------------------------------------------------------------ (y,z) pass, register form
// For the planes of a large film (Py 256 or 512, Pz <= 16): one CTA of 384
// threads per kx.  The y transforms of the 3 nz data lines are four-step
// register FFTs (fr::line_fft: T lanes per line, E = Py/T points per lane, one
// warp-synchronous exchange); lane t of a line loads x[t + T j] straight from
// SPEC and stores its outputs in natural order to the plane P[3][nz][Py].
// Then each thread takes whole ky columns: the z transforms of the three
// components (zero-padded to Pz), the 3x3 real tensor multiply and the inverse
// z transforms in registers, data layers back to P.  The inverse y transforms
// read P and store the data rows straight to SPEC.  Shared-memory traffic is
// about a third of the Stockham form's, with no z-spectrum buffer.
template <int PY, int PZ, int NTH = 384>
struct YZR {
    static constexpr int NT = NTH;
    static constexpr int T = fr::Split<PY>::T;
    static constexpr int E = fr::Split<PY>::E;
    static constexpr int LPR = NT / T;                  // lines per round
    static constexpr int EX = E * (T + 1);              // exchange elements per line
    static size_t smem(int nz) { return ((size_t)3 * nz * PY + (size_t)LPR * EX + PY) * sizeof(float2); }
};

template <int PY, int PZ, int NTH>
__global__ void __launch_bounds__(NTH, NTH >= 384 ? 1 : 4) k_yz_reg(ConvK c, const float2* __restrict__ twy,
                                                                    float2* __restrict__ spec,
                                                                    const float* __restrict__ ten6)
{
    using Y = YZR<PY, PZ, NTH>;
    constexpr int NT = Y::NT, T = Y::T, E = Y::E;
    extern __shared__ float2 sm[];
    const int kx = blockIdx.x;
    const int nz = c.nz, ny = c.ny;
    const int nlines = 3 * nz;
    float2* P = sm;                                // [3][nz][PY]
    float2* ex = P + (size_t)nlines * PY;          // [LPR][EX]
    float2* twl = ex + (size_t)Y::LPR * Y::EX;     // [PY]
    const float* Tk = ten6 + (size_t)kx * PZ * PY * 6;
    if (threadIdx.x == 0) {
        const unsigned bytes = (unsigned)(PZ * PY * 6 * sizeof(float));
        if ((((uintptr_t)Tk) & 15) == 0 && (bytes & 15) == 0)
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(Tk), "r"(bytes) : "memory");
    }
    for (int k = threadIdx.x; k < PY; k += NT) twl[k] = twy[k];
    pdl_trigger();
    pdl_wait();
    tl_start(c.tl);
    if (c.run_if && *c.run_if == 0) return;
    // replica blockIdx.y of a packed size class (one for a single film)
    float2* sp = spec + (size_t)blockIdx.y * c.Kx * nlines * ny + (size_t)kx * nlines * ny;
    __syncthreads();
    const int lr = threadIdx.x / T, t = threadIdx.x % T;
    const unsigned mask = T >= 32 ? 0xffffffffu : (((1u << T) - 1u) << (((threadIdx.x & 31) / T) * T));
    float2* exl = ex + (size_t)lr * Y::EX;
    // forward y transforms: SPEC rows -> P (natural order)
    for (int l0 = 0; l0 < nlines; l0 += Y::LPR) {
        const int l = l0 + lr;
        const bool act = l < nlines;   // whole T-lane groups share act
        if (act) {
            float2 v[E];
#pragma unroll
            for (int j = 0; j < E; j++) {
                const int y = t + T * j;
                v[j] = y < ny ? sp[(size_t)l * ny + y] : make_float2(0.f, 0.f);
            }
            fr::line_fft<PY, -1, float2>(v, exl, t, mask, twl);
#pragma unroll
            for (int r = 0; r < E; r++) P[(size_t)l * PY + fr::out_index<PY>(t, r)] = v[r];
        }
    }
    __syncthreads();
    // z transforms, tensor multiply, inverse z transforms: one ky column per thread
    const float gg = c.g;
    for (int ky = threadIdx.x; ky < PY; ky += NT) {
        float2 s0[PZ], s1[PZ], s2[PZ];
#pragma unroll
        for (int z = 0; z < PZ; z++) {
            const bool in = z < nz;
            s0[z] = in ? P[((size_t)0 * nz + z) * PY + ky] : make_float2(0.f, 0.f);
            s1[z] = in ? P[((size_t)1 * nz + z) * PY + ky] : make_float2(0.f, 0.f);
            s2[z] = in ? P[((size_t)2 * nz + z) * PY + ky] : make_float2(0.f, 0.f);
        }
        fr::RegFFT<PZ, -1, float2>::run(s0);
        fr::RegFFT<PZ, -1, float2>::run(s1);
        fr::RegFFT<PZ, -1, float2>::run(s2);
#pragma unroll
        for (int kz = 0; kz < PZ; kz++) {
            const float* Tp = Tk + ((size_t)kz * PY + ky) * 6;
            const float t0 = __ldg(Tp) * gg, t1 = __ldg(Tp + 1) * gg, t2 = __ldg(Tp + 2) * gg;
            const float t3 = __ldg(Tp + 3) * gg, t4 = __ldg(Tp + 4) * gg, t5 = __ldg(Tp + 5) * gg;
            const float2 a = s0[kz], b = s1[kz], d = s2[kz];
            s0[kz] = make_float2(t0 * a.x + t1 * b.x + t2 * d.x, t0 * a.y + t1 * b.y + t2 * d.y);
            s1[kz] = make_float2(t1 * a.x + t3 * b.x + t4 * d.x, t1 * a.y + t3 * b.y + t4 * d.y);
            s2[kz] = make_float2(t2 * a.x + t4 * b.x + t5 * d.x, t2 * a.y + t4 * b.y + t5 * d.y);
        }
        fr::RegFFT<PZ, +1, float2>::run(s0);
        fr::RegFFT<PZ, +1, float2>::run(s1);
        fr::RegFFT<PZ, +1, float2>::run(s2);
#pragma unroll
        for (int z = 0; z < PZ; z++) {
            if (z < nz) {
                P[((size_t)0 * nz + z) * PY + ky] = s0[z];
                P[((size_t)1 * nz + z) * PY + ky] = s1[z];
                P[((size_t)2 * nz + z) * PY + ky] = s2[z];
            }
        }
    }
    __syncthreads();
    // inverse y transforms: P -> SPEC data rows
    for (int l0 = 0; l0 < nlines; l0 += Y::LPR) {
        const int l = l0 + lr;
        if (l < nlines) {
            float2 v[E];
#pragma unroll
            for (int j = 0; j < E; j++) v[j] = P[(size_t)l * PY + t + T * j];
            fr::line_fft<PY, +1, float2>(v, exl, t, mask, twl);
#pragma unroll
            for (int r = 0; r < E; r++) {
                const int y = fr::out_index<PY>(t, r);
                if (y < ny) sp[(size_t)l * ny + y] = v[r];
            }
        }
    }
    tl_end(c.tl);
}

// ------------------------------------------------------------------ (y,z) pass, three threads per column
// The register form for a film's 256-wide planes with 1024 threads per kx:
// the y transforms as in k_yz_reg (line l = (comp, z) stored at
// Z[comp][z][ky]); the column work split three ways so that no thread holds
// all three components: (a) one thread per (comp, ky) takes the z transform
// of its column in registers and writes the Pz spectrum values back in
// place (Z[comp][kz][ky]); (b) one thread per (kz, ky) applies the 3x3 real
// tensor in place; (c) one thread per (comp, ky) takes the inverse z
// transform and writes the data layers back.  The same operations as
// k_yz_reg, element for element, at 64 registers per thread, so more than
// twice the warps per SM.
template <int PY, int PZ>
struct YZC {
    static constexpr int NT = 1024;   // four tensor items per thread (768 left a third of the sixth round busy)
    static constexpr int T = fr::Split<PY>::T;
    static constexpr int E = fr::Split<PY>::E;
    static constexpr int EX = E * (T + 1);              // exchange elements per line
    static size_t smem(int nz) { return ((size_t)3 * PZ * PY + (size_t)3 * nz * EX + PY) * sizeof(float2); }
};

// QT: the tensor is stored for ky <= PY/2 and kz <= PZ/2 only (a tensor
// with the per-axis parities of a point-dipole tensor on an orthogonal
// lattice: XY and YZ odd in ky, XZ and YZ odd in kz), TEN[kx][kz][ky][6]
// with a per-kx stride padded to 16 bytes, mirrored with those signs.
template <int PY, int PZ, bool QT>
__global__ void __launch_bounds__(YZC<PY, PZ>::NT, 1) k_yz_col3(ConvK c, const float2* __restrict__ twy,
                                                   float2* __restrict__ spec, const float* __restrict__ ten6)
{
    using Y = YZC<PY, PZ>;
    constexpr int NT = Y::NT, T = Y::T, E = Y::E;
    constexpr int QY = PY / 2 + 1, QZ = PZ / 2 + 1;
    constexpr int KS = QT ? ((QZ * QY * 6 + 3) & ~3) : PZ * PY * 6;   // tensor floats per kx
    extern __shared__ float2 sm[];
    const int kx = blockIdx.x;
    const int nz = c.nz, ny = c.ny;
    const int nlines = 3 * nz;
    float2* Z = sm;                                  // [3][PZ][PY]
    float2* ex = Z + (size_t)3 * PZ * PY;            // [3 nz][EX]
    float2* twl = ex + (size_t)nlines * Y::EX;       // [PY]
    const float* Tk = ten6 + (size_t)kx * KS;
    if (threadIdx.x == 0) {
        const unsigned bytes = (unsigned)(KS * sizeof(float));
        if ((((uintptr_t)Tk) & 15) == 0 && (bytes & 15) == 0)
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(Tk), "r"(bytes) : "memory");
    }
    for (int k = threadIdx.x; k < PY; k += NT) twl[k] = twy[k];
    pdl_trigger();
    pdl_wait();
    tl_start(c.tl);
    if (c.run_if && *c.run_if == 0) return;
    float2* sp = spec + (size_t)blockIdx.y * c.Kx * nlines * ny + (size_t)kx * nlines * ny;
    __syncthreads();
    const int lr = threadIdx.x / T, t = threadIdx.x % T;
    const unsigned mask = T >= 32 ? 0xffffffffu : (((1u << T) - 1u) << (((threadIdx.x & 31) / T) * T));
    // forward y transforms: SPEC row (comp, z) -> Z[comp][z][*] (natural order)
    {
        const int l = lr;
        if (l < nlines) {
            const int comp = l / nz, z = l % nz;
            float2* exl = ex + (size_t)l * Y::EX;
            float2 v[E];
#pragma unroll
            for (int j = 0; j < E; j++) {
                const int y = t + T * j;
                v[j] = y < ny ? sp[(size_t)l * ny + y] : make_float2(0.f, 0.f);
            }
            fr::line_fft<PY, -1, float2>(v, exl, t, mask, twl);
            float2* Zl = Z + ((size_t)comp * PZ + z) * PY;
#pragma unroll
            for (int r = 0; r < E; r++) Zl[fr::out_index<PY>(t, r)] = v[r];
        }
    }
    __syncthreads();
    // (a) z transform of one (comp, ky) column, in place
    for (int item = threadIdx.x; item < 3 * PY; item += NT) {
        const int comp = item / PY, ky = item % PY;
        float2* col = Z + (size_t)comp * PZ * PY + ky;
        float2 v[PZ];
#pragma unroll
        for (int z = 0; z < PZ; z++) v[z] = z < nz ? col[(size_t)z * PY] : make_float2(0.f, 0.f);
        fr::RegFFT<PZ, -1, float2>::run(v);
#pragma unroll
        for (int z = 0; z < PZ; z++) col[(size_t)z * PY] = v[z];
    }
    __syncthreads();
    // (b) 3x3 real tensor at each (kz, ky); a thread's tensor loads are all
    // issued before its first multiply
    const float gg = c.g;
    constexpr int NI = (PZ * PY + NT - 1) / NT;
    float tt[NI][6];
#pragma unroll
    for (int q = 0; q < NI; q++) {
        const int item = threadIdx.x + q * NT;
        if (item < PZ * PY) {
            if (QT) {
                const int kz = item / PY, ky = item % PY;
                const int kyq = ky <= PY / 2 ? ky : PY - ky, kzq = kz <= PZ / 2 ? kz : PZ - kz;
                const float* Tp = Tk + ((size_t)kzq * QY + kyq) * 6;
#pragma unroll
                for (int e = 0; e < 6; e++) tt[q][e] = __ldg(Tp + e);
                const float sy = ky > PY / 2 ? -1.f : 1.f, sz = kz > PZ / 2 ? -1.f : 1.f;
                tt[q][1] *= sy;
                tt[q][2] *= sz;
                tt[q][4] *= sy * sz;
            } else {
                const float* Tp = Tk + (size_t)item * 6;
#pragma unroll
                for (int e = 0; e < 6; e++) tt[q][e] = __ldg(Tp + e);
            }
        }
    }
#pragma unroll
    for (int q = 0; q < NI; q++) {
        const int item = threadIdx.x + q * NT;
        if (item >= PZ * PY) break;
        const int kz = item / PY, ky = item % PY;
        const float t0 = tt[q][0] * gg, t1 = tt[q][1] * gg, t2 = tt[q][2] * gg;
        const float t3 = tt[q][3] * gg, t4 = tt[q][4] * gg, t5 = tt[q][5] * gg;
        float2* z0 = Z + (size_t)kz * PY + ky;
        const float2 a = z0[0], b = z0[(size_t)PZ * PY], d = z0[(size_t)2 * PZ * PY];
        z0[0] = make_float2(t0 * a.x + t1 * b.x + t2 * d.x, t0 * a.y + t1 * b.y + t2 * d.y);
        z0[(size_t)PZ * PY] = make_float2(t1 * a.x + t3 * b.x + t4 * d.x, t1 * a.y + t3 * b.y + t4 * d.y);
        z0[(size_t)2 * PZ * PY] = make_float2(t2 * a.x + t4 * b.x + t5 * d.x, t2 * a.y + t4 * b.y + t5 * d.y);
    }
    __syncthreads();
    // (c) inverse z transform, data layers back
    for (int item = threadIdx.x; item < 3 * PY; item += NT) {
        const int comp = item / PY, ky = item % PY;
        float2* col = Z + (size_t)comp * PZ * PY + ky;
        float2 v[PZ];
#pragma unroll
        for (int z = 0; z < PZ; z++) v[z] = col[(size_t)z * PY];
        fr::RegFFT<PZ, +1, float2>::run(v);
#pragma unroll
        for (int z = 0; z < PZ; z++)
            if (z < nz) col[(size_t)z * PY] = v[z];
    }
    __syncthreads();
    // inverse y transforms: Z[comp][z][*] -> SPEC data rows
    {
        const int l = lr;
        if (l < nlines) {
            const int comp = l / nz, z = l % nz;
            float2* exl = ex + (size_t)l * Y::EX;
            const float2* Zl = Z + ((size_t)comp * PZ + z) * PY;
            float2 v[E];
#pragma unroll
            for (int j = 0; j < E; j++) v[j] = Zl[t + T * j];
            fr::line_fft<PY, +1, float2>(v, exl, t, mask, twl);
#pragma unroll
            for (int r = 0; r < E; r++) {
                const int y = fr::out_index<PY>(t, r);
                if (y < ny) sp[(size_t)l * ny + y] = v[r];
            }
        }
    }
    tl_end(c.tl);
}

// ------------------------------------------------------------------ split (y,z) passes, FP32
// Planes larger than shared memory (a 256^3 open cube pads to 512 x 512):
// the (y,z) pass as three passes through S2[kx][ky][comp][z] (data layers
// z < nz only; the layout of the generic split kernels in kernels.cu), each
// line transformed in registers by a T-lane group (fr::line_fft):
//   k_sy_fast   CTA (kx, comp, LN data layers): y transforms of the layers'
//               rows, zero-padded to PY; transposed in shared memory so that
//               each ky stores LN consecutive z;
//   k_sz_fast   CTA (kx, COLS ky columns): z transforms of the columns' three
//               components, zero-padded to PZ; 3x3 tensor multiply (ky-major
//               real tensor, scaled by the strength); inverse z transforms,
//               data layers back to S2;
//   k_syi_fast  CTA (kx, comp, LN layers): inverse y transforms, data rows
//               to SPEC[kx][comp][z][y].
// Each shared-memory line buffer serves as the four-step exchange buffer
// and, between transforms, as the line's natural-order spectrum.
constexpr int SPL_NT = 256;   // threads of the y passes
constexpr int SPZ_NT = 192;   // threads of the z pass (a multiple of 3 lines)

template <int PY, typename C = float2>
struct SPY {
    static constexpr int T = fr::Split<PY>::T, E = fr::Split<PY>::E;
    static constexpr int LN = SPL_NT / T;     // data layers per CTA
    static constexpr int EX = E * (T + 1);    // exchange elements per line
    static constexpr int TS = LN + 1;         // transpose row stride, [ky][layer]
    static constexpr int BUF = LN * EX > PY * TS ? LN * EX : PY * TS;
    static constexpr size_t SMEM = (size_t)(PY + BUF) * sizeof(C);
};

template <int PZ, typename C = float2>
struct SPZ {
    static constexpr int T = fr::Split<PZ>::T, E = fr::Split<PZ>::E;
    static constexpr int LN = SPZ_NT / T;     // lines per CTA
    static constexpr int COLS = LN / 3;       // ky columns per CTA
    static constexpr int EX = E * (T + 1);    // >= PZ: exchange, then spectrum
    static constexpr size_t SMEM = (size_t)(PZ + LN * EX) * sizeof(C);
};

// lanes of this thread's T-lane group within its warp
__device__ __forceinline__ unsigned group_mask(int T)
{
    return T >= 32 ? 0xffffffffu : (((1u << T) - 1u) << (((threadIdx.x & 31) / T) * T));
}

// FP32 lines fit two CTAs per SM; FP64 lines hold twice the registers
template <typename C> struct SplitOcc { static constexpr int Y = 2, YI = 3, Z = 3; };
template <> struct SplitOcc<double2> { static constexpr int Y = 1, YI = 1, Z = 2; };

template <int PY, typename C = float2>
__global__ void __launch_bounds__(SPL_NT, SplitOcc<C>::Y) k_sy_fast(ConvK c, const C* __restrict__ twy,
                                                                   const C* __restrict__ spec, C* __restrict__ s2)
{
    using Y = SPY<PY, C>;
    constexpr int T = Y::T, E = Y::E, LN = Y::LN;
    extern __shared__ __align__(16) unsigned char smraw_sy[];
    C* sm = reinterpret_cast<C*>(smraw_sy);
    C* twl = sm;
    C* buf = sm + PY;
    for (int k = threadIdx.x; k < PY; k += SPL_NT) twl[k] = twy[k];
    pdl_trigger();
    pdl_wait();
    if (c.run_if && *c.run_if == 0) return;
    const int nz = c.nz, ny = c.ny;
    const int kx = blockIdx.x, comp = blockIdx.y, z0 = blockIdx.z * LN;
    const int lr = threadIdx.x / T, t = threadIdx.x % T;
    const int nl = min(LN, nz - z0);
    const bool act = lr < nl;   // whole T-lane groups share act
    __syncthreads();
    C v[E];
    if (act) {
        const C* src = spec + (((size_t)kx * 3 + comp) * nz + z0 + lr) * ny;
#pragma unroll
        for (int j = 0; j < E; j++) {
            const int y = t + T * j;
            v[j] = y < ny ? src[y] : cmk<C>(0, 0);
        }
        fr::line_fft<PY, -1, C>(v, buf + (size_t)lr * Y::EX, t, group_mask(T), twl);
    }
    __syncthreads();   // exchange buffers -> transpose buffer
    if (act) {
#pragma unroll
        for (int r = 0; r < E; r++) buf[fr::out_index<PY>(t, r) * Y::TS + lr] = v[r];
    }
    __syncthreads();
    // S2[kx][ky][comp][z0 + l]: LN consecutive threads store one ky's layers
    const int l = threadIdx.x % LN, kq = threadIdx.x / LN;
    C* dst = s2 + ((size_t)kx * PY * 3 + comp) * nz + z0 + l;
    if (l < nl) {
#pragma unroll 4
        for (int k = 0; k < PY / T; k++) {
            const int ky = kq + T * k;
            dst[(size_t)ky * 3 * nz] = buf[ky * Y::TS + l];
        }
    }
}

// Column of local line group c in z-pass CTA b: consecutive columns, or
// with a quarter tensor (ConvK::quarter) mirrored pairs (i, Py - i) with
// i = b COLS/2 + c/2, the self-mirrored columns 0 and Py/2 in CTA 0.
template <int COLS>
__device__ __forceinline__ int sz_column(int b, int c, int Py, bool quarter)
{
    if (!quarter) return b * COLS + c;
    const int i = b * (COLS / 2) + (c >> 1);
    if (i == 0) return (c & 1) ? Py / 2 : 0;
    return (c & 1) ? Py - i : i;
}

template <int PZ, bool QT, typename C = float2>
__global__ void __launch_bounds__(SPZ_NT, SplitOcc<C>::Z) k_sz_fast(ConvK c, const C* __restrict__ twz,
                                                                   C* __restrict__ s2,
                                                                   const decltype(C().x)* __restrict__ ten6)
{
    typedef decltype(C().x) R;
    using Z = SPZ<PZ, C>;
    constexpr int T = Z::T, E = Z::E, COLS = Z::COLS, EX = Z::EX;
    constexpr int QZ = PZ / 2 + 1;
    extern __shared__ __align__(16) unsigned char smraw_sz[];
    C* sm = reinterpret_cast<C*>(smraw_sz);
    C* twl = sm;
    C* buf = sm + PZ;
    const int nz = c.nz, Py = c.Py;
    const int kx = blockIdx.x, b = blockIdx.y, ky0 = b * COLS;
    const int ncol = QT ? COLS : min(COLS, Py - ky0);
    if (threadIdx.x == 0) {
        // the columns' tensor rows (constant across steps) start towards L2
        // while the z transforms run
        const R* Tb;
        unsigned bytes;
        if (QT) {
            Tb = ten6 + ((size_t)kx * (Py / 2 + 1) + b * (COLS / 2)) * QZ * 6;
            bytes = (unsigned)((COLS / 2) * QZ * 6 * sizeof(R));
        } else {
            Tb = ten6 + ((size_t)kx * Py + ky0) * PZ * 6;
            bytes = (unsigned)(ncol * PZ * 6 * sizeof(R));
        }
        if ((((uintptr_t)Tb) & 15) == 0 && (bytes & 15) == 0)
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(Tb), "r"(bytes) : "memory");
    }
    for (int k = threadIdx.x; k < PZ; k += SPZ_NT) twl[k] = twz[k];
    pdl_trigger();
    pdl_wait();
    if (c.run_if && *c.run_if == 0) return;
    const int lr = threadIdx.x / T, t = threadIdx.x % T;
    const int col = lr / 3, comp = lr - 3 * col;
    const bool act = lr < 3 * COLS && col < ncol;   // whole T-lane groups share act
    const unsigned mask = group_mask(T);
    C* exl = buf + (size_t)lr * EX;
    const int kyl = sz_column<COLS>(b, col, Py, QT);
    C* colp = s2 + (((size_t)kx * Py + kyl) * 3 + comp) * nz;
    __syncthreads();
    C v[E];
    if (act) {
#pragma unroll
        for (int j = 0; j < E; j++) {
            const int z = t + T * j;
            v[j] = z < nz ? colp[z] : cmk<C>(0, 0);
        }
        fr::line_fft<PZ, -1, C>(v, exl, t, mask, twl);
#pragma unroll
        for (int r = 0; r < E; r++) exl[fr::out_index<PZ>(t, r)] = v[r];
    }
    __syncthreads();
    // tensor multiply, point p = (column, kz): consecutive threads take
    // consecutive kz, so the tensor rows [kx][ky][kz][6] stream contiguously
    // (a quarter tensor: rows ky <= Py/2, kz <= Pz/2, mirrored with the
    // parity signs of XY, XZ, YZ)
    const R gg = (R)c.g;
    for (int p = threadIdx.x; p < ncol * PZ; p += SPZ_NT) {
        const int cl = p / PZ, kz = p % PZ;
        const R* Tp;
        R sy = 1, sz = 1;
        if (QT) {
            const int ky = sz_column<COLS>(b, cl, Py, true);
            const int kyq = ky <= Py / 2 ? ky : Py - ky;
            const int kzq = kz <= PZ / 2 ? kz : PZ - kz;
            if (ky > Py / 2) sy = -1;
            if (kz > PZ / 2) sz = -1;
            Tp = ten6 + (((size_t)kx * (Py / 2 + 1) + kyq) * QZ + kzq) * 6;
        } else {
            Tp = ten6 + (((size_t)kx * Py + ky0) * PZ + p) * 6;
        }
        const R t0 = __ldg(Tp), t1 = sy * __ldg(Tp + 1), t2 = sz * __ldg(Tp + 2);
        const R t3 = __ldg(Tp + 3), t4 = sy * sz * __ldg(Tp + 4), t5 = __ldg(Tp + 5);
        C* bb = buf + (size_t)cl * 3 * EX + kz;
        const C s0 = bb[0], s1 = bb[EX], s2v = bb[2 * EX];
        bb[0] = cmk<C>(gg * (t0 * s0.x + t1 * s1.x + t2 * s2v.x), gg * (t0 * s0.y + t1 * s1.y + t2 * s2v.y));
        bb[EX] = cmk<C>(gg * (t1 * s0.x + t3 * s1.x + t4 * s2v.x), gg * (t1 * s0.y + t3 * s1.y + t4 * s2v.y));
        bb[2 * EX] = cmk<C>(gg * (t2 * s0.x + t4 * s1.x + t5 * s2v.x), gg * (t2 * s0.y + t4 * s1.y + t5 * s2v.y));
    }
    __syncthreads();
    if (act) {
#pragma unroll
        for (int j = 0; j < E; j++) v[j] = exl[t + T * j];
        __syncwarp(mask);   // every lane has read the spectrum before the exchange overwrites it
        fr::line_fft<PZ, +1, C>(v, exl, t, mask, twl);
#pragma unroll
        for (int r = 0; r < E; r++) {
            const int z = fr::out_index<PZ>(t, r);
            if (z < nz) colp[z] = v[r];
        }
    }
}

template <int PY, typename C = float2>
__global__ void __launch_bounds__(SPL_NT, SplitOcc<C>::YI) k_syi_fast(ConvK c, const C* __restrict__ twy,
                                                                     const C* __restrict__ s2, C* __restrict__ spec)
{
    using Y = SPY<PY, C>;
    constexpr int T = Y::T, E = Y::E, LN = Y::LN;
    extern __shared__ __align__(16) unsigned char smraw_syi[];
    C* sm = reinterpret_cast<C*>(smraw_syi);
    C* twl = sm;
    C* buf = sm + PY;
    for (int k = threadIdx.x; k < PY; k += SPL_NT) twl[k] = twy[k];
    pdl_trigger();
    pdl_wait();
    if (c.run_if && *c.run_if == 0) return;
    const int nz = c.nz, ny = c.ny;
    const int kx = blockIdx.x, comp = blockIdx.y, z0 = blockIdx.z * LN;
    const int nl = min(LN, nz - z0);
    {
        const int l = threadIdx.x % LN, kq = threadIdx.x / LN;
        const C* src = s2 + ((size_t)kx * PY * 3 + comp) * nz + z0 + l;
        if (l < nl) {
#pragma unroll 4
            for (int k = 0; k < PY / T; k++) {
                const int ky = kq + T * k;
                buf[ky * Y::TS + l] = src[(size_t)ky * 3 * nz];
            }
        }
    }
    __syncthreads();
    const int lr = threadIdx.x / T, t = threadIdx.x % T;
    const bool act = lr < nl;
    C v[E];
    if (act) {
#pragma unroll
        for (int j = 0; j < E; j++) v[j] = buf[(t + T * j) * Y::TS + lr];
    }
    __syncthreads();   // transpose buffer -> exchange buffers
    if (act) {
        fr::line_fft<PY, +1, C>(v, buf + (size_t)lr * Y::EX, t, group_mask(T), twl);
        C* dst = spec + (((size_t)kx * 3 + comp) * nz + z0 + lr) * ny;
#pragma unroll
        for (int r = 0; r < E; r++) {
            const int y = fr::out_index<PY>(t, r);
            if (y < ny) dst[y] = v[r];
        }
    }
}

// Sizes the register split passes take: power-of-two Py 32..512 and Pz
// 8..512, Py a multiple of the z pass's columns per CTA.
template <typename C>
static bool split_fast_ok_t(const ConvK& c)
{
    auto p2 = [](int v, int lo) { return v >= lo && v <= 512 && (v & (v - 1)) == 0; };
    if (c.nrep != 1 || !p2(c.Py, 32) || !p2(c.Pz, 8)) return false;
    const int T = c.Pz <= 4 ? 1 : (c.Pz <= 32 ? (c.Pz <= 8 ? 2 : 4) : (c.Pz <= 128 ? 8 : 16));
    const int COLS = (SPZ_NT / T) / 3;
    return c.Py % COLS == 0;
}
static bool split_fast_ok(const ConvK& c) { return split_fast_ok_t<float2>(c); }

template <int PY, int PZ, typename C>
static cudaError_t launch_split_t(const ConvK& c, const C* twy, const C* twz, C* spec, const decltype(C().x)* ten6,
                                  cudaStream_t st)
{
    using Y = SPY<PY, C>;
    using Z = SPZ<PZ, C>;
    C* s2 = static_cast<C*>(c.spec2);
    const dim3 gy(c.Kx, 3, (c.nz + Y::LN - 1) / Y::LN);
    cudaError_t e = mlb::launch_pdl(k_sy_fast<PY, C>, gy, dim3(SPL_NT), Y::SMEM, st, c, twy, (const C*)spec, s2);
    if (e != cudaSuccess) return e;
    if (c.quarter && c.Py % Z::COLS == 0)
        e = mlb::launch_pdl(k_sz_fast<PZ, true, C>, dim3(c.Kx, c.Py / Z::COLS), dim3(SPZ_NT), Z::SMEM, st, c, twz, s2,
                            ten6);
    else if (c.quarter)
        e = cudaErrorInvalidValue;
    else
        e = mlb::launch_pdl(k_sz_fast<PZ, false, C>, dim3(c.Kx, (c.Py + Z::COLS - 1) / Z::COLS), dim3(SPZ_NT), Z::SMEM,
                            st, c, twz, s2, ten6);
    if (e != cudaSuccess) return e;
    return mlb::launch_pdl(k_syi_fast<PY, C>, gy, dim3(SPL_NT), Y::SMEM, st, c, twy, (const C*)s2, spec);
}

template <int PY, typename C>
static cudaError_t launch_split_py(const ConvK& c, const C* twy, const C* twz, C* spec, const decltype(C().x)* ten6,
                                   cudaStream_t st)
{
    switch (c.Pz) {
    case 8: return launch_split_t<PY, 8, C>(c, twy, twz, spec, ten6, st);
    case 16: return launch_split_t<PY, 16, C>(c, twy, twz, spec, ten6, st);
    case 32: return launch_split_t<PY, 32, C>(c, twy, twz, spec, ten6, st);
    case 64: return launch_split_t<PY, 64, C>(c, twy, twz, spec, ten6, st);
    case 128: return launch_split_t<PY, 128, C>(c, twy, twz, spec, ten6, st);
    case 256: return launch_split_t<PY, 256, C>(c, twy, twz, spec, ten6, st);
    case 512: return launch_split_t<PY, 512, C>(c, twy, twz, spec, ten6, st);
    }
    return cudaErrorInvalidValue;
}

template <typename C>
static cudaError_t launch_split_fast(const ConvK& c, const C* twy, const C* twz, C* spec, const decltype(C().x)* ten6,
                                     cudaStream_t st)
{
    switch (c.Py) {
    case 32: return launch_split_py<32, C>(c, twy, twz, spec, ten6, st);
    case 64: return launch_split_py<64, C>(c, twy, twz, spec, ten6, st);
    case 128: return launch_split_py<128, C>(c, twy, twz, spec, ten6, st);
    case 256: return launch_split_py<256, C>(c, twy, twz, spec, ten6, st);
    case 512: return launch_split_py<512, C>(c, twy, twz, spec, ten6, st);
    }
    return cudaErrorInvalidValue;
}

// The split y passes alone (forward: SPEC -> S2 = c.spec2, inverse: S2 ->
// SPEC) for FP32 power-of-two Py in 32..512; used by LongRange2D, whose
// layer mixing reads S2[kx][ky][comp][z] with each k-point's 3 nz values
// contiguous.
template <int PY>
static cudaError_t launch_split_y_t(const ConvK& c, const float2* twy, float2* spec, bool fwd, cudaStream_t st)
{
    using Y = SPY<PY>;
    float2* s2 = static_cast<float2*>(c.spec2);
    const dim3 gy(c.Kx, 3, (c.nz + Y::LN - 1) / Y::LN);
    if (fwd)
        return mlb::launch_pdl(k_sy_fast<PY, float2>, gy, dim3(SPL_NT), Y::SMEM, st, c, twy, (const float2*)spec, s2);
    return mlb::launch_pdl(k_syi_fast<PY, float2>, gy, dim3(SPL_NT), Y::SMEM, st, c, twy, (const float2*)s2, spec);
}

template <int P, typename C>
static cudaError_t cfg_split_c()
{
    const auto a = cudaFuncAttributeMaxDynamicSharedMemorySize;
    cudaError_t e;
    if constexpr (P >= 32) {
        if ((e = cudaFuncSetAttribute(k_sy_fast<P, C>, a, (int)SPY<P, C>::SMEM)) != cudaSuccess) return e;
        if ((e = cudaFuncSetAttribute(k_syi_fast<P, C>, a, (int)SPY<P, C>::SMEM)) != cudaSuccess) return e;
    }
    if ((e = cudaFuncSetAttribute(k_sz_fast<P, true, C>, a, (int)SPZ<P, C>::SMEM)) != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_sz_fast<P, false, C>, a, (int)SPZ<P, C>::SMEM);
}

template <int P>
static cudaError_t cfg_split()
{
    cudaError_t e = cfg_split_c<P, float2>();
    if (e != cudaSuccess) return e;
    return cfg_split_c<P, double2>();
}

// ------------------------------------------------------------------ fused step
// (fused_site_v, the per-site arithmetic, is in fused.cuh)
template <int LT, bool EXS, bool ANI, bool TH, bool ADD, typename R = float>
__device__ __forceinline__ void fused_site(const FastKT<R>& F, int NX, int NY, int NZ, int x, int y, int z, int i,
                                           const R* __restrict__ sx, const R* __restrict__ sy,
                                           const R* __restrict__ sz, const R* __restrict__ ax,
                                           const R* __restrict__ ay, const R* __restrict__ az,
                                           R* __restrict__ ox, R* __restrict__ oy, R* __restrict__ oz)
{
    R Ax = 0, Ay = 0, Az = 0;
    if (ADD) { Ax = __ldg(ax + i); Ay = __ldg(ay + i); Az = __ldg(az + i); }
    R rx, ry, rz;
    fused_site_v<LT, EXS, ANI, TH, ADD>(F, NX, NY, NZ, x, y, z, i, sx, sy, sz, Ax, Ay, Az, rx, ry, rz);
    ox[i] = rx; oy[i] = ry; oz[i] = rz;
}

// R = float (FP32 state) or double (FP64 state, constants in FastKT<double>)
template <int LT, bool EXS, bool ANI, bool TH, bool ADD, typename R = float>
__global__ void __launch_bounds__(256) k_fused_fast(FastKT<R> F0, const R* __restrict__ sx, const R* __restrict__ sy,
                                                    const R* __restrict__ sz, const R* __restrict__ ax,
                                                    const R* __restrict__ ay, const R* __restrict__ az,
                                                    R* __restrict__ ox, R* __restrict__ oy, R* __restrict__ oz)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= F0.nx || y >= F0.ny) return;
    const FastKT<R> F = fastk_resolved(F0);
    const int i = x + F.nx * (y + F.ny * z);
    fused_site<LT, EXS, ANI, TH, ADD, R>(F, F.nx, F.ny, F.nz, x, y, z, i, sx, sy, sz, ax, ay, az, ox, oy, oz);
}

// ------------------------------------------------------------------ fused x pass of a step
// One CTA owns ROWS consecutive rows r = z ny + y (the flattened (z, y) row
// index, r0 .. r0 + ROWS - 1), all three components, and runs on them, in
// shared memory:
//   1. the inverse x transform of the (y,z)-pass output (two rows per
//      complex line, Hermitian completion) -> the dipole field of the rows,
//      written to its slot;
//   2. the fused field terms + LLG update of the rows' sites with that field
//      as the addend -> the new spins (exchange neighbours read from the
//      current spin arrays, which no CTA writes);
//   3. (fwd) the forward x transform of the new spins (two rows per complex
//      line, split) -> the spectrum rows of the next step.
// The spectrum rows a CTA reads in 1 and writes in 3 are its own.  Every
// arithmetic step repeats k_ix_fast, fused_site and k_fx_fast operation for
// operation, so the result is bitwise that of the three separate kernels.
// 32- to 256-point lines (register transforms, a line per T-lane group)
// take 512 threads: the transforms occupy the same L T lanes, and the site
// step has two items per thread (384 threads left a third of them idle in
// the last of three rounds); two CTAs per SM at 64 registers.  512-point
// lines (shared-memory Stockham, TPL threads per line) take 384.
template <int PX, bool TH = false>
struct XSCfg {
    static constexpr int NT = XReg<PX>::OK ? 512 : 384;
    static constexpr int TPL = fr::Tpl<PX>::V;
    static constexpr int L = 384 / TPL;                 // complex lines = 3 ROWS / 2
    static constexpr int ROWS = 2 * L / 3;
    static constexpr int R2 = ROWS / 2;
    static constexpr int KX = PX / 2 + 1;
    // line stride in shared memory: one complex past the line, so that the
    // same k of consecutive lines falls in different banks
    static constexpr int LS = PX + 1;
    static constexpr int LINE = L * LS;
    static constexpr int SPEC = 3 * ROWS * KX;
    static constexpr int BUF = LINE > SPEC ? LINE : SPEC;
    // thermal: the rows' normals, drawn while the spectrum loads are in
    // flight, [3][ROWS][PX] floats (where two CTAs per SM still fit)
    static constexpr bool PRE = TH && PX <= 256;
    static constexpr int NOISE = PRE ? 3 * ROWS * PX : 0;
    // 32- to 256-point lines: register four-step transforms, one exchange buffer per line
    static constexpr int EX = XReg<PX>::OK ? L * XReg<PX>::EX : 0;
    static constexpr int SMEM = (PX + 2 * BUF + EX) * 8 + NOISE * 4;
    static_assert(L % 3 == 0 && ROWS % 2 == 0, "line layout");
    static_assert(XReg<PX>::OK ? L * XReg<PX>::T <= NT : L * TPL == NT, "lines per CTA");
};

template <int PX, int LT, bool EXS, bool ANI, bool TH>
__global__ void __launch_bounds__(XSCfg<PX, TH>::NT, 2) k_xstep(ConvK c, FastK F0, int fwd, const float2* __restrict__ tw,
                                                  float2* __restrict__ spec, const float* __restrict__ sx,
                                                  const float* __restrict__ sy, const float* __restrict__ sz,
                                                  float* __restrict__ hx, float* __restrict__ hy,
                                                  float* __restrict__ hz, float* __restrict__ ox,
                                                  float* __restrict__ oy, float* __restrict__ oz)
{
    using X = XSCfg<PX, TH>;
    constexpr int KX = X::KX, NT = X::NT, ROWS = X::ROWS, R2 = X::R2, LS = X::LS;
    extern __shared__ float2 sm[];
    float2* twl = sm;               // [PX]
    float2* A = twl + PX;           // [L][LS] lines
    float2* B = A + X::BUF;         // [L][LS] scratch
    float2* EXB = B + X::BUF;       // [L][XReg<PX>::EX] exchange buffers (XReg<PX>::OK)
    float* noise = reinterpret_cast<float*>(EXB + X::EX);   // [3][ROWS][PX] (X::PRE)
    const int nx = c.nx, ny = c.ny, nz = c.nz;
    const int nr = nz * ny;                     // rows (z, y), flattened
    const int row0 = blockIdx.x * ROWS;
    const int rows_here = min(ROWS, nr - row0);
    for (int k = threadIdx.x; k < PX; k += NT) twl[k] = tw[k];
    pdl_trigger();
    pdl_wait();
    unsigned long long* tls = c.tl ? c.tl + 2 : nullptr;
    tl_start(tls);
    // captured steps: the next step's block (the other of the pair; no
    // kernel of this step reads it)
    if (F0.adv_next && blockIdx.x == 0 && threadIdx.x == 0) {
        const DevStep* cu = F0.adv_cur;
        DevStep* nx_ = F0.adv_next;
        nx_->th_counter = cu->th_counter + 1ull;
        for (int a = 0; a < 3; a++) {
            nx_->B[a] = cu->B[a] + cu->dB[a];
            nx_->dB[a] = cu->dB[a];
        }
    }
    if (c.run_if && *c.run_if == 0) return;
    // the rows' spins and their z-neighbour rows, into L2 while the inverse
    // transform runs (the step reads them after it)
    if (threadIdx.x < 9) {
        const int comp = threadIdx.x % 3, which = threadIdx.x / 3;
        const int r = which == 0 ? row0 : (which == 1 ? row0 - ny : row0 + ny);
        const float* base = comp == 0 ? sx : (comp == 1 ? sy : sz);
        if (r >= 0 && r + rows_here <= nr) {
            const float* p = base + (size_t)r * nx;
            const unsigned bytes = (unsigned)(rows_here * nx * sizeof(float));
            if ((((uintptr_t)p) & 15) == 0 && (bytes & 15) == 0)
                asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
        }
    }
    const FastK F = fastk_resolved(F0);
    // 1. line l = comp R2 + p: Z[k] = S_row(2p)[k] + i S_row(2p+1)[k] for
    // k < KX, Hermitian completion Z[PX - k] from the conjugates; one item
    // per (kx, comp, p), the row pair's two spectrum values (adjacent in
    // SPEC[kx][comp][row]) loaded together when the pair is 16-byte aligned
    constexpr int NPI = KX * 3 * R2;
    constexpr int IS = (NPI + NT - 1) / NT;
    {
        float4 v[IS];
        const bool pair_ld = (nr & 1) == 0;   // row0 is even: (kx 3 + comp) nr + row0 + 2p is even
#pragma unroll
        for (int it = 0; it < IS; it++) {
            const int idx = threadIdx.x + it * NT;
            const int kx = idx / (3 * R2), rem = idx % (3 * R2);
            const int comp = rem / R2, p = rem % R2;
            v[it] = make_float4(0.f, 0.f, 0.f, 0.f);
            if (idx < NPI && 2 * p < rows_here) {
                const float2* src = spec + ((size_t)kx * 3 + comp) * nr + row0 + 2 * p;
                if (pair_ld && 2 * p + 1 < rows_here) {
                    v[it] = *reinterpret_cast<const float4*>(src);
                } else {
                    const float2 a = src[0];
                    const float2 b = 2 * p + 1 < rows_here ? src[1] : make_float2(0.f, 0.f);
                    v[it] = make_float4(a.x, a.y, b.x, b.y);
                }
            }
        }
        // the normals of this thread's sites in the step below, while the
        // loads are in flight
        constexpr int IP = (R2 * PX + NT - 1) / NT;
        if (X::PRE) {
#pragma unroll 1
            for (int it = 0; it < IP; it++) {
                const int idx = threadIdx.x + it * NT;
                if (idx >= R2 * PX) break;
                const int p = idx / PX, x = idx % PX;
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int row = 2 * p + h;
                    if (row < rows_here && x < nx) {
                        const float3 g = thermal_normal3(F, (row0 + row) * nx + x);
                        float* q = noise + row * PX + x;
                        q[0] = g.x; q[ROWS * PX] = g.y; q[2 * ROWS * PX] = g.z;
                    }
                }
            }
        }
#pragma unroll
        for (int it = 0; it < IS; it++) {
            const int idx = threadIdx.x + it * NT;
            if (idx >= NPI) continue;
            const int kx = idx / (3 * R2), l = idx % (3 * R2);   // l = comp R2 + p
            float2* Zl = A + l * LS;
            float2 a = make_float2(v[it].x, v[it].y), b = make_float2(v[it].z, v[it].w);
            Zl[kx] = make_float2(a.x - b.y, a.y + b.x);
            if (kx > 0 && kx < PX - KX + 1) {
                a = cconj(a); b = cconj(b);
                Zl[PX - kx] = make_float2(a.x - b.y, a.y + b.x);
            }
        }
    }
    __syncthreads();
    const int l = threadIdx.x / X::TPL, tl = threadIdx.x % X::TPL;
    const float2* R;
    if constexpr (XReg<PX>::OK) {
        xreg_lines<PX, +1>(A, LS, X::L, EXB, twl);
        R = A;
    } else {
        R = fr::sm_fft<PX, +1, X::TPL, float2, LS>(A, B, l, tl, twl, true);
    }
    float2* W = (R == A) ? B : A;   // free buffer: the new spins' lines (FWD)
    // 2. field of the rows to the slot, then the step of every site: one
    // (row pair, x) per item, the pair's two rows the real and imaginary
    // parts of one line element
    constexpr int IP = (R2 * PX + NT - 1) / NT;
    // (z, y) of the CTA's first row; a later row's by counting forward (no
    // division per site)
    const int zr0 = row0 / ny, yr0 = row0 - zr0 * ny;
#pragma unroll 1
    for (int it = 0; it < IP; it++) {
        const int idx = threadIdx.x + it * NT;
        if (idx >= R2 * PX) break;
        const int p = idx / PX, x = idx % PX;
        const float2 Ax2 = R[(0 * R2 + p) * LS + x], Ay2 = R[(1 * R2 + p) * LS + x], Az2 = R[(2 * R2 + p) * LS + x];
        float2 o0 = make_float2(0.f, 0.f), o1 = o0, o2 = o0;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int row = 2 * p + h;
            if (row < rows_here && x < nx) {
                const float Ax = h ? Ax2.y : Ax2.x, Ay = h ? Ay2.y : Ay2.x, Az = h ? Az2.y : Az2.x;
                const int r = row0 + row;
                int zz = zr0, y = yr0 + row;
                while (y >= ny) { y -= ny; zz++; }
                const size_t i = (size_t)r * nx + x;
                hx[i] = Ax; hy[i] = Ay; hz[i] = Az;
                float rx, ry, rz;
                float3 g;
                if (X::PRE) {
                    const float* q = noise + row * PX + x;
                    g = make_float3(q[0], q[ROWS * PX], q[2 * ROWS * PX]);
                }
                fused_site_v<LT, EXS, ANI, TH, true>(F, nx, ny, nz, x, y, zz, (int)i, sx, sy, sz, Ax, Ay, Az, rx, ry,
                                                     rz, X::PRE ? &g : nullptr);
                ox[i] = rx; oy[i] = ry; oz[i] = rz;
                if (h) { o0.y = rx; o1.y = ry; o2.y = rz; }
                else { o0.x = rx; o1.x = ry; o2.x = rz; }
            }
        }
        if (fwd) { W[(0 * R2 + p) * LS + x] = o0; W[(1 * R2 + p) * LS + x] = o1; W[(2 * R2 + p) * LS + x] = o2; }
    }
    if (!fwd) {
        tl_end(tls);
        return;
    }
    __syncthreads();
    // 3. forward transform of the new spins' lines, split into the two rows
    const float2* Q;
    if constexpr (XReg<PX>::OK) {
        xreg_lines<PX, -1>(W, LS, X::L, EXB, twl);
        Q = W;
    } else {
        Q = fr::sm_fft<PX, -1, X::TPL, float2, LS>(W, const_cast<float2*>(R), l, tl, twl, true);
    }
    constexpr int IQ = (X::SPEC + NT - 1) / NT;
#pragma unroll
    for (int it = 0; it < IQ; it++) {
        const int idx = threadIdx.x + it * NT;
        const int kx = idx / (3 * ROWS), rem = idx % (3 * ROWS);
        const int comp = rem / ROWS, row = rem % ROWS;
        if (idx >= X::SPEC || row >= rows_here) continue;
        const float2* Z = Q + (comp * R2 + (row >> 1)) * LS;
        const float2 zk = Z[kx], zn = Z[(PX - kx) & (PX - 1)];
        float2 o;
        if ((row & 1) == 0) o = make_float2(0.5f * (zk.x + zn.x), 0.5f * (zk.y - zn.y));
        else o = make_float2(0.5f * (zk.y + zn.y), 0.5f * (zn.x - zk.x));
        spec[((size_t)kx * 3 + comp) * nr + row0 + row] = o;
    }
    tl_end(tls);
}

// Packed ensemble: tile b covers sites [bstart[b], bstart[b] + blockDim) of
// packed replica brep[b]; rinfo[r] = {nx, ny, nz, first packed site}.  CTAs
// walk the tile table with stride gridDim.x (persistent when the grid is
// smaller than the table).  Each replica takes its own applied field and
// thermal deviation (E.rB, E.rsig); the CTA of a replica's first tile
// writes the next step's field B + dB to E.rBn.
template <int LT, bool EXS, bool ANI, bool TH, bool ADD>
__global__ void k_fused_ens(FastK F0, EnsLaunch E, const float* __restrict__ sx, const float* __restrict__ sy,
                            const float* __restrict__ sz, const float* __restrict__ ax, const float* __restrict__ ay,
                            const float* __restrict__ az, float* __restrict__ ox, float* __restrict__ oy,
                            float* __restrict__ oz)
{
    FastK F = fastk_resolved(F0);
    for (int b = blockIdx.x; b < E.nblk; b += gridDim.x) {
        const int rep = __ldg(E.brep + b);
        const int4 r = __ldg(E.rinfo + rep);
        const int start = __ldg(E.bstart + b);
        F.B[0] = (float)E.rB[3 * rep]; F.B[1] = (float)E.rB[3 * rep + 1]; F.B[2] = (float)E.rB[3 * rep + 2];
        if (TH) F.sigma = __ldg(E.rsig + rep);
        if (start == 0 && threadIdx.x < 3)
            E.rBn[3 * rep + threadIdx.x] = E.rB[3 * rep + threadIdx.x] + E.rdB[3 * rep + threadIdx.x];
        const int local = start + threadIdx.x;
        const int n = r.x * r.y * r.z;
        if (local >= n) continue;
        const int x = local % r.x;
        const int y = (local / r.x) % r.y;
        const int z = local / (r.x * r.y);
        fused_site<LT, EXS, ANI, TH, ADD>(F, r.x, r.y, r.z, x, y, z, r.w + local, sx, sy, sz, ax, ay, az, ox, oy, oz);
    }
}

// FP64 per-replica sums (x, y, z, x^2, y^2, z^2): one block per replica.
__global__ void __launch_bounds__(256) k_ens_moments(const int4* __restrict__ rinfo, const float* __restrict__ sx,
                                                     const float* __restrict__ sy, const float* __restrict__ sz,
                                                     double* __restrict__ out)
{
    const int4 r = rinfo[blockIdx.x];
    const int n = r.x * r.y * r.z;
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const double a = sx[r.w + k], b = sy[r.w + k], c = sz[r.w + k];
        acc[0] += a; acc[1] += b; acc[2] += c;
        acc[3] += a * a; acc[4] += b * b; acc[5] += c * c;
    }
    __shared__ double sh[6][8];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < 6; q++) {
        double v = acc[q];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) sh[q][w] = v;
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        double v = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) v += sh[threadIdx.x][k];
        out[blockIdx.x * 6 + threadIdx.x] = v;
    }
}

// ------------------------------------------------------------------ dispatch
namespace mlb {

static bool pow2_in(int v, int lo, int hi) { return v >= lo && v <= hi && (v & (v - 1)) == 0; }

// the register (y,z) kernel: planes of width 64 to 512 with z padded to at
// most 16 and the plane in shared memory (384 threads for a film's 256- and
// 512-wide planes, 128 for the small planes of packed replicas)
static bool yz_reg_ok(int PY, int PZ, const ConvK& c)
{
    if (PZ > 16) return false;
    size_t sm;
    switch (PY) {
    case 64: sm = YZR<64, 16, 128>::smem(c.nz); break;
    case 128: sm = YZR<128, 16, 128>::smem(c.nz); break;
    case 256: sm = YZR<256, 16, 384>::smem(c.nz); break;
    case 512: sm = YZR<512, 16, 384>::smem(c.nz); break;
    default: return false;
    }
    return sm <= 227 * 1024;
}

// shared memory of k_yz_fast: data rows and scratch, z spectra, twiddles
static size_t yz_fast_smem(int PY, int PZ, int nz)
{
    return ((size_t)2 * 3 * nz * PY + (size_t)3 * PZ * PY + PY) * sizeof(float2);
}

bool conv_fast_ok(const ConvK& c)
{
    if (c.general || !pow2_in(c.Px, 16, 512)) return false;
    // large planes: fast x passes around the split (y,z) passes
    if (c.split) return true;
    if (!pow2_in(c.Py, 16, 512) || !pow2_in(c.Pz, 1, 32)) return false;
    return yz_fast_smem(c.Py, c.Pz, c.nz) <= 227 * 1024;
}

static cudaError_t launch_yz_any(const ConvK& c, const float2* twy, float2* spec, const float* ten6,
                                 cudaStream_t st);

// The register split passes for FP64 state (generic x passes around them):
// real (6-component) tensors only.
bool split_fast_ok_f64(const ConvK& c) { return !c.general && split_fast_ok_t<double2>(c); }

cudaError_t launch_split_fast_f64(const ConvK& c, const FftLen L[3], const double2* tw, double2* spec,
                                  const double* ten6, cudaStream_t st)
{
    Prof pf("k_conv_yz_split", st);
    return launch_split_fast<double2>(c, tw + L[1].tw_off, tw + L[2].tw_off, spec, ten6, st);
}

// The 256-wide single-CTA-plane (y,z) kernel runs this pass (so the pass may
// read a quarter tensor): FP32 fast path, one system, automatic variant.
template <int PZ>
static bool col3_fits(const ConvK& c)
{
    return 3 * c.nz <= YZC<256, PZ>::NT / YZC<256, PZ>::T && YZC<256, PZ>::smem(c.nz) <= 227 * 1024;
}
bool yz_col3_ok(const ConvK& c)
{
    if (c.split || c.general || c.nrep != 1 || c.yz_variant != 0 || c.Py != 256 || !conv_fast_ok(c)) return false;
    switch (c.Pz) {
    case 1: return col3_fits<1>(c);
    case 2: return col3_fits<2>(c);
    case 4: return col3_fits<4>(c);
    case 8: return col3_fits<8>(c);
    case 16: return col3_fits<16>(c);
    }
    return false;
}

bool split_y_fast_ok(const ConvK& c)
{
    return c.nrep == 1 && c.Py >= 32 && c.Py <= 512 && (c.Py & (c.Py - 1)) == 0;
}

cudaError_t launch_split_y_fast(const ConvK& c, const FftLen L[3], const float2* tw, float2* spec, bool fwd,
                                cudaStream_t st)
{
    const float2* twy = tw + L[1].tw_off;
    Prof pf(fwd ? "k_sy_fast" : "k_syi_fast", st);
    switch (c.Py) {
    case 32: return launch_split_y_t<32>(c, twy, spec, fwd, st);
    case 64: return launch_split_y_t<64>(c, twy, spec, fwd, st);
    case 128: return launch_split_y_t<128>(c, twy, spec, fwd, st);
    case 256: return launch_split_y_t<256>(c, twy, spec, fwd, st);
    case 512: return launch_split_y_t<512>(c, twy, spec, fwd, st);
    }
    return cudaErrorInvalidValue;
}


// (y,z) pass of the fast path: the whole-plane kernel, or the split passes
static cudaError_t yz_pass(const ConvK& c, const FftLen L[3], const float2* tw, float2* spec, const float* ten6,
                           cudaStream_t st)
{
    if (c.split) {
        if (!split_fast_ok(c)) return launch_conv_split_yz(c, L[1], L[2], tw, spec, ten6, nullptr, 4, st);
        Prof pf("k_conv_yz_split", st);
        return launch_split_fast<float2>(c, tw + L[1].tw_off, tw + L[2].tw_off, spec, ten6, st);
    }
    Prof pf("k_conv_yz", st);
    return launch_yz_any(c, tw + L[1].tw_off, spec, ten6, st);
}

template <int PX>
static cudaError_t launch_x(const ConvK& c, const float2* tw, const float* s[3], float2* spec, float* h[3],
                            cudaStream_t st, bool fwd)
{
    using X = XCfg<PX>;
    dim3 grid((c.nz * c.ny + X::ROWS - 1) / X::ROWS, 1, 3 * c.nrep);
    const size_t smem = X::SMEM;
    if (fwd) {
        return launch_pdl(k_fx_fast<PX, float>, grid, dim3(256), smem, st, c, tw, s[0], s[1], s[2], spec);
    } else {
        return launch_pdl(k_ix_fast<PX, float>, grid, dim3(256), smem, st, c, tw, spec, h[0], h[1], h[2]);
    }
    return cudaGetLastError();
}

template <int PX>
static cudaError_t launch_x_d(const ConvK& c, const double2* tw, const double* s[3], double2* spec, double* h[3],
                              cudaStream_t st, bool fwd)
{
    using X = XCfg<PX>;
    dim3 grid((c.nz * c.ny + X::ROWS - 1) / X::ROWS, 1, 3 * c.nrep);
    const size_t smem = X::SMEM_D;
    if (fwd) return launch_pdl(k_fx_fast<PX, double>, grid, dim3(256), smem, st, c, tw, s[0], s[1], s[2], spec);
    return launch_pdl(k_ix_fast<PX, double>, grid, dim3(256), smem, st, c, tw, spec, h[0], h[1], h[2]);
}

static cudaError_t launch_x_any_d(const ConvK& c, const double2* tw, const double* s[3], double2* spec,
                                  double* h[3], cudaStream_t st, bool fwd)
{
    switch (c.Px) {
    case 16: return launch_x_d<16>(c, tw, s, spec, h, st, fwd);
    case 32: return launch_x_d<32>(c, tw, s, spec, h, st, fwd);
    case 64: return launch_x_d<64>(c, tw, s, spec, h, st, fwd);
    case 128: return launch_x_d<128>(c, tw, s, spec, h, st, fwd);
    case 256: return launch_x_d<256>(c, tw, s, spec, h, st, fwd);
    case 512: return launch_x_d<512>(c, tw, s, spec, h, st, fwd);
    }
    return cudaErrorInvalidValue;
}

static cudaError_t launch_x_any(const ConvK& c, const float2* tw, const float* s[3], float2* spec, float* h[3],
                                cudaStream_t st, bool fwd)
{
    switch (c.Px) {
    case 16: return launch_x<16>(c, tw, s, spec, h, st, fwd);
    case 32: return launch_x<32>(c, tw, s, spec, h, st, fwd);
    case 64: return launch_x<64>(c, tw, s, spec, h, st, fwd);
    case 128: return launch_x<128>(c, tw, s, spec, h, st, fwd);
    case 256: return launch_x<256>(c, tw, s, spec, h, st, fwd);
    case 512: return launch_x<512>(c, tw, s, spec, h, st, fwd);
    }
    return cudaErrorInvalidValue;
}

template <int PY, int PZ>
static cudaError_t launch_yz_t(const ConvK& c, const float2* twy, float2* spec, const float* ten6, cudaStream_t st)
{
    constexpr int RPZ = PZ <= 16 ? PZ : 16;
    if (c.yz_variant == 1 && yz_fast_smem(PY, PZ, c.nz) <= 227 * 1024) {
        const size_t smem = yz_fast_smem(PY, PZ, c.nz);
        return launch_pdl(k_yz_fast<PY, PZ>, dim3(c.Kx, c.nrep), dim3(YZT<PY, PZ>::N), smem, st, c, twy, spec, ten6);
    }
    if constexpr (PY == 256 && PZ <= 16) {
        if (c.yz_variant != 2 && 3 * c.nz <= YZC<PY, PZ>::NT / YZC<PY, PZ>::T &&
            YZC<PY, PZ>::smem(c.nz) <= 227 * 1024) {
            if (c.quarter)
                return launch_pdl(k_yz_col3<PY, PZ, true>, dim3(c.Kx, c.nrep), dim3(YZC<PY, PZ>::NT),
                                  YZC<PY, PZ>::smem(c.nz), st, c, twy, spec, ten6);
            return launch_pdl(k_yz_col3<PY, PZ, false>, dim3(c.Kx, c.nrep), dim3(YZC<PY, PZ>::NT),
                              YZC<PY, PZ>::smem(c.nz), st, c, twy, spec, ten6);
        }
    }
    // a quarter tensor is read by the kernel above only
    if (c.quarter) return cudaErrorInvalidValue;
    if constexpr (PY >= 256) {
        if (yz_reg_ok(PY, PZ, c))
            return launch_pdl(k_yz_reg<PY, RPZ, 384>, dim3(c.Kx, c.nrep), dim3(384), YZR<PY, RPZ, 384>::smem(c.nz), st,
                              c, twy, spec, ten6);
    } else if constexpr (PY >= 64) {
        // small planes (packed replicas): 128-thread CTAs, several per SM
        if (yz_reg_ok(PY, PZ, c))
            return launch_pdl(k_yz_reg<PY, RPZ, 128>, dim3(c.Kx, c.nrep), dim3(128), YZR<PY, RPZ, 128>::smem(c.nz), st,
                              c, twy, spec, ten6);
    }
    const size_t smem = yz_fast_smem(PY, PZ, c.nz);
    return launch_pdl(k_yz_fast<PY, PZ>, dim3(c.Kx, c.nrep), dim3(YZT<PY, PZ>::N), smem, st, c, twy, spec, ten6);
}

template <int PY>
static cudaError_t launch_yz_py(const ConvK& c, const float2* twy, float2* spec, const float* ten6, cudaStream_t st)
{
    switch (c.Pz) {
    case 1: return launch_yz_t<PY, 1>(c, twy, spec, ten6, st);
    case 2: return launch_yz_t<PY, 2>(c, twy, spec, ten6, st);
    case 4: return launch_yz_t<PY, 4>(c, twy, spec, ten6, st);
    case 8: return launch_yz_t<PY, 8>(c, twy, spec, ten6, st);
    case 16: return launch_yz_t<PY, 16>(c, twy, spec, ten6, st);
    case 32: return launch_yz_t<PY, 32>(c, twy, spec, ten6, st);
    }
    return cudaErrorInvalidValue;
}

static cudaError_t launch_yz_any(const ConvK& c, const float2* twy, float2* spec, const float* ten6, cudaStream_t st)
{
    switch (c.Py) {
    case 16: return launch_yz_py<16>(c, twy, spec, ten6, st);
    case 32: return launch_yz_py<32>(c, twy, spec, ten6, st);
    case 64: return launch_yz_py<64>(c, twy, spec, ten6, st);
    case 128: return launch_yz_py<128>(c, twy, spec, ten6, st);
    case 256: return launch_yz_py<256>(c, twy, spec, ten6, st);
    case 512: return launch_yz_py<512>(c, twy, spec, ten6, st);
    }
    return cudaErrorInvalidValue;
}

// Shared-memory limits of every instantiation, set once before any launch
// (a first launch may happen while a graph is being captured).
template <int PX>
static cudaError_t cfg_x()
{
    const cudaFuncAttribute co = cudaFuncAttributePreferredSharedMemoryCarveout;
    const int mx = (int)cudaSharedmemCarveoutMaxShared;
    cudaError_t e = cudaFuncSetAttribute(k_fx_fast<PX, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e != cudaSuccess || (e = cudaFuncSetAttribute(k_fx_fast<PX, float>, co, mx)) != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_ix_fast<PX, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e != cudaSuccess || (e = cudaFuncSetAttribute(k_ix_fast<PX, float>, co, mx)) != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_fx_fast<PX, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    if (e != cudaSuccess || (e = cudaFuncSetAttribute(k_fx_fast<PX, double>, co, mx)) != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_ix_fast<PX, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_ix_fast<PX, double>, co, mx);
}
template <int PY>
static cudaError_t cfg_yz()
{
    const cudaFuncAttribute a = cudaFuncAttributeMaxDynamicSharedMemorySize;
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(k_yz_fast<PY, 1>, a, 227 * 1024)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_yz_fast<PY, 2>, a, 227 * 1024)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_yz_fast<PY, 4>, a, 227 * 1024)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_yz_fast<PY, 8>, a, 227 * 1024)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_yz_fast<PY, 16>, a, 227 * 1024)) != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_yz_fast<PY, 32>, a, 227 * 1024);
}

template <int PX>
static cudaError_t cfg_xs();

template <int PY, int NTH>
static cudaError_t cfg_yzr()
{
    const cudaFuncAttribute a = cudaFuncAttributeMaxDynamicSharedMemorySize;
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(k_yz_reg<PY, 1, NTH>, a, 227 * 1024)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_yz_reg<PY, 2, NTH>, a, 227 * 1024)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_yz_reg<PY, 4, NTH>, a, 227 * 1024)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_yz_reg<PY, 8, NTH>, a, 227 * 1024)) != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_yz_reg<PY, 16, NTH>, a, 227 * 1024);
}

static cudaError_t cfg_yzc()
{
    const cudaFuncAttribute a = cudaFuncAttributeMaxDynamicSharedMemorySize;
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(k_yz_col3<256, 1, false>, a, 227 * 1024)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_yz_col3<256, 2, false>, a, 227 * 1024)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_yz_col3<256, 4, false>, a, 227 * 1024)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_yz_col3<256, 8, false>, a, 227 * 1024)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_yz_col3<256, 16, false>, a, 227 * 1024)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_yz_col3<256, 1, true>, a, 227 * 1024)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_yz_col3<256, 2, true>, a, 227 * 1024)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_yz_col3<256, 4, true>, a, 227 * 1024)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_yz_col3<256, 8, true>, a, 227 * 1024)) != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_yz_col3<256, 16, true>, a, 227 * 1024);
}

cudaError_t conv_fast_configure()
{
    cudaError_t e;
    if ((e = cfg_yzc()) != cudaSuccess) return e;
    if ((e = cfg_x<16>()) || (e = cfg_x<32>()) || (e = cfg_x<64>()) || (e = cfg_x<128>()) || (e = cfg_x<256>()) ||
        (e = cfg_x<512>()))
        return e;
    if ((e = cfg_yz<16>()) || (e = cfg_yz<32>()) || (e = cfg_yz<64>()) || (e = cfg_yz<128>()) || (e = cfg_yz<256>()) ||
        (e = cfg_yz<512>()))
        return e;
    if ((e = cfg_xs<32>()) || (e = cfg_xs<64>()) || (e = cfg_xs<128>()) || (e = cfg_xs<256>()) || (e = cfg_xs<512>()))
        return e;
    if ((e = cfg_yzr<64, 128>()) || (e = cfg_yzr<128, 128>()) || (e = cfg_yzr<256, 384>()) || (e = cfg_yzr<512, 384>()))
        return e;
    if ((e = cfg_split<8>()) || (e = cfg_split<16>()) || (e = cfg_split<32>()) || (e = cfg_split<64>()) ||
        (e = cfg_split<128>()) || (e = cfg_split<256>()) || (e = cfg_split<512>()))
        return e;
    return cudaSuccess;
}

cudaError_t launch_conv_fast(const ConvK& c, const FftLen L[3], const float2* tw, const float* s[3], float2* spec,
                             const float* ten6, float* h[3], cudaStream_t st)
{
    cudaError_t e;
    {
        Prof pf("k_conv_fx", st);
        e = launch_x_any(c, tw + L[0].tw_off, s, spec, h, st, true);
    }
    if (e != cudaSuccess) return e;
    e = yz_pass(c, L, tw, spec, ten6, st);
    if (e != cudaSuccess) return e;
    {
        Prof pf("k_conv_ix", st);
        e = launch_x_any(c, tw + L[0].tw_off, s, spec, h, st, false);
    }
    return e;
}

// ------------------------------------------------------------------ fused x pass dispatch
bool x_fast_ok(const ConvK& c) { return pow2_in(c.Px, 16, 512) && c.Px == c.nx; }

// The register-free Stockham x passes for FP64 state (power-of-two Px
// 16..512, periodic or zero-padded x): 16 bytes per complex, so at most
// (PX + 2 BUF) * 16 bytes of shared memory per CTA.
bool x_fast_ok_f64(const ConvK& c)
{
    if (!pow2_in(c.Px, 16, 512) || c.nrep != 1) return false;
    switch (c.Px) {
    case 16: return XCfg<16>::SMEM_D <= 227 * 1024;
    case 32: return XCfg<32>::SMEM_D <= 227 * 1024;
    case 64: return XCfg<64>::SMEM_D <= 227 * 1024;
    case 128: return XCfg<128>::SMEM_D <= 227 * 1024;
    case 256: return XCfg<256>::SMEM_D <= 227 * 1024;
    case 512: return XCfg<512>::SMEM_D <= 227 * 1024;
    }
    return false;
}

cudaError_t launch_x_pass_f64(const ConvK& c, const FftLen L[3], const double2* tw, const double* s[3],
                              double2* spec, double* h[3], bool fwd, cudaStream_t st)
{
    if (!x_fast_ok_f64(c)) return cudaErrorInvalidValue;
    Prof pf(fwd ? "k_conv_fx" : "k_conv_ix", st);
    return launch_x_any_d(c, tw + L[0].tw_off, s, spec, h, st, fwd);
}

cudaError_t launch_x_pass_fast(const ConvK& c, const FftLen L[3], const float2* tw, const float* s[3], float2* spec,
                               float* h[3], bool fwd, cudaStream_t st)
{
    if (!x_fast_ok(c)) return cudaErrorInvalidValue;
    Prof pf(fwd ? "k_conv_fx" : "k_conv_ix", st);
    return launch_x_any(c, tw + L[0].tw_off, s, spec, h, st, fwd);
}

cudaError_t launch_conv_fast_fyz(const ConvK& c, const FftLen L[3], const float2* tw, const float* s[3], float2* spec,
                                 const float* ten6, bool with_fx, cudaStream_t st)
{
    cudaError_t e = cudaSuccess;
    if (with_fx) {
        Prof pf("k_conv_fx", st);
        e = launch_x_any(c, tw + L[0].tw_off, s, spec, nullptr, st, true);
    }
    if (e != cudaSuccess) return e;
    return yz_pass(c, L, tw, spec, ten6, st);
}

cudaError_t launch_conv_fast_ix(const ConvK& c, const FftLen L[3], const float2* tw, float2* spec, float* h[3],
                                cudaStream_t st)
{
    Prof pf("k_conv_ix", st);
    return launch_x_any(c, tw + L[0].tw_off, nullptr, spec, h, st, false);
}

bool xstep_ok(const ConvK& c, const FastK& F)
{
    return c.nrep == 1 && F.ex && (c.Px == 32 || c.Px == 64 || c.Px == 128 || c.Px == 256 || c.Px == 512);
}

template <int PX, int LT, bool ANI, bool TH>
static cudaError_t xstep_t(const ConvK& c, const FastK& F, int fwd, const float2* tw, float2* spec,
                           const float* s[3], float* h[3], float* o[3], cudaStream_t st)
{
    using X = XSCfg<PX, TH>;
    dim3 grid((c.nz * c.ny + X::ROWS - 1) / X::ROWS, 1, 1);
    return launch_pdl(k_xstep<PX, LT, true, ANI, TH>, grid, dim3(X::NT), (size_t)X::SMEM, st, c, F, fwd, tw, spec,
                      s[0], s[1], s[2], h[0], h[1], h[2], o[0], o[1], o[2]);
}
template <int PX, int LT>
static cudaError_t xstep_lt(const ConvK& c, const FastK& F, int fwd, const float2* tw, float2* spec,
                            const float* s[3], float* h[3], float* o[3], cudaStream_t st)
{
    if (F.ani) {
        if (F.th) return xstep_t<PX, LT, true, true>(c, F, fwd, tw, spec, s, h, o, st);
        return xstep_t<PX, LT, true, false>(c, F, fwd, tw, spec, s, h, o, st);
    }
    if (F.th) return xstep_t<PX, LT, false, true>(c, F, fwd, tw, spec, s, h, o, st);
    return xstep_t<PX, LT, false, false>(c, F, fwd, tw, spec, s, h, o, st);
}
template <int PX>
static cudaError_t xstep_px(const ConvK& c, const FastK& F, int fwd, const float2* tw, float2* spec,
                            const float* s[3], float* h[3], float* o[3], cudaStream_t st)
{
    if (F.llg_type == LLG_CART) return xstep_lt<PX, LLG_CART>(c, F, fwd, tw, spec, s, h, o, st);
    return xstep_lt<PX, LLG_QUAT>(c, F, fwd, tw, spec, s, h, o, st);
}

cudaError_t launch_xstep(const ConvK& c, const FftLen L[3], const float2* tw, float2* spec, const FastK& F,
                         bool fwd, const float* s[3], float* h[3], float* o[3], cudaStream_t st)
{
    Prof pf(fwd ? "k_xstep" : "k_xstep_ix", st);
    const float2* t = tw + L[0].tw_off;
    switch (c.Px) {
    case 32: return xstep_px<32>(c, F, fwd, t, spec, s, h, o, st);
    case 64: return xstep_px<64>(c, F, fwd, t, spec, s, h, o, st);
    case 128: return xstep_px<128>(c, F, fwd, t, spec, s, h, o, st);
    case 256: return xstep_px<256>(c, F, fwd, t, spec, s, h, o, st);
    case 512: return xstep_px<512>(c, F, fwd, t, spec, s, h, o, st);
    }
    return cudaErrorInvalidValue;
}

template <int PX, int LT, bool ANI, bool TH>
static cudaError_t cfg_xs1()
{
    cudaError_t e = cudaFuncSetAttribute(k_xstep<PX, LT, true, ANI, TH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         XSCfg<PX, TH>::SMEM);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_xstep<PX, LT, true, ANI, TH>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                (int)cudaSharedmemCarveoutMaxShared);
}
template <int PX>
static cudaError_t cfg_xs()
{
    cudaError_t e;
    if ((e = cfg_xs1<PX, LLG_CART, false, false>()) || (e = cfg_xs1<PX, LLG_CART, false, true>()) ||
        (e = cfg_xs1<PX, LLG_CART, true, false>()) || (e = cfg_xs1<PX, LLG_CART, true, true>()) ||
        (e = cfg_xs1<PX, LLG_QUAT, false, false>()) || (e = cfg_xs1<PX, LLG_QUAT, false, true>()) ||
        (e = cfg_xs1<PX, LLG_QUAT, true, false>()) || (e = cfg_xs1<PX, LLG_QUAT, true, true>()))
        return e;
    return cudaSuccess;
}

template <int LT, bool EXS, bool ANI, bool TH, bool ADD, typename R>
static void fused_t(const FastKT<R>& F, const R* s[3], const R* a[3], R* o[3], cudaStream_t st)
{
    dim3 blk(32, 8, 1);
    dim3 grid((F.nx + 31) / 32, (F.ny + 7) / 8, F.nz);
    k_fused_fast<LT, EXS, ANI, TH, ADD, R><<<grid, blk, 0, st>>>(F, s[0], s[1], s[2], a[0], a[1], a[2], o[0], o[1],
                                                                 o[2]);
}

template <int LT, bool EXS, bool ANI, bool TH, typename R>
static void fused_add(const FastKT<R>& F, const R* s[3], const R* a[3], R* o[3], cudaStream_t st)
{
    if (a[0]) fused_t<LT, EXS, ANI, TH, true>(F, s, a, o, st);
    else fused_t<LT, EXS, ANI, TH, false>(F, s, a, o, st);
}
template <int LT, bool EXS, bool ANI, typename R>
static void fused_th(const FastKT<R>& F, const R* s[3], const R* a[3], R* o[3], cudaStream_t st)
{
    if (F.th) fused_add<LT, EXS, ANI, true>(F, s, a, o, st);
    else fused_add<LT, EXS, ANI, false>(F, s, a, o, st);
}
template <int LT, bool EXS, typename R>
static void fused_ani(const FastKT<R>& F, const R* s[3], const R* a[3], R* o[3], cudaStream_t st)
{
    if (F.ani) fused_th<LT, EXS, true>(F, s, a, o, st);
    else fused_th<LT, EXS, false>(F, s, a, o, st);
}
template <int LT, typename R>
static void fused_ex(const FastKT<R>& F, const R* s[3], const R* a[3], R* o[3], cudaStream_t st)
{
    if (F.ex) fused_ani<LT, true>(F, s, a, o, st);
    else fused_ani<LT, false>(F, s, a, o, st);
}

template <int LT, bool EXS, bool ANI, bool TH, bool ADD>
static void ens_t(const FastK& F, const EnsLaunch& E, const float* s[3], const float* a[3], float* o[3], cudaStream_t st)
{
    const int grid = E.grid > 0 && E.grid < E.nblk ? E.grid : E.nblk;
    k_fused_ens<LT, EXS, ANI, TH, ADD><<<grid, E.bs, 0, st>>>(F, E, s[0], s[1], s[2], a[0], a[1], a[2], o[0], o[1],
                                                             o[2]);
}
template <int LT, bool EXS, bool ANI, bool TH>
static void ens_add(const FastK& F, const EnsLaunch& E, const float* s[3], const float* a[3], float* o[3], cudaStream_t st)
{
    if (a[0]) ens_t<LT, EXS, ANI, TH, true>(F, E, s, a, o, st);
    else ens_t<LT, EXS, ANI, TH, false>(F, E, s, a, o, st);
}
template <int LT, bool EXS, bool ANI>
static void ens_th(const FastK& F, const EnsLaunch& E, const float* s[3], const float* a[3], float* o[3], cudaStream_t st)
{
    if (F.th) ens_add<LT, EXS, ANI, true>(F, E, s, a, o, st);
    else ens_add<LT, EXS, ANI, false>(F, E, s, a, o, st);
}
template <int LT, bool EXS>
static void ens_ani(const FastK& F, const EnsLaunch& E, const float* s[3], const float* a[3], float* o[3], cudaStream_t st)
{
    if (F.ani) ens_th<LT, EXS, true>(F, E, s, a, o, st);
    else ens_th<LT, EXS, false>(F, E, s, a, o, st);
}

cudaError_t launch_fused_ens(const FastK& F, const EnsLaunch& E, const float* s[3], const float* a[3], float* o[3],
                             cudaStream_t st)
{
    Prof pf("k_fused_ens", st);
    if (F.llg_type == LLG_CART) {
        if (F.ex) ens_ani<LLG_CART, true>(F, E, s, a, o, st);
        else ens_ani<LLG_CART, false>(F, E, s, a, o, st);
    } else {
        if (F.ex) ens_ani<LLG_QUAT, true>(F, E, s, a, o, st);
        else ens_ani<LLG_QUAT, false>(F, E, s, a, o, st);
    }
    return cudaGetLastError();
}

cudaError_t launch_ens_moments(const int4* rinfo, int nrep, const float* s[3], double* out, cudaStream_t st)
{
    k_ens_moments<<<nrep, 256, 0, st>>>(rinfo, s[0], s[1], s[2], out);
    return cudaGetLastError();
}

cudaError_t launch_fused_fast(const FastK& F, const float* s[3], const float* a[3], float* o[3], cudaStream_t st)
{
    Prof pf("k_fused_step", st);
    if (F.llg_type == LLG_CART) fused_ex<LLG_CART>(F, s, a, o, st);
    else fused_ex<LLG_QUAT>(F, s, a, o, st);
    return cudaGetLastError();
}

cudaError_t launch_fused_fast_f64(const FastKT<double>& F, const double* s[3], const double* a[3], double* o[3],
                                  cudaStream_t st)
{
    Prof pf("k_fused_step", st);
    if (F.llg_type == LLG_CART) fused_ex<LLG_CART>(F, s, a, o, st);
    else fused_ex<LLG_QUAT>(F, s, a, o, st);
    return cudaGetLastError();
}

} // namespace mlb
