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
    for (int k = 0; k < 64; k++) {
        const double a = 2.0 * M_PI * k / 64.0;
        h[k] = make_float2((float)cos(a), (float)(-sin(a)));
    }
    return cudaMemcpyToSymbol(fr::c_w64, h, sizeof(h));
}

} // namespace mlb

using fr::Split;

// ------------------------------------------------------------------ x passes
template <int PX>
struct XCfg {
    static constexpr int T = Split<PX>::T;
    static constexpr int E = Split<PX>::E;
    static constexpr int LINES = 256 / (T > 0 ? T : 1) > 32 ? 32 : 256 / T; // lines per CTA
    static constexpr int ROWS = 2 * LINES;
    static constexpr int EX = E * (T + 1) > PX ? E * (T + 1) : PX;         // per-line buffer
    static constexpr int KX = PX / 2 + 1;
};

template <int PX>
__global__ void __launch_bounds__(256) k_fx_fast(ConvK c, const float2* __restrict__ tw, const float* __restrict__ sx,
                                                 const float* __restrict__ sy, const float* __restrict__ sz,
                                                 float2* __restrict__ spec)
{
    using X = XCfg<PX>;
    constexpr int T = X::T, E = X::E;
    extern __shared__ float2 sm[];
    float2* twl = sm + X::LINES * X::EX;
    for (int k = threadIdx.x; k < PX; k += blockDim.x) twl[k] = tw[k];
    __syncthreads();
    const int comp = blockIdx.z, zz = blockIdx.y;
    const int row0 = blockIdx.x * X::ROWS;
    const float* src = comp == 0 ? sx : (comp == 1 ? sy : sz);
    const int g = threadIdx.x / T, t = threadIdx.x % T;
    const bool active = g < X::LINES;
    float2* ex = sm + g * X::EX;
    const int ya = row0 + 2 * g, yb = ya + 1;
    const unsigned mask = T >= 32 ? 0xffffffffu : (((1u << T) - 1u) << ((threadIdx.x & 31) / T * T));
    if (active) {
        float2 v[E];
#pragma unroll
        for (int j = 0; j < E; j++) {
            const int x = t + T * j;
            float a = 0.f, b = 0.f;
            if (x < c.nx) {
                if (ya < c.ny) a = __ldg(src + ((size_t)zz * c.ny + ya) * c.nx + x);
                if (yb < c.ny) b = __ldg(src + ((size_t)zz * c.ny + yb) * c.nx + x);
            }
            v[j] = make_float2(a, b);
        }
        fr::line_fft<PX, -1>(v, ex, t, mask, twl);
        // stage Z in natural order
#pragma unroll
        for (int r = 0; r < E; r++) ex[fr::out_index<PX>(t, r)] = v[r];
    }
    __syncthreads();
    // split the two real rows and store SPEC[kx][comp][zz][row]
    const int rows_here = min(X::ROWS, c.ny - row0);
    for (int idx = threadIdx.x; idx < X::KX * X::ROWS; idx += blockDim.x) {
        const int kx = idx / X::ROWS, row = idx % X::ROWS;
        if (row >= rows_here) continue;
        const float2* Z = sm + (row >> 1) * X::EX;
        const float2 zk = Z[kx], zn = Z[(PX - kx) & (PX - 1)];
        float2 o;
        if ((row & 1) == 0) o = make_float2(0.5f * (zk.x + zn.x), 0.5f * (zk.y - zn.y));
        else o = make_float2(0.5f * (zk.y + zn.y), 0.5f * (zn.x - zk.x));
        spec[(((size_t)kx * 3 + comp) * c.nz + zz) * c.ny + row0 + row] = o;
    }
}

template <int PX>
__global__ void __launch_bounds__(256) k_ix_fast(ConvK c, const float2* __restrict__ tw, const float2* __restrict__ spec,
                                                 float* __restrict__ hx, float* __restrict__ hy,
                                                 float* __restrict__ hz)
{
    using X = XCfg<PX>;
    constexpr int T = X::T, E = X::E, KX = X::KX;
    extern __shared__ float2 sm[];
    float2* S = sm;                              // [ROWS][KX] spectra
    float2* EXB = sm + X::ROWS * KX;             // per-line buffers
    float2* twl = EXB + X::LINES * X::EX;        // twiddles
    for (int k = threadIdx.x; k < PX; k += blockDim.x) twl[k] = tw[k];
    const int comp = blockIdx.z, zz = blockIdx.y;
    const int row0 = blockIdx.x * X::ROWS;
    const int rows_here = min(X::ROWS, c.ny - row0);
    float* dst = comp == 0 ? hx : (comp == 1 ? hy : hz);
    for (int idx = threadIdx.x; idx < KX * X::ROWS; idx += blockDim.x) {
        const int kx = idx / X::ROWS, row = idx % X::ROWS;
        float2 v = make_float2(0.f, 0.f);
        if (row < rows_here) v = spec[(((size_t)kx * 3 + comp) * c.nz + zz) * c.ny + row0 + row];
        S[row * KX + kx] = v;
    }
    __syncthreads();
    const int g = threadIdx.x / T, t = threadIdx.x % T;
    const bool active = g < X::LINES;
    float2* ex = EXB + g * X::EX;
    const unsigned mask = T >= 32 ? 0xffffffffu : (((1u << T) - 1u) << ((threadIdx.x & 31) / T * T));
    if (active) {
        const float2* A = S + (2 * g) * KX;
        const float2* B = S + (2 * g + 1) * KX;
        float2 v[E];
#pragma unroll
        for (int j = 0; j < E; j++) {
            const int k = t + T * j;
            float2 a, b;
            if (k < KX) { a = A[k]; b = B[k]; }
            else { a = cconj(A[PX - k]); b = cconj(B[PX - k]); }
            v[j] = make_float2(a.x - b.y, a.y + b.x); // A + iB
        }
        fr::line_fft<PX, +1>(v, ex, t, mask, twl);
#pragma unroll
        for (int r = 0; r < E; r++) ex[fr::out_index<PX>(t, r)] = v[r];
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < X::ROWS * c.nx; idx += blockDim.x) {
        const int row = idx / c.nx, x = idx % c.nx;
        if (row >= rows_here) continue;
        const float2 z = EXB[(row >> 1) * X::EX + x];
        dst[((size_t)zz * c.ny + row0 + row) * c.nx + x] = (row & 1) ? z.y : z.x;
    }
}

// ------------------------------------------------------------------ (y,z) pass
template <int PY>
struct YCfg {
    static constexpr int T = Split<PY>::T;
    static constexpr int E = Split<PY>::E;
    static constexpr int EX = E * (T + 1);
};

// threads of k_yz_fast: 768 (80 registers each), 512 for PY = 512 whose
// 32-element lanes need more registers
template <int PY>
struct YZT {
    static constexpr int N = PY >= 512 ? 512 : 768;
};

template <int PY, int PZ>
__global__ void __launch_bounds__(YZT<PY>::N, 1) k_yz_fast(ConvK c, const float2* __restrict__ twy,
                                                           float2* __restrict__ spec, const float* __restrict__ ten6)
{
    using Y = YCfg<PY>;
    constexpr int YZ_THREADS = YZT<PY>::N;
    constexpr int T = Y::T, E = Y::E;
    extern __shared__ float2 sm[];
    const int kx = blockIdx.x;
    const int nz = c.nz, ny = c.ny;
    const int nlines = 3 * nz;
    const int LIN = min(nlines, YZ_THREADS / T);                 // y lines in flight
    const int R2 = max(3 * PZ * PY, LIN * Y::EX);
    float2* P = sm;                          // [3][nz][PY] data rows
    float2* Q = P + 3 * nz * PY;             // [3][PZ][PY] z spectra (z phase)
    float2* EXB = Q;                         // [LIN][EX] line buffers (y phases)
    float2* twl = Q + R2;                    // [PY]
    const float* Tk = ten6 + (size_t)kx * PZ * PY * 6;
    if (threadIdx.x == 0) {
        // pull this kx's tensor chunk into L2 while the y transforms run
        const unsigned bytes = (unsigned)(PZ * PY * 6 * sizeof(float));
        if ((((uintptr_t)Tk) & 15) == 0 && (bytes & 15) == 0)
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(Tk), "r"(bytes) : "memory");
    }
    for (int k = threadIdx.x; k < PY; k += blockDim.x) twl[k] = twy[k];
    __syncthreads();
    float2* sp = spec + (size_t)kx * 3 * nz * ny;
    const int g = threadIdx.x / T, t = threadIdx.x % T;
    const unsigned mask = T >= 32 ? 0xffffffffu : (((1u << T) - 1u) << ((threadIdx.x & 31) / T * T));
    // forward y FFT of every data line (c, z)
    for (int l0 = 0; l0 < nlines; l0 += LIN) {
        const int l = l0 + g;
        if (g < LIN && l < nlines) {
            const float2* in = sp + (size_t)l * ny;
            float2 v[E];
#pragma unroll
            for (int j = 0; j < E; j++) {
                const int y = t + T * j;
                v[j] = y < ny ? in[y] : make_float2(0.f, 0.f);
            }
            fr::line_fft<PY, -1>(v, EXB + g * Y::EX, t, mask, twl);
            float2* out = P + (size_t)l * PY;
#pragma unroll
            for (int r = 0; r < E; r++) out[fr::out_index<PY>(t, r)] = v[r];
        }
    }
    __syncthreads();
    // forward z FFT: one (component, ky) column per thread
    for (int w = threadIdx.x; w < 3 * PY; w += blockDim.x) {
        const int a = w / PY, ky = w % PY;
        float2 s[PZ];
#pragma unroll
        for (int z = 0; z < PZ; z++) s[z] = z < nz ? P[((size_t)a * nz + z) * PY + ky] : make_float2(0.f, 0.f);
        fr::RegFFT<PZ, -1, float2>::run(s);
#pragma unroll
        for (int z = 0; z < PZ; z++) Q[((size_t)a * PZ + z) * PY + ky] = s[z];
    }
    __syncthreads();
    // tensor multiply (row a of the symmetric tensor) and inverse z FFT
    const float gg = c.g;
    for (int w = threadIdx.x; w < 3 * PY; w += blockDim.x) {
        const int a = w / PY, ky = w % PY;
        // row a of [[0,1,2],[1,3,4],[2,4,5]]
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
    // inverse y FFT, store the data rows
    for (int l0 = 0; l0 < nlines; l0 += LIN) {
        const int l = l0 + g;
        if (g < LIN && l < nlines) {
            const float2* in = P + (size_t)l * PY;
            float2 v[E];
#pragma unroll
            for (int j = 0; j < E; j++) v[j] = in[t + T * j];
            fr::line_fft<PY, +1>(v, EXB + g * Y::EX, t, mask, twl);
            float2* out = sp + (size_t)l * ny;
#pragma unroll
            for (int r = 0; r < E; r++) {
                const int y = fr::out_index<PY>(t, r);
                if (y < ny) out[y] = v[r];
            }
        }
    }
}

// ------------------------------------------------------------------ fused step
// Uniform-parameter systems: ms, alpha, gamma, anisotropy and thermal scale
// the same on every site, exchange as a six-direction stencil.  Constants
// are folded on the host (FastK).
template <int LT, bool EXS, bool ANI, bool TH, bool ADD>
__global__ void __launch_bounds__(256) k_fused_fast(FastK F, const float* __restrict__ sx, const float* __restrict__ sy,
                                                    const float* __restrict__ sz, const float* __restrict__ ax,
                                                    const float* __restrict__ ay, const float* __restrict__ az,
                                                    float* __restrict__ ox, float* __restrict__ oy,
                                                    float* __restrict__ oz)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= F.nx || y >= F.ny) return;
    const int nxy = F.nx * F.ny;
    const int i = x + F.nx * y + nxy * z;
    const float Sx = __ldg(sx + i), Sy = __ldg(sy + i), Sz = __ldg(sz + i);
    float Hx = F.B[0], Hy = F.B[1], Hz = F.B[2];
    if (F.zdctr) {
        const float kk = (float)(*F.zdctr);
        Hx += kk * F.dB[0]; Hy += kk * F.dB[1]; Hz += kk * F.dB[2];
    }
    if (EXS) {
        float ex = 0.f, ey = 0.f, ez = 0.f;
#define MLB_NB(cond, wrapcond, off, woff, J)                                                       \
        if ((J) != 0.f) {                                                                          \
            int f = -1;                                                                            \
            if (cond) f = i + (off);                                                               \
            else if (wrapcond) f = i + (woff);                                                     \
            if (f >= 0) {                                                                          \
                ex += (J) * __ldg(sx + f); ey += (J) * __ldg(sy + f); ez += (J) * __ldg(sz + f);   \
            }                                                                                      \
        }
        MLB_NB(x + 1 < F.nx, F.pbc[0], 1, 1 - F.nx, F.J[0])
        MLB_NB(x > 0, F.pbc[0], -1, F.nx - 1, F.J[1])
        MLB_NB(y + 1 < F.ny, F.pbc[1], F.nx, F.nx - nxy, F.J[2])
        MLB_NB(y > 0, F.pbc[1], -F.nx, nxy - F.nx, F.J[3])
        MLB_NB(z + 1 < F.nz, F.pbc[2], nxy, nxy - nxy * F.nz, F.J[4])
        MLB_NB(z > 0, F.pbc[2], -nxy, nxy * F.nz - nxy, F.J[5])
#undef MLB_NB
        Hx += ex; Hy += ey; Hz += ez;
    }
    if (ANI) {
        const float v = F.ani_c * (Sx * F.axis[0] + Sy * F.axis[1] + Sz * F.axis[2]);
        Hx += v * F.axis[0]; Hy += v * F.axis[1]; Hz += v * F.axis[2];
    }
    float Tx = 0.f, Ty = 0.f, Tz = 0.f;
    if (TH) {
        const uint64_t ctr = F.counter + (F.dctr ? *F.dctr : 0ull);
        const float3 nrm = philox_normal3(F.seed, ctr, (uint32_t)i, 0x6d6c6232u);
        Tx = F.sigma * nrm.x; Ty = F.sigma * nrm.y; Tz = F.sigma * nrm.z;
        Hx += Tx; Hy += Ty; Hz += Tz;
    }
    if (ADD) {
        Hx += F.addw * __ldg(ax + i); Hy += F.addw * __ldg(ay + i); Hz += F.addw * __ldg(az + i);
    }
    float nx_, ny_, nz_;
    if (LT == LLG_CART) {
        if (F.dt_zero) { nx_ = Sx; ny_ = Sy; nz_ = Sz; }
        else {
            // h = H - Hth; dM = -p gaa M x H - d (a/ms) gaa M x (M x h)
            const float hx = F.tof ? Hx - Tx : Hx, hy = F.tof ? Hy - Ty : Hy, hz = F.tof ? Hz - Tz : Hz;
            const float mhx = Sy * hz - Sz * hy, mhy = Sz * hx - Sx * hz, mhz = Sx * hy - Sy * hx;
            const float mmx = Sy * mhz - Sz * mhy, mmy = Sz * mhx - Sx * mhz, mmz = Sx * mhy - Sy * mhx;
            const float MHx = Sy * Hz - Sz * Hy, MHy = Sz * Hx - Sx * Hz, MHz = Sx * Hy - Sy * Hx;
            nx_ = Sx + F.dt * (F.c_prec * MHx - F.c_damp * mmx);
            ny_ = Sy + F.dt * (F.c_prec * MHy - F.c_damp * mmy);
            nz_ = Sz + F.dt * (F.c_prec * MHz - F.c_damp * mmz);
        }
    } else {
        float Hpx, Hpy, Hpz;
        if (F.tof) {
            const float hx = Hx - Tx, hy = Hy - Ty, hz = Hz - Tz;
            const float shx = Sy * hz - Sz * hy, shy = Sz * hx - Sx * hz, shz = Sx * hy - Sy * hx;
            Hpx = F.precess * Hx + F.c_damp * shx;
            Hpy = F.precess * Hy + F.c_damp * shy;
            Hpz = F.precess * Hz + F.c_damp * shz;
        } else {
            const float shx = Sy * Hz - Sz * Hy, shy = Sz * Hx - Sx * Hz, shz = Sx * Hy - Sy * Hx;
            Hpx = Hx + F.c_damp * shx; Hpy = Hy + F.c_damp * shy; Hpz = Hz + F.c_damp * shz;
        }
        const float HL2 = Hpx * Hpx + Hpy * Hpy + Hpz * Hpz;
        if (HL2 > 0.f) {
            const float iHL = rsqrtf(HL2);
            const float HL = HL2 * iHL;
            float sn, cs;
            sincosf(F.c_rot * HL, &sn, &cs);
            const float qw = cs, qx = sn * Hpx * iHL, qy = sn * Hpy * iHL, qz = sn * Hpz * iHL;
            const float tw = -qx * Sx - qy * Sy - qz * Sz;
            const float tx = qw * Sx + qy * Sz - qz * Sy;
            const float ty = qw * Sy + qz * Sx - qx * Sz;
            const float tz = qw * Sz + qx * Sy - qy * Sx;
            nx_ = -tw * qx + qw * tx - ty * qz + tz * qy;
            ny_ = -tw * qy + qw * ty - tz * qx + tx * qz;
            nz_ = -tw * qz + qw * tz - tx * qy + ty * qx;
        } else { nx_ = Sx; ny_ = Sy; nz_ = Sz; }
    }
    if (F.renorm) {
        const float mm = nx_ * nx_ + ny_ * ny_ + nz_ * nz_;
        if (mm != 0.f) {
            const float inv = F.ms * rsqrtf(mm);
            nx_ *= inv; ny_ *= inv; nz_ *= inv;
        }
    }
    ox[i] = nx_; oy[i] = ny_; oz[i] = nz_;
}

// ------------------------------------------------------------------ dispatch
namespace mlb {

static bool pow2_in(int v, int lo, int hi) { return v >= lo && v <= hi && (v & (v - 1)) == 0; }

// shared memory of k_yz_fast: data rows, z spectra, line buffers, twiddles
static size_t yz_fast_smem(int PY, int PZ, int nz)
{
    const int T = PY <= 4 ? 1 : (PY <= 32 ? (PY <= 8 ? 2 : 4) : (PY <= 128 ? 8 : 16));
    const int E = PY / T;
    const int threads = PY >= 512 ? 512 : 768;
    const int lines = std::min(3 * nz, threads / T);
    const size_t r2 = std::max((size_t)3 * PZ * PY, (size_t)lines * E * (T + 1));
    return ((size_t)3 * nz * PY + r2 + PY) * sizeof(float2);
}

bool conv_fast_ok(const ConvK& c)
{
    if (c.general || !pow2_in(c.Px, 16, 512) || !pow2_in(c.Py, 16, 512) || !pow2_in(c.Pz, 1, 16)) return false;
    return yz_fast_smem(c.Py, c.Pz, c.nz) <= 227 * 1024;
}

template <int PX>
static cudaError_t launch_x(const ConvK& c, const float2* tw, const float* s[3], float2* spec, float* h[3],
                            cudaStream_t st, bool fwd)
{
    using X = XCfg<PX>;
    dim3 grid((c.ny + X::ROWS - 1) / X::ROWS, c.nz, 3);
    if (fwd) {
        const size_t smem = ((size_t)X::LINES * X::EX + PX) * sizeof(float2);
        static bool cfg = false;
        if (!cfg) { cudaFuncSetAttribute(k_fx_fast<PX>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024); cfg = true; }
        k_fx_fast<PX><<<grid, 256, smem, st>>>(c, tw, s[0], s[1], s[2], spec);
    } else {
        const size_t smem = ((size_t)X::ROWS * X::KX + (size_t)X::LINES * X::EX + PX) * sizeof(float2);
        static bool cfg = false;
        if (!cfg) { cudaFuncSetAttribute(k_ix_fast<PX>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024); cfg = true; }
        k_ix_fast<PX><<<grid, 256, smem, st>>>(c, tw, spec, h[0], h[1], h[2]);
    }
    return cudaGetLastError();
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
    const size_t smem = yz_fast_smem(PY, PZ, c.nz);
    static bool cfg = false;
    if (!cfg) { cudaFuncSetAttribute(k_yz_fast<PY, PZ>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024); cfg = true; }
    k_yz_fast<PY, PZ><<<c.Kx, YZT<PY>::N, smem, st>>>(c, twy, spec, ten6);
    return cudaGetLastError();
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

cudaError_t launch_conv_fast(const ConvK& c, const FftLen L[3], const float2* tw, const float* s[3], float2* spec,
                             const float* ten6, float* h[3], cudaStream_t st)
{
    cudaError_t e;
    {
        Prof pf("k_conv_fx", st);
        e = launch_x_any(c, tw + L[0].tw_off, s, spec, h, st, true);
    }
    if (e != cudaSuccess) return e;
    {
        Prof pf("k_conv_yz", st);
        e = launch_yz_any(c, tw + L[1].tw_off, spec, ten6, st);
    }
    if (e != cudaSuccess) return e;
    {
        Prof pf("k_conv_ix", st);
        e = launch_x_any(c, tw + L[0].tw_off, s, spec, h, st, false);
    }
    return e;
}

template <int LT, bool EXS, bool ANI, bool TH, bool ADD>
static void fused_t(const FastK& F, const float* s[3], const float* a[3], float* o[3], cudaStream_t st)
{
    dim3 blk(32, 8, 1);
    dim3 grid((F.nx + 31) / 32, (F.ny + 7) / 8, F.nz);
    k_fused_fast<LT, EXS, ANI, TH, ADD><<<grid, blk, 0, st>>>(F, s[0], s[1], s[2], a[0], a[1], a[2], o[0], o[1], o[2]);
}

template <int LT, bool EXS, bool ANI, bool TH>
static void fused_add(const FastK& F, const float* s[3], const float* a[3], float* o[3], cudaStream_t st)
{
    if (a[0]) fused_t<LT, EXS, ANI, TH, true>(F, s, a, o, st);
    else fused_t<LT, EXS, ANI, TH, false>(F, s, a, o, st);
}
template <int LT, bool EXS, bool ANI>
static void fused_th(const FastK& F, const float* s[3], const float* a[3], float* o[3], cudaStream_t st)
{
    if (F.th) fused_add<LT, EXS, ANI, true>(F, s, a, o, st);
    else fused_add<LT, EXS, ANI, false>(F, s, a, o, st);
}
template <int LT, bool EXS>
static void fused_ani(const FastK& F, const float* s[3], const float* a[3], float* o[3], cudaStream_t st)
{
    if (F.ani) fused_th<LT, EXS, true>(F, s, a, o, st);
    else fused_th<LT, EXS, false>(F, s, a, o, st);
}
template <int LT>
static void fused_ex(const FastK& F, const float* s[3], const float* a[3], float* o[3], cudaStream_t st)
{
    if (F.ex) fused_ani<LT, true>(F, s, a, o, st);
    else fused_ani<LT, false>(F, s, a, o, st);
}

cudaError_t launch_fused_fast(const FastK& F, const float* s[3], const float* a[3], float* o[3], cudaStream_t st)
{
    Prof pf("k_fused_step", st);
    if (F.llg_type == LLG_CART) fused_ex<LLG_CART>(F, s, a, o, st);
    else fused_ex<LLG_QUAT>(F, s, a, o, st);
    return cudaGetLastError();
}

} // namespace mlb
