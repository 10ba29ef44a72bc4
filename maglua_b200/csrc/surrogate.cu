// surrogate.cu -- learned spectral surrogate of the dipolar-field update
// (no counterpart in the reference; it stands in for the LongRange
// convolution, M/cpu/longrange/spinoperationlongrange.cpp:354-440, between
// exact evaluations).
//
// The network maps the magnetisation change since the last exact
// evaluation, X = m - m0 (channels ch = c * nz + z on the in-plane grid), to
// the dipolar-field change dH:
//   dH[co](s) = sum_{o, ci} W[o][co][ci] X[ci](s + o)                          stencil branch
//             + sum_{kx<mx, ky} w_kx/(nx ny) Re(e^{i k.s} sum_ci R_k[co][ci] Xhat_k[ci])  spectral branch
// Both branches are evaluated as BF16 x BF16 -> FP32 GEMMs on the tcgen05
// tensor cores (operands staged in shared memory, accumulators in TMEM):
//   k_sur_xdft   Xhat over x: [(y, ch) rows] x [x] times the DFT rows [(kx, re/im)] x [x];
//   k_sur_ydft   DFT over y of the retained kx and the per-mode channel mixing,
//   k_sur_zrows  inverse DFT over y into each row's B tile (CUDA cores, FP32:
//                a few MFLOP);
//   k_sur_out    per 128-site M-tile: 25 shifted views of the staged halo tile
//                (one MMA per stencil offset, no im2col copy) plus the inverse
//                x-DFT [x] x [(kx, re/im)] times the mixed spectrum of this row,
//                FP32 epilogue adds H0 (or writes dH for training) and leaves
//                per-CTA residual sums for the schedule (k_sur_advance).
// Training kernels (FP32, CUDA cores): loss and its gradient G, the stencil
// gradient sum_s G[co](s) X[ci](s + o), the mode gradient
// w_kx/(nx ny) Ghat_k[co] conj(Xhat_k[ci]) and Adam.
#include "device.cuh"
#include "kparams.h"
#include "launch.h"
#include "umma.cuh"

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

namespace {

// After a completion wait gives up (SurK::wait_polls polls; the error flag
// is set) a second bounded wait lets the launch's own MMAs finish before the
// accumulator is read and its TMEM freed.
constexpr uint32_t kDrainPolls = 1u << 26;

__device__ __forceinline__ uint32_t pack2(float a, float b)
{
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
}

__device__ __forceinline__ uint8_t* align1k(uint8_t* p)
{
    const uintptr_t u = reinterpret_cast<uintptr_t>(p);
    return reinterpret_cast<uint8_t*>((u + 1023) & ~(uintptr_t)1023);
}

__device__ __forceinline__ const float* chan_plane(const float* const* a, int ch, int nz, size_t plane)
{
    return a[ch / nz] + (size_t)(ch % nz) * plane;
}

// ------------------------------------------------------------------ x-DFT
// grid (nx / 64, ny / (128 / CP)), 256 threads.  Xp[xc][kx][ch][y] (float2)
// = sum over this chunk's 64 x of (a - b)[ch](x, y) e^{-2 pi i kx x / nx}:
// D (128 x 32, TMEM) = A (rows (y, ch) x 64 x) B^T (rows (kx, re/im) x 64 x).
// When Xb is set, the BF16 input is also written as CP/8 planes of 8-channel
// site records, Xb[p][y][x][8] (16 bytes each), for the output kernel's halo.
constexpr int XK = 64;                    // x per CTA
template <int CP>
__global__ void __launch_bounds__(256) k_sur_xdft(SurK k, const float* a0, const float* a1, const float* a2,
                                                  const float* b0, const float* b1, const float* b2,
                                                  const __nv_bfloat16* __restrict__ F, float2* __restrict__ Xp,
                                                  uint4* __restrict__ Xb, int* err)
{
    if (k.skip_if && *k.skip_if) return;
    constexpr int RPT = 128 / CP;
    constexpr int QC = XK / 8;            // 16-byte chunks per row
    constexpr uint32_t SBO = QC * 128;
    extern __shared__ uint8_t smraw[];
    uint8_t* As = align1k(smraw);          // 128 rows x 64 K, 16 KB
    uint8_t* Bs = As + 128 * XK * 2;       // 32 rows x 64 K, 4 KB
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t slot;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int xc = blockIdx.x, x0 = xc * XK, y0 = blockIdx.y * RPT;
    const size_t plane = (size_t)k.nx * k.ny;
    if (tid == 0) umma::mbar_init(&bar, 1);
    if (warp == 0) {
        umma::tmem_alloc(&slot, 32);
        umma::tmem_relinquish();
    }
    // A: row m = (yl, ch), chunk q = 8 consecutive x; core (m/8, q) at (m/8)*SBO + q*128
    float4 va[4][2], vb[4][2];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int u = tid + 256 * i, m = u / QC, q = u % QC, yl = m / CP, ch = m % CP;
        va[i][0] = va[i][1] = vb[i][0] = vb[i][1] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (ch < k.C) {
            const size_t off = (size_t)(ch % k.nz) * plane + (size_t)(y0 + yl) * k.nx + x0 + q * 8;
            const int c = ch / k.nz;
            const float* pa = (c == 0 ? a0 : (c == 1 ? a1 : a2)) + off;
            va[i][0] = __ldg(reinterpret_cast<const float4*>(pa));
            va[i][1] = __ldg(reinterpret_cast<const float4*>(pa) + 1);
            if (b0) {
                const float* pb = (c == 0 ? b0 : (c == 1 ? b1 : b2)) + off;
                vb[i][0] = __ldg(reinterpret_cast<const float4*>(pb));
                vb[i][1] = __ldg(reinterpret_cast<const float4*>(pb) + 1);
            }
        }
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int u = tid + 256 * i, m = u / QC, q = u % QC;
        const float4 v0 = va[i][0], v1 = va[i][1], w0 = vb[i][0], w1 = vb[i][1];
        *reinterpret_cast<uint4*>(As + (m >> 3) * SBO + q * 128 + (m & 7) * 16) =
            make_uint4(pack2(v0.x - w0.x, v0.y - w0.y), pack2(v0.z - w0.z, v0.w - w0.w),
                       pack2(v1.x - w1.x, v1.y - w1.y), pack2(v1.z - w1.z, v1.w - w1.w));
    }
    {
        const int n = tid / QC, q = tid % QC;   // 32 rows x QC chunks = 256 units
        const uint4 v = __ldg(reinterpret_cast<const uint4*>(F + (size_t)n * k.nx + x0 + q * 8));
        *reinterpret_cast<uint4*>(Bs + (n >> 3) * SBO + q * 128 + (n & 7) * 16) = v;
    }
    umma::fence_async_smem();
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t taddr = slot;
    if (tid == 0) {
        const uint32_t id = umma::idesc_bf16_f32(128, 32);
        const uint32_t a = umma::smem_u32(As), b = umma::smem_u32(Bs);
#pragma unroll
        for (int ks = 0; ks < XK / 16; ks++)
            umma::mma_bf16(taddr, umma::desc_nosw(a + ks * 256, 128, SBO), umma::desc_nosw(b + ks * 256, 128, SBO),
                           id, ks > 0 ? 1u : 0u);
        umma::mma_commit(&bar);
    }
    if (Xb) {
        // records (p, yl, x): channels 8p .. 8p+7 of row yl, gathered from the A
        // tile (the MMAs only read it)
        constexpr int NPL = CP / 8;
        for (int u = tid; u < NPL * RPT * XK; u += 256) {
            const int x = u % XK, yl = (u / XK) % RPT, p = u / (XK * RPT);
            const int mr = yl * CP + 8 * p;    // first row of the record, a multiple of 8
            const uint8_t* src = As + (mr >> 3) * SBO + (x >> 3) * 128 + (x & 7) * 2;
            uint32_t w[4];
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const uint32_t lo = *reinterpret_cast<const uint16_t*>(src + (2 * e) * 16);
                const uint32_t hi = *reinterpret_cast<const uint16_t*>(src + (2 * e + 1) * 16);
                w[e] = lo | (hi << 16);
            }
            Xb[((size_t)p * k.ny + y0 + yl) * k.nx + x0 + x] = make_uint4(w[0], w[1], w[2], w[3]);
        }
    }
    if (warp == 0) {
        const bool ok = umma::mbar_wait(&bar, 0, k.wait_polls);
        if (!ok) {
            if (lane == 0) atomicOr(err, 1);
            umma::mbar_wait(&bar, 0, kDrainPolls);
        }
        umma::fence_before_sync();
    }
    __syncthreads();
    umma::fence_after_sync();
    // epilogue: warps w and w + 4 share TMEM lanes 32 (w % 4) .., columns 0-15 / 16-31
    float v[16];
    umma::tmem_ld16(taddr + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(16 * (warp >> 2)), v);
    const int m = 32 * (warp & 3) + lane, yl = m / CP, ch = m % CP;
    if (ch < k.C) {
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const int kx = 8 * (warp >> 2) + j;
            if (kx < k.mx)
                Xp[(((size_t)xc * k.mx + kx) * k.C + ch) * k.ny + y0 + yl] = make_float2(v[2 * j], v[2 * j + 1]);
        }
    }
    umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) umma::tmem_dealloc(taddr, 32);
}

// ------------------------------------------------------------------ y-DFT + mixing
// grid (mx, C), 256 threads: the x chunks' partial sums of line (kx, ci) are
// staged once, then Yh[kx][j][ci] = sum_y line[y] twy[j][y]
// (twy = e^{-2 pi i ky_j y / ny}).  When R is given, the last CTA of each kx
// to finish (cnt[kx] counts them and is reset) mixes the modes of that kx,
//   Zh[kx][j][co] = sum_ci R[kx][j][co][ci] Yh[kx][j][ci].
__global__ void __launch_bounds__(256) k_sur_ydft(SurK k, const float2* __restrict__ Xp,
                                                  const float2* __restrict__ twy, const float2* __restrict__ R,
                                                  float2* __restrict__ Yh, float2* __restrict__ Zh,
                                                  unsigned int* cnt)
{
    if (k.skip_if && *k.skip_if) return;
    extern __shared__ float2 line[];      // [ny]
    __shared__ int last;
    __shared__ float2 zh[16 * 32];        // [j][co] of this kx
    const int kx = blockIdx.x, ci = blockIdx.y, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int y = threadIdx.x; y < k.ny; y += blockDim.x) {
        float2 acc = make_float2(0.f, 0.f);
        for (int xc = 0; xc < k.nxc; xc++) {
            const float2 a = Xp[(((size_t)xc * k.mx + kx) * k.C + ci) * k.ny + y];
            acc.x += a.x;
            acc.y += a.y;
        }
        line[y] = acc;
    }
    __syncthreads();
    for (int j = warp; j < k.my; j += 8) {
        float re = 0.f, im = 0.f;
        // twiddles by recurrence from this lane's first one: t(y + 32) = t(y) t(32)
        float2 t = lane < k.ny ? __ldg(twy + (size_t)j * k.ny + lane) : make_float2(1.f, 0.f);
        const float2 st = __ldg(twy + (size_t)j * k.ny + (32 % k.ny));
        for (int y = lane; y < k.ny; y += 32) {
            const float2 a = line[y];
            re += a.x * t.x - a.y * t.y;
            im += a.x * t.y + a.y * t.x;
            t = make_float2(t.x * st.x - t.y * st.y, t.x * st.y + t.y * st.x);
        }
        for (int s = 16; s > 0; s >>= 1) {
            re += __shfl_xor_sync(0xffffffffu, re, s);
            im += __shfl_xor_sync(0xffffffffu, im, s);
        }
        if (lane == 0) Yh[((size_t)kx * k.my + j) * k.C + ci] = make_float2(re, im);
    }
    if (!R) return;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(cnt + kx, 1u) == (unsigned)(k.C - 1);
    __syncthreads();
    if (!last) return;
    __threadfence();
    for (int o = threadIdx.x; o < k.my * k.C; o += blockDim.x) {
        const int j = o / k.C, co = o % k.C;
        const float2* r = R + (((size_t)kx * k.my + j) * k.C + co) * k.C;
        const float2* yv = Yh + ((size_t)kx * k.my + j) * k.C;
        float re = 0.f, im = 0.f;
        for (int c2 = 0; c2 < k.C; c2++) {
            const float2 a = __ldg(r + c2), b = __ldcg(yv + c2);
            re += a.x * b.x - a.y * b.y;
            im += a.x * b.y + a.y * b.x;
        }
        zh[o] = make_float2(re, im);
    }
    if (threadIdx.x == 0) cnt[kx] = 0u;
    __syncthreads();
    for (int o = threadIdx.x; o < k.my * k.C; o += blockDim.x) Zh[(size_t)kx * k.my * k.C + o] = zh[o];
}

// ------------------------------------------------------------------ inverse y-DFT
// grid ny / ZR, 256 threads.  For each of its rows the B tile of the output
// GEMM: Zb[y][co][2 kx + ri] = w_kx/(nx ny) sum_j Zh[kx][j][co] e^{+2 pi i ky_j y / ny}
// in the canonical K-major layout (core (co/8, k/8) at (co/8)*512 + (k/8)*128).
constexpr int ZR = 4;
__global__ void __launch_bounds__(256) k_sur_zrows(SurK k, const float2* __restrict__ Zh,
                                                   const float2* __restrict__ twy, uint8_t* __restrict__ Zb)
{
    if (k.skip_if && *k.skip_if) return;
    extern __shared__ float2 zs[];        // [mx][my][C], then [my][ZR] twiddles
    float2* tw = zs + (size_t)k.mx * k.my * k.C;
    for (int o = threadIdx.x; o < k.mx * k.my * k.C; o += blockDim.x) zs[o] = __ldg(Zh + o);
    for (int o = threadIdx.x; o < k.my * ZR; o += blockDim.x)
        tw[o] = __ldg(twy + (size_t)(o / ZR) * k.ny + blockIdx.x * ZR + o % ZR);
    __syncthreads();
    const float inv = 1.f / ((float)k.nx * (float)k.ny);
    const int tile = k.CP * 64;
    for (int o = threadIdx.x; o < ZR * k.C * k.mx; o += blockDim.x) {
        const int co = o % k.C, kx = (o / k.C) % k.mx, yl = o / (k.mx * k.C);
        const int y = blockIdx.x * ZR + yl;
        float re = 0.f, im = 0.f;
#pragma unroll 4
        for (int j = 0; j < k.my; j++) {
            const float2 z = zs[((size_t)kx * k.my + j) * k.C + co];
            const float2 w = tw[j * ZR + yl];   // conjugated: e^{+i ...}
            re += z.x * w.x + z.y * w.y;
            im += z.y * w.x - z.x * w.y;
        }
        const float s = (kx == 0 ? 1.f : 2.f) * inv;
        const int kk = 2 * kx;
        *reinterpret_cast<uint32_t*>(Zb + (size_t)y * tile + (co >> 3) * 512 + (kk >> 3) * 128 + (co & 7) * 16 +
                                     (kk & 7) * 2) = pack2(s * re, s * im);
    }
}

// ------------------------------------------------------------------ output GEMM
// grid (nx / TW, ny), 256 threads.  Halo planes hold X as BF16, 8 channels per
// 16-byte site record: plane p, row r (y - rad .. y + rad), site s (x0 - rad
// .. x0 + TW + rad).  The stencil operand for offset (oy, ox) of M-tile t is
// the view starting at site (128 t + ox + rad) of row (oy + rad): rows 16 B
// apart (SBO 128 per 8 sites), the two 8-channel planes LBO apart.
struct OutArgs {
    const uint4* Xb;        // BF16 input records [p][y][x] written by the x-DFT
    const float* h0[3];     // H0 (mode 0)
    float* out[3];          // H (mode 0) or dH (mode 1)
    const uint8_t* Wc;      // stencil weights, canonical B tiles per offset
    const uint8_t* Fc;      // inverse x-DFT rows, canonical A layout over all nx
    const uint8_t* Zb;      // per-row B tiles of the mixed spectrum
    SurDev* dev;
    double* part;           // mode 0: per-CTA sums of dH^2 and H^2
    int* err;
    int mode;               // 0: out = h0 + ratio * dH; 1: out = dH
};

// One bulk copy global -> shared of `bytes` (a multiple of 16, both
// addresses 16-byte aligned), completing on the mbarrier bar.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     umma::smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(umma::smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(umma::smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// Output rows per CTA: the rows' MMAs are issued together into one TMEM
// accumulator per row and complete on one barrier, and the weights and
// inverse x-DFT rows are staged once for all of them; warp w takes row w / 4
// in the epilogue (TMEM lanes 32 (w % 4) ..).  Per launch of the 512x512x4
// film's radius-3 network: 1, 2, 4 rows per CTA gave surrogate steps of
// 115.8, 107.1, 104.8 us (k = 5), the same outputs bit for bit.
constexpr int SUR_ROWS = 4;

// grid (nx / 128, ny / SUR_ROWS), 128 SUR_ROWS threads (thread t owns output
// site x0 + t % 128 of row y0 + t / 128, TMEM lane t % 128).  Halo planes
// [p][DIA + SUR_ROWS - 1 rows][HW sites] of 16-byte records: the stencil
// operand of row j and offset (oy, ox) is the view starting at record ox of
// halo row j + oy.
template <int CP, int RAD>
__global__ void __launch_bounds__(128 * SUR_ROWS) k_sur_out(SurK k, OutArgs q)
{
    pdl_trigger();
    pdl_wait();
    if (k.skip_if && *k.skip_if) return;
    constexpr int NR = SUR_ROWS;
    constexpr int NPL = CP / 8, DIA = 2 * RAD + 1, HW = 128 + 2 * RAD, HR = DIA + NR - 1;
    constexpr uint32_t PL = (HR * HW * 16 + 127) & ~127u;      // bytes per halo plane
    constexpr uint32_t WT = CP * CP * 2;                        // bytes per offset tile
    constexpr uint32_t ZT = CP * 64;                            // bytes per row's spectrum tile
    constexpr uint32_t NCOL = NR * CP < 32 ? 32 : NR * CP;      // TMEM columns: one accumulator per row
    extern __shared__ uint8_t smraw[];
    uint8_t* Hs = align1k(smraw);
    uint8_t* Ws = Hs + NPL * PL;
    uint8_t* Fs = Ws + DIA * DIA * WT;                          // 128 x 32 BF16
    uint8_t* Zs = Fs + 8192;                                    // [NR] CP x 32 BF16
    __shared__ __align__(8) uint64_t bar;
    __shared__ __align__(8) uint64_t lbar;   // the staged operands' bulk copies
    __shared__ uint32_t slot;
    __shared__ double red[2][4 * NR];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int y0 = blockIdx.y * NR, x0 = blockIdx.x * 128;
    const int row = tid >> 7, y = y0 + row;
    if (tid == 0) {
        umma::mbar_init(&bar, 1);
        umma::mbar_init(&lbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (warp == 0) {
        umma::tmem_alloc(&slot, NCOL);
        umma::tmem_relinquish();
    }
    __syncthreads();   // the barriers' initialisation
    // operands by bulk copies issued by warp 0, on lbar: the halo records
    // (p, r, s) = 8 channels at (x0 + s - RAD, y0 + r - RAD), periodic, as
    // three runs per halo row (the RAD records left of x0 and right of
    // x0 + 127, wrapped at the lattice's x edges, and the 128 between), the
    // stencil weights, the CTA's inverse x-DFT rows and the rows' spectrum tiles
    constexpr uint32_t HALO = NPL * HR * HW * 16;
    constexpr uint32_t TX = HALO + DIA * DIA * WT + 8192 + NR * ZT;
    if (warp == 0) {
        if (lane == 0) mbar_expect_tx(&lbar, TX);
        __syncwarp();
        for (int it = lane; it < NPL * HR * 3 + 3; it += 32) {
            if (it < NPL * HR * 3) {
                const int piece = it % 3, r = (it / 3) % HR, p = it / (3 * HR);
                int yy = (y0 + r - RAD) % k.ny;
                yy = yy < 0 ? yy + k.ny : yy;
                const uint4* src = q.Xb + ((size_t)p * k.ny + yy) * k.nx;
                uint8_t* dst = Hs + p * PL + r * HW * 16;
                if (piece == 0 && RAD > 0) {
                    const int xx = x0 - RAD < 0 ? x0 - RAD + k.nx : x0 - RAD;
                    bulk_g2s(dst, src + xx, RAD * 16, &lbar);
                } else if (piece == 1) {
                    bulk_g2s(dst + RAD * 16, src + x0, 128 * 16, &lbar);
                } else if (piece == 2 && RAD > 0) {
                    const int xx = x0 + 128 >= k.nx ? x0 + 128 - k.nx : x0 + 128;
                    bulk_g2s(dst + (RAD + 128) * 16, src + xx, RAD * 16, &lbar);
                }
            } else if (it == NPL * HR * 3) {
                bulk_g2s(Ws, q.Wc, DIA * DIA * WT, &lbar);
            } else if (it == NPL * HR * 3 + 1) {
                bulk_g2s(Fs, q.Fc + (size_t)x0 * 64, 8192, &lbar);
            } else {
                bulk_g2s(Zs, q.Zb + (size_t)y0 * ZT, NR * ZT, &lbar);
            }
        }
    }
    // this thread's H0 while the copies land
    const int x = x0 + (tid & 127);
    float h0v[CP];
#pragma unroll
    for (int co = 0; co < CP; co++) {
        h0v[co] = 0.f;
        if (q.mode == 0 && co < k.C) {
            const int c = co / k.nz;
            const float* hp = c == 0 ? q.h0[0] : (c == 1 ? q.h0[1] : q.h0[2]);
            h0v[co] = __ldg(hp + ((size_t)(co % k.nz) * k.ny + y) * k.nx + x);
        }
    }
    // the operands landed (a wait that gives up flags the error and waits,
    // bounded again, for the copies before their buffers are read)
    if (!umma::mbar_wait(&lbar, 0, k.wait_polls)) {
        if (lane == 0) atomicOr(q.err, 1);
        umma::mbar_wait(&lbar, 0, kDrainPolls);
    }
    umma::fence_async_smem();
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t taddr = slot;
    if (warp == 0) {
        if (lane == 0) {
            const uint32_t id = umma::idesc_bf16_f32(128, CP);
            const uint32_t hs = umma::smem_u32(Hs), ws = umma::smem_u32(Ws), fs = umma::smem_u32(Fs),
                           zs = umma::smem_u32(Zs);
            // each row's accumulator takes its MMAs in the order of a
            // one-row tile (offsets, then the spectral pair); the rows
            // alternate per offset so that each weight tile's descriptor
            // serves every row at once
#pragma unroll
            for (int o = 0; o < DIA * DIA; o++) {
#pragma unroll
                for (int kk = 0; kk < CP / 16; kk++) {
                    const uint64_t bd = umma::desc_nosw(ws + o * WT + kk * 256, 128, (CP / 8) * 128);
#pragma unroll
                    for (int j = 0; j < NR; j++) {
                        const uint32_t site = (uint32_t)((j + o / DIA) * HW + o % DIA) * 16;
                        umma::mma_bf16(taddr + (uint32_t)(j * CP), umma::desc_nosw(hs + 2 * kk * PL + site, PL, 128),
                                       bd, id, (o | kk) ? 1u : 0u);
                    }
                }
            }
#pragma unroll
            for (int ks = 0; ks < 2; ks++)
#pragma unroll
                for (int j = 0; j < NR; j++)
                    umma::mma_bf16(taddr + (uint32_t)(j * CP), umma::desc_nosw(fs + ks * 256, 128, 512),
                                   umma::desc_nosw(zs + j * ZT + ks * 256, 128, 512), id, 1u);
            umma::mma_commit(&bar);
        }
        __syncwarp();
        const bool ok = umma::mbar_wait(&bar, 0, k.wait_polls);
        if (!ok) {
            if (lane == 0) atomicOr(q.err, 1);
            umma::mbar_wait(&bar, 0, kDrainPolls);
        }
        umma::fence_before_sync();
    }
    __syncthreads();
    umma::fence_after_sync();
    double s_dh = 0.0, s_h = 0.0;
#pragma unroll
    for (int cb = 0; cb < CP / 16; cb++) {
        float v[16];
        umma::tmem_ld16(taddr + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(row * CP + 16 * cb), v);
#pragma unroll
        for (int j = 0; j < 16; j++) {
            const int co = 16 * cb + j;
            if (co >= k.C) continue;
            const size_t idx = ((size_t)(co % k.nz) * k.ny + y) * k.nx + x;
            const int c = co / k.nz;
            float* o = c == 0 ? q.out[0] : (c == 1 ? q.out[1] : q.out[2]);
            if (q.mode == 0) {
                const float dh = k.ratio * v[j];
                const float h = h0v[co] + dh;
                o[idx] = h;
                s_dh += (double)dh * dh;
                s_h += (double)h * h;
            } else {
                o[idx] = v[j];
            }
        }
    }
    umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) umma::tmem_dealloc(taddr, NCOL);
    if (q.mode == 1 || !q.part) return;
    // residual statistics: this CTA's sums (k_sur_advance reduces them)
    for (int s = 16; s > 0; s >>= 1) {
        s_dh += __shfl_xor_sync(0xffffffffu, s_dh, s);
        s_h += __shfl_xor_sync(0xffffffffu, s_h, s);
    }
    if (lane == 0) { red[0][warp] = s_dh; red[1][warp] = s_h; }
    __syncthreads();
    if (tid == 0) {
        double a = 0, b = 0;
        for (int w = 0; w < 4 * NR; w++) { a += red[0][w]; b += red[1][w]; }
        const size_t cta = (size_t)blockIdx.y * gridDim.x + blockIdx.x;
        q.part[2 * cta] = a;
        q.part[2 * cta + 1] = b;
    }
}

// ------------------------------------------------------------------ schedule
// After an exact evaluation: m0 = m, H0 = H, the cycle restarts.
__global__ void __launch_bounds__(256) k_sur_snapshot(SurDev* d, int n, const float* m0_, const float* m1_,
                                                      const float* m2_, const float* h0_, const float* h1_,
                                                      const float* h2_, float* sm0, float* sm1, float* sm2,
                                                      float* sh0, float* sh1, float* sh2)
{
    if (!d->exact) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) { d->cycle = 0; d->nexact += 1; }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        sm0[i] = m0_[i]; sm1[i] = m1_[i]; sm2[i] = m2_[i];
        sh0[i] = h0_[i]; sh1[i] = h1_[i]; sh2[i] = h2_[i];
    }
}

// End of a step (one CTA of 256 threads).  After a surrogate step: the
// residual check, bound = eps |dH| / |H| from the output kernel's per-CTA
// sums, fails when bound > tol.  The next step is exact every k steps,
// after a failed check, and always when the bound is zero.
__global__ void __launch_bounds__(256) k_sur_advance(SurDev* d, const double* part, int np)
{
    pdl_wait();
    __shared__ double red[2][8];
    if (!d->exact && part) {
        double a = 0.0, b = 0.0;
        for (int i = threadIdx.x; i < np; i += blockDim.x) {
            a += part[2 * i];
            b += part[2 * i + 1];
        }
        for (int s = 16; s > 0; s >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, s);
            b += __shfl_xor_sync(0xffffffffu, b, s);
        }
        if ((threadIdx.x & 31) == 0) { red[0][threadIdx.x >> 5] = a; red[1][threadIdx.x >> 5] = b; }
        __syncthreads();
        if (threadIdx.x == 0) {
            double sdh = 0.0, sh = 0.0;
            for (int w = 0; w < 8; w++) { sdh += red[0][w]; sh += red[1][w]; }
            const float bound = sh > 0 ? (float)((double)d->eps * sqrt(sdh / sh)) : 0.f;
            d->last_bound = bound;
            d->nsur += 1;
            if (bound > d->tol) {
                d->fail = 1;        // the next step evaluates the exact convolution
                d->nfail += 1;
            }
        }
    }
    if (threadIdx.x == 0) {
        d->cycle += 1;
        d->exact = (d->cycle >= d->k || d->fail || !(d->tol > 0.f)) ? 1 : 0;
        d->fail = 0;
    }
}

// ------------------------------------------------------------------ training
// G = 2 (P - T) with T = Hx - H0 (H0 may be null: T = Hx); per-block FP64
// partials of sum T^2, sum (P - T)^2 and sum Hx^2.
__global__ void __launch_bounds__(256) k_sur_loss(int n3, const float* P0, const float* P1, const float* P2,
                                                  const float* X0, const float* X1, const float* X2,
                                                  const float* H0, const float* H1, const float* H2, float* G0,
                                                  float* G1, float* G2, int n, double* part)
{
    double st = 0.0, se = 0.0, sx = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x) {
        const int c = i / n, j = i % n;
        const float* P = c == 0 ? P0 : (c == 1 ? P1 : P2);
        const float* X = c == 0 ? X0 : (c == 1 ? X1 : X2);
        const float* H = c == 0 ? H0 : (c == 1 ? H1 : H2);
        float* G = c == 0 ? G0 : (c == 1 ? G1 : G2);
        const float x = X[j];
        const float t = H ? x - H[j] : x;
        const float e = P[j] - t;
        G[j] = 2.f * e;
        st += (double)t * t;
        se += (double)e * e;
        sx += (double)x * x;
    }
    __shared__ double sh[3][8];
    for (int s = 16; s > 0; s >>= 1) {
        st += __shfl_xor_sync(0xffffffffu, st, s);
        se += __shfl_xor_sync(0xffffffffu, se, s);
        sx += __shfl_xor_sync(0xffffffffu, sx, s);
    }
    if ((threadIdx.x & 31) == 0) {
        sh[0][threadIdx.x >> 5] = st;
        sh[1][threadIdx.x >> 5] = se;
        sh[2][threadIdx.x >> 5] = sx;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double v = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) v += sh[threadIdx.x][w];
        part[blockIdx.x * 3 + threadIdx.x] = v;
    }
}

// Stencil gradient partials: one CTA per (row block of RB rows, 128-wide x
// chunk); part[cta][(o * C + co) * C + ci] = sum over its sites of
// G[co](s) X[ci](s + o), X = a - b in FP32.
constexpr int GW_RB = 4;
__global__ void __launch_bounds__(256) k_sur_grad_w(SurK k, const float* a0, const float* a1, const float* a2,
                                                    const float* b0, const float* b1, const float* b2,
                                                    const float* g0, const float* g1, const float* g2,
                                                    float* part)
{
    extern __shared__ float gsm[];
    const int rad = k.rad, dia = 2 * rad + 1, C = k.C;
    const int hw = 128 + 2 * rad, hr = GW_RB + 2 * rad;
    float* Xs = gsm;                        // [C][hr][hw]
    float* Gs = Xs + (size_t)C * hr * hw;   // [C][RB][128]
    const int x0 = blockIdx.x * 128, y0 = blockIdx.y * GW_RB;
    const size_t plane = (size_t)k.nx * k.ny;
    const float* A[3] = {a0, a1, a2};
    const float* B[3] = {b0, b1, b2};
    const float* Gp[3] = {g0, g1, g2};
    for (int u = threadIdx.x; u < C * hr * hw; u += blockDim.x) {
        const int s = u % hw, r = (u / hw) % hr, ch = u / (hw * hr);
        int yy = y0 + r - rad, xx = x0 + s - rad;
        yy = ((yy % k.ny) + k.ny) % k.ny;
        xx = ((xx % k.nx) + k.nx) % k.nx;
        const size_t off = (size_t)yy * k.nx + xx;
        float v = chan_plane(A, ch, k.nz, plane)[off];
        if (b0) v -= chan_plane(B, ch, k.nz, plane)[off];
        Xs[u] = v;
    }
    for (int u = threadIdx.x; u < C * GW_RB * 128; u += blockDim.x) {
        const int s = u % 128, r = (u / 128) % GW_RB, ch = u / (128 * GW_RB);
        Gs[u] = chan_plane(Gp, ch, k.nz, plane)[(size_t)(y0 + r) * k.nx + x0 + s];
    }
    __syncthreads();
    const int nout = dia * dia * C * C;
    float* dst = part + (size_t)(blockIdx.y * gridDim.x + blockIdx.x) * nout;
    for (int o = threadIdx.x; o < nout; o += blockDim.x) {
        const int ci = o % C, co = (o / C) % C, off = o / (C * C);
        const int oy = off / dia, ox = off % dia;
        float acc = 0.f;
        for (int r = 0; r < GW_RB; r++) {
            const float* g = Gs + ((size_t)co * GW_RB + r) * 128;
            const float* x = Xs + ((size_t)ci * hr + r + oy) * hw + ox;
            for (int s = 0; s < 128; s++) acc += g[s] * x[s];
        }
        dst[o] = acc;
    }
}

// out[j] = sum_b part[b * n + j]
__global__ void k_sur_colsum(const float* part, int nb, int n, float* out)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    double s = 0;
    for (int b = 0; b < nb; b++) s += part[(size_t)b * n + j];
    out[j] = (float)s;
}

// dR[kx][j][co][ci] = w_kx/(nx ny) Ghat[kx][j][co] conj(Xhat[kx][j][ci])
__global__ void k_sur_grad_r(SurK k, const float2* Gh, const float2* Xh, float2* dR)
{
    const int total = k.mx * k.my * k.C * k.C;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const int ci = i % k.C, co = (i / k.C) % k.C, mj = i / (k.C * k.C);
    const int kx = mj / k.my;
    const float s = (kx == 0 ? 1.f : 2.f) / ((float)k.nx * (float)k.ny);
    const float2 g = Gh[(size_t)mj * k.C + co], x = Xh[(size_t)mj * k.C + ci];
    dR[i] = make_float2(s * (g.x * x.x + g.y * x.y), s * (g.y * x.x - g.x * x.y));
}

// Adam on the FP32 master parameters (stencil, then modes as real pairs);
// gradients scaled by 1 / sum T^2 (gscale[0]).  Writes the BF16 stencil
// tiles in their canonical B layout.
struct AdamArgs {
    float* w;            // [dia^2][C][C]
    float* r;            // [mx][my][C][C][2]
    const float* gw;
    const float* gr;
    float* mw; float* vw; float* mr; float* vr;
    uint8_t* wc;         // canonical BF16 tiles
    const double* sums;  // sum T^2
    float lr, b1, b2, eps, bc1, bc2;
    int nw, nr, C, CP;
};

__global__ void k_sur_adam(AdamArgs a)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const double st = a.sums[0];
    const float sc = st > 0 ? (float)(1.0 / st) : 0.f;
    if (i < a.nw) {
        const float g = a.gw[i] * sc;
        const float m = a.b1 * a.mw[i] + (1.f - a.b1) * g;
        const float v = a.b2 * a.vw[i] + (1.f - a.b2) * g * g;
        a.mw[i] = m;
        a.vw[i] = v;
        const float w = a.w[i] - a.lr * (m / a.bc1) / (sqrtf(v / a.bc2) + a.eps);
        a.w[i] = w;
        const int ci = i % a.C, co = (i / a.C) % a.C, o = i / (a.C * a.C);
        const int CP = a.CP;
        uint8_t* tile = a.wc + (size_t)o * CP * CP * 2;
        const size_t byte = (size_t)(co >> 3) * (CP / 8) * 128 + (ci >> 3) * 128 + (co & 7) * 16 + (ci & 7) * 2;
        *reinterpret_cast<__nv_bfloat16*>(tile + byte) = __float2bfloat16_rn(w);
    } else if (i < a.nw + a.nr) {
        const int j = i - a.nw;
        const float g = a.gr[j] * sc;
        const float m = a.b1 * a.mr[j] + (1.f - a.b1) * g;
        const float v = a.b2 * a.vr[j] + (1.f - a.b2) * g * g;
        a.mr[j] = m;
        a.vr[j] = v;
        a.r[j] -= a.lr * (m / a.bc1) / (sqrtf(v / a.bc2) + a.eps);
    }
}

} // namespace

namespace mlb {

size_t sur_out_smem(int CP, int rad)
{
    const int dia = 2 * rad + 1, hw = 128 + 2 * rad;
    const size_t pl = (size_t)(((dia + SUR_ROWS - 1) * hw * 16 + 127) & ~127);
    return 1024 + (CP / 8) * pl + (size_t)dia * dia * CP * CP * 2 + 8192 + (size_t)SUR_ROWS * CP * 64;
}

int sur_out_ctas(int nx, int ny) { return (nx / 128) * (ny / SUR_ROWS); }

template <int CP, int RAD>
static cudaError_t out_attr()
{
    return cudaFuncSetAttribute(k_sur_out<CP, RAD>, cudaFuncAttributeMaxDynamicSharedMemorySize, 226 * 1024);
}

size_t sur_gw_smem(int C, int rad)
{
    const int hw = 128 + 2 * rad, hr = GW_RB + 2 * rad;
    return sizeof(float) * ((size_t)C * hr * hw + (size_t)C * GW_RB * 128);
}

cudaError_t sur_configure()
{
    cudaError_t e;
    const int big = 226 * 1024;   // the static shared memory of these kernels is under 1 KB
    if ((e = out_attr<16, 0>()) || (e = out_attr<16, 1>()) || (e = out_attr<16, 2>()) || (e = out_attr<16, 3>())) return e;
    if ((e = out_attr<32, 0>()) || (e = out_attr<32, 1>()) || (e = out_attr<32, 2>()) || (e = out_attr<32, 3>())) return e;
    if ((e = cudaFuncSetAttribute(k_sur_xdft<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, big))) return e;
    if ((e = cudaFuncSetAttribute(k_sur_xdft<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, big))) return e;
    if ((e = cudaFuncSetAttribute(k_sur_ydft, cudaFuncAttributeMaxDynamicSharedMemorySize, 128 * 1024))) return e;
    if ((e = cudaFuncSetAttribute(k_sur_zrows, cudaFuncAttributeMaxDynamicSharedMemorySize, 128 * 1024))) return e;
    return cudaFuncSetAttribute(k_sur_grad_w, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
}

cudaError_t launch_sur_xdft(const SurK& k, const float* const a[3], const float* const b[3],
                            const __nv_bfloat16* F, float2* Xp, uint4* Xb, int* err, cudaStream_t st)
{
    Prof pf("k_sur_xdft", st);
    const size_t sm = 1024 + 128 * XK * 2 + 32 * XK * 2;
    dim3 g(k.nx / XK, k.ny / (128 / k.CP));
    const float* bb[3] = {b ? b[0] : nullptr, b ? b[1] : nullptr, b ? b[2] : nullptr};
    if (k.CP == 16)
        k_sur_xdft<16><<<g, 256, sm, st>>>(k, a[0], a[1], a[2], bb[0], bb[1], bb[2], F, Xp, Xb, err);
    else
        k_sur_xdft<32><<<g, 256, sm, st>>>(k, a[0], a[1], a[2], bb[0], bb[1], bb[2], F, Xp, Xb, err);
    return cudaGetLastError();
}

size_t sur_ydft_smem(const SurK& k) { return sizeof(float2) * (size_t)k.ny; }

cudaError_t launch_sur_ydft(const SurK& k, const float2* Xp, const float2* twy, const float2* R, float2* Yh,
                            float2* Zh, unsigned int* cnt, cudaStream_t st)
{
    Prof pf("k_sur_ydft", st);
    k_sur_ydft<<<dim3(k.mx, k.C), 256, sur_ydft_smem(k), st>>>(k, Xp, twy, R, Yh, Zh, cnt);
    return cudaGetLastError();
}

cudaError_t launch_sur_zrows(const SurK& k, const float2* Zh, const float2* twy, uint8_t* Zb, cudaStream_t st)
{
    Prof pf("k_sur_zrows", st);
    k_sur_zrows<<<k.ny / ZR, 256, sizeof(float2) * (k.mx * k.my * k.C + k.my * ZR), st>>>(k, Zh, twy, Zb);
    return cudaGetLastError();
}


cudaError_t launch_sur_out(const SurK& k, const uint4* Xb, const float* const h0[3], float* const out[3],
                           const uint8_t* Wc, const uint8_t* Fc, const uint8_t* Zb, SurDev* dev, double* part,
                           int* err, int mode, cudaStream_t st)
{
    Prof pf("k_sur_out", st);
    OutArgs q;
    memset(&q, 0, sizeof(q));
    q.Xb = Xb;
    for (int c = 0; c < 3; c++) {
        q.h0[c] = h0 ? h0[c] : nullptr;
        q.out[c] = out[c];
    }
    q.Wc = Wc; q.Fc = Fc; q.Zb = Zb; q.dev = dev; q.part = part; q.err = err; q.mode = mode;
    dim3 g(k.nx / 128, k.ny / SUR_ROWS);
    const size_t sm = sur_out_smem(k.CP, k.rad);
    cudaError_t e = cudaSuccess;
#define MLB_SUR_OUT(CPV, RV) launch_pdl(k_sur_out<CPV, RV>, g, dim3(128 * SUR_ROWS), sm, st, k, q)
    if (k.CP == 16) {
        switch (k.rad) {
        case 0: e = MLB_SUR_OUT(16, 0); break;
        case 1: e = MLB_SUR_OUT(16, 1); break;
        case 2: e = MLB_SUR_OUT(16, 2); break;
        default: e = MLB_SUR_OUT(16, 3); break;
        }
    } else {
        switch (k.rad) {
        case 0: e = MLB_SUR_OUT(32, 0); break;
        case 1: e = MLB_SUR_OUT(32, 1); break;
        case 2: e = MLB_SUR_OUT(32, 2); break;
        default: e = MLB_SUR_OUT(32, 3); break;
        }
    }
#undef MLB_SUR_OUT
    return e != cudaSuccess ? e : cudaGetLastError();
}

cudaError_t launch_sur_snapshot(SurDev* d, int n, const float* const m[3], const float* const h[3],
                                float* const sm[3], float* const sh[3], cudaStream_t st)
{
    Prof pf("k_sur_snapshot", st);
    const int nb = (int)std::min<long long>((n + 255) / 256, 148 * 8);
    k_sur_snapshot<<<nb, 256, 0, st>>>(d, n, m[0], m[1], m[2], h[0], h[1], h[2], sm[0], sm[1], sm[2],
                                                    sh[0], sh[1], sh[2]);
    return cudaGetLastError();
}

cudaError_t launch_sur_advance(SurDev* d, const double* part, int np, cudaStream_t st)
{
    return launch_pdl(k_sur_advance, dim3(1), dim3(256), 0, st, d, part, np);
}

cudaError_t launch_sur_loss(int n, const float* const P[3], const float* const X[3], const float* const H0[3],
                            float* const G[3], double* part, int nb, double* out, cudaStream_t st)
{
    const float* h[3] = {H0 ? H0[0] : nullptr, H0 ? H0[1] : nullptr, H0 ? H0[2] : nullptr};
    k_sur_loss<<<nb, 256, 0, st>>>(3 * n, P[0], P[1], P[2], X[0], X[1], X[2], h[0], h[1], h[2], G[0], G[1], G[2], n,
                                   part);
    return launch_partial_final(part, nb, 3, out, st);
}

cudaError_t launch_sur_grad_w(const SurK& k, const float* const a[3], const float* const b[3],
                              const float* const g[3], float* part, float* gw, cudaStream_t st)
{
    dim3 grid(k.nx / 128, k.ny / GW_RB);
    const float* bb[3] = {b ? b[0] : nullptr, b ? b[1] : nullptr, b ? b[2] : nullptr};
    k_sur_grad_w<<<grid, 256, sur_gw_smem(k.C, k.rad), st>>>(k, a[0], a[1], a[2], bb[0], bb[1], bb[2], g[0], g[1],
                                                             g[2], part);
    const int dia = 2 * k.rad + 1;
    const int n = dia * dia * k.C * k.C;
    k_sur_colsum<<<(n + 255) / 256, 256, 0, st>>>(part, (int)(grid.x * grid.y), n, gw);
    return cudaGetLastError();
}

cudaError_t launch_sur_grad_r(const SurK& k, const float2* Gh, const float2* Xh, float2* dR, cudaStream_t st)
{
    const int total = k.mx * k.my * k.C * k.C;
    k_sur_grad_r<<<(total + 255) / 256, 256, 0, st>>>(k, Gh, Xh, dR);
    return cudaGetLastError();
}

cudaError_t launch_sur_adam(float* w, float* r, const float* gw, const float* gr, float* mw, float* vw, float* mr,
                            float* vr, uint8_t* wc, const double* sums, float lr, int step, int nw, int nr, int C,
                            int CP, cudaStream_t st)
{
    AdamArgs a;
    a.w = w; a.r = r; a.gw = gw; a.gr = gr; a.mw = mw; a.vw = vw; a.mr = mr; a.vr = vr; a.wc = wc; a.sums = sums;
    a.lr = lr; a.b1 = 0.9f; a.b2 = 0.999f; a.eps = 1e-8f;
    a.bc1 = 1.f - powf(0.9f, (float)step);
    a.bc2 = 1.f - powf(0.999f, (float)step);
    a.nw = nw; a.nr = nr; a.C = C; a.CP = CP;
    k_sur_adam<<<(nw + nr + 255) / 256, 256, 0, st>>>(a);
    return cudaGetLastError();
}

} // namespace mlb
