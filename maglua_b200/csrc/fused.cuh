// fused.cuh -- one site of the fused step (field terms + LLG update) for
// uniform-parameter FP32 systems, shared by the fused-step kernels
// (conv_fast.cu) and the surrogate's output kernel (surrogate.cu).
#pragma once
#include "device.cuh"
#include "kparams.h"

#include <math.h>
#include <stdint.h>

// The step block's per-step values (swept field, thermal counter) read once
// per thread instead of once per site: the same values, so the same results.
template <typename R>
__device__ __forceinline__ FastKT<R> fastk_resolved(const FastKT<R>& F)
{
    FastKT<R> G = F;
    if (F.Bdev) {
        G.B[0] = (R)F.Bdev[0]; G.B[1] = (R)F.Bdev[1]; G.B[2] = (R)F.Bdev[2];
        G.Bdev = nullptr;
    }
    if (F.dctr) {
        G.counter = F.counter + *F.dctr;
        G.dctr = nullptr;
    }
    return G;
}

// Cubic anisotropy field of one axis set at the reduced moment (sx, sy, sz)
// = S / ms (M/cpu/anisotropy/..._cubic.cpp:308-390): axes n[0..2], n[3..5],
// n[6..8], constants K[0..2]; quirk keeps (n2s2 + n3s3) in the first K1 term.
template <typename R>
__device__ __forceinline__ void cubic_field(R sx, R sy, R sz, const R* n, const R* K, int quirk, R& hx, R& hy,
                                            R& hz)
{
    const R n1s = n[0] * sx + n[1] * sy + n[2] * sz;
    const R n2s = n[3] * sx + n[4] * sy + n[5] * sz;
    const R n3s = n[6] * sx + n[7] * sy + n[8] * sz;
    const R n1s2 = n1s * n1s, n2s2 = n2s * n2s, n3s2 = n3s * n3s;
    const R n1s3 = n1s2 * n1s, n2s3 = n2s2 * n2s, n3s3 = n3s2 * n3s;
    const R n1s4 = n1s2 * n1s2, n2s4 = n2s2 * n2s2, n3s4 = n3s2 * n3s2;
    const R q = quirk ? n3s3 : n3s2;
    const R a1 = (R)2 * K[0] * n1s * (n2s2 + q), a2 = (R)2 * K[0] * n2s * (n1s2 + n3s2), a3 = (R)2 * K[0] * n3s * (n1s2 + n2s2);
    const R p = n1s * n2s * n3s;
    const R b1 = (R)2 * K[1] * p * n2s * n3s, b2 = (R)2 * K[1] * p * n1s * n3s, b3 = (R)2 * K[1] * p * n1s * n2s;
    const R c1 = (R)4 * K[2] * n1s3 * (n2s4 + n3s4), c2 = (R)4 * K[2] * n2s3 * (n1s4 + n3s4), c3 = (R)4 * K[2] * n3s3 * (n1s4 + n2s4);
    hx = (n[0] * a1 + n[3] * a2 + n[6] * a3) + (n[0] * b1 + n[3] * b2 + n[6] * b3) + (n[0] * c1 + n[3] * c2 + n[6] * c3);
    hy = (n[1] * a1 + n[4] * a2 + n[7] * a3) + (n[1] * b1 + n[4] * b2 + n[7] * b3) + (n[1] * c1 + n[4] * c2 + n[7] * c3);
    hz = (n[2] * a1 + n[5] * a2 + n[8] * a3) + (n[2] * b1 + n[5] * b2 + n[8] * b3) + (n[2] * c1 + n[5] * c2 + n[8] * c3);
}

// ------------------------------------------------------------------ fused step
// Uniform-parameter systems: ms, alpha, gamma, anisotropy and thermal scale
// the same on every site, exchange as a six-direction stencil.  Constants
// are folded on the host (FastK).
// One site of the fused step.  (x, y, z) are the site's coordinates inside
// its lattice of NX x NY x NZ sites and i its index in the (packed) arrays;
// neighbours are addressed relative to i, so several lattices can share the
// arrays back to back.
// The new spin of the site is returned in (rx, ry, rz); (Ax, Ay, Az) is the
// materialised addend (the dipole slot), used when ADD.
// reciprocal square root and sine/cosine in the state precision
__device__ __forceinline__ float fs_rsqrt(float v) { return rsqrtf(v); }
__device__ __forceinline__ double fs_rsqrt(double v) { return rsqrt(v); }
__device__ __forceinline__ void fs_sincos(float a, float* s, float* c) { sincosf(a, s, c); }
__device__ __forceinline__ void fs_sincos(double a, double* s, double* c) { sincos(a, s, c); }

// The spins come through ld(c, j) (component c of site j): global loads, or
// shared-memory copies of some rows (the fused x pass).
template <typename R>
struct GlobalSpins {
    const R* __restrict__ s[3];
    __device__ __forceinline__ R operator()(int c, int j) const { return __ldg(s[c] + j); }
};

// The thermal site's three standard normals are those of thermal_normal3();
// a caller that drew them earlier passes them in pre (else nullptr).
template <typename R>
__device__ __forceinline__ float3 thermal_normal3(const FastKT<R>& F, int i)
{
    const uint64_t ctr = F.counter + (F.dctr ? *F.dctr : 0ull);
    return philox_normal3(F.seed, ctr, (uint32_t)i, 0x6d6c6232u);
}

template <int LT, bool EXS, bool ANI, bool TH, bool ADD, typename R, class LD>
__device__ __forceinline__ void fused_site_ld(const FastKT<R>& F, int NX, int NY, int NZ, int x, int y, int z, int i,
                                              const LD& ld, R Ax, R Ay, R Az, R& rx, R& ry, R& rz,
                                              const float3* pre = nullptr)
{
    const int nxy = NX * NY;
    const R Sx = ld(0, i), Sy = ld(1, i), Sz = ld(2, i);
    R Hx, Hy, Hz;
    if (F.Bdev) { Hx = (R)F.Bdev[0]; Hy = (R)F.Bdev[1]; Hz = (R)F.Bdev[2]; }
    else { Hx = F.B[0]; Hy = F.B[1]; Hz = F.B[2]; }
    if (EXS) {
        // the six neighbours (+x, -x, +y, -y, +z, -z; wrapped where periodic,
        // absent (-1) at an open edge); all eighteen loads are issued before
        // the first sum (an absent neighbour loads the site itself and is not
        // added), then the terms are added in the fixed neighbour order
        int f[6];
        f[0] = x + 1 < NX ? i + 1 : (F.pbc[0] ? i + 1 - NX : -1);
        f[1] = x > 0 ? i - 1 : (F.pbc[0] ? i + NX - 1 : -1);
        f[2] = y + 1 < NY ? i + NX : (F.pbc[1] ? i + NX - nxy : -1);
        f[3] = y > 0 ? i - NX : (F.pbc[1] ? i + nxy - NX : -1);
        f[4] = z + 1 < NZ ? i + nxy : (F.pbc[2] ? i + nxy - nxy * NZ : -1);
        f[5] = z > 0 ? i - nxy : (F.pbc[2] ? i + nxy * NZ - nxy : -1);
        R nb[6][3];
#pragma unroll
        for (int k = 0; k < 6; k++) {
            const int j = f[k] >= 0 ? f[k] : i;
            nb[k][0] = ld(0, j); nb[k][1] = ld(1, j); nb[k][2] = ld(2, j);
        }
        R ex = 0, ey = 0, ez = 0;
#pragma unroll
        for (int k = 0; k < 6; k++) {
            const R J = F.J[k];
            if (J != (R)0 && f[k] >= 0) {
                ex += J * nb[k][0]; ey += J * nb[k][1]; ez += J * nb[k][2];
            }
        }
        Hx += ex; Hy += ey; Hz += ez;
    }
    if (ANI) {
        if (F.ani == 2) {
            // one uniform cubic axis set
            R cx, cy, cz;
            cubic_field<R>(Sx * F.cub_ims, Sy * F.cub_ims, Sz * F.cub_ims, F.cub_n, F.cub_K, F.cub_quirk, cx, cy,
                           cz);
            Hx += cx; Hy += cy; Hz += cz;
        } else {
            const R v = F.ani_c * (Sx * F.axis[0] + Sy * F.axis[1] + Sz * F.axis[2]);
            Hx += v * F.axis[0]; Hy += v * F.axis[1]; Hz += v * F.axis[2];
        }
    }
    R Tx = 0, Ty = 0, Tz = 0;
    if (TH) {
        const float3 nrm = pre ? *pre : thermal_normal3(F, i);
        Tx = F.sigma * nrm.x; Ty = F.sigma * nrm.y; Tz = F.sigma * nrm.z;
        Hx += Tx; Hy += Ty; Hz += Tz;
    }
    if (ADD) {
        Hx += F.addw * Ax; Hy += F.addw * Ay; Hz += F.addw * Az;
    }
    R nx_, ny_, nz_;
    if (LT == LLG_CART) {
        if (F.dt_zero) { nx_ = Sx; ny_ = Sy; nz_ = Sz; }
        else {
            // h = H - Hth; dM = -p gaa M x H - d (a/ms) gaa M x (M x h)
            const R hx = F.tof ? Hx - Tx : Hx, hy = F.tof ? Hy - Ty : Hy, hz = F.tof ? Hz - Tz : Hz;
            const R mhx = Sy * hz - Sz * hy, mhy = Sz * hx - Sx * hz, mhz = Sx * hy - Sy * hx;
            const R mmx = Sy * mhz - Sz * mhy, mmy = Sz * mhx - Sx * mhz, mmz = Sx * mhy - Sy * mhx;
            const R MHx = Sy * Hz - Sz * Hy, MHy = Sz * Hx - Sx * Hz, MHz = Sx * Hy - Sy * Hx;
            nx_ = Sx + F.dt * (F.c_prec * MHx - F.c_damp * mmx);
            ny_ = Sy + F.dt * (F.c_prec * MHy - F.c_damp * mmy);
            nz_ = Sz + F.dt * (F.c_prec * MHz - F.c_damp * mmz);
        }
    } else {
        R Hpx, Hpy, Hpz;
        if (F.tof) {
            const R hx = Hx - Tx, hy = Hy - Ty, hz = Hz - Tz;
            const R shx = Sy * hz - Sz * hy, shy = Sz * hx - Sx * hz, shz = Sx * hy - Sy * hx;
            Hpx = F.precess * Hx + F.c_damp * shx;
            Hpy = F.precess * Hy + F.c_damp * shy;
            Hpz = F.precess * Hz + F.c_damp * shz;
        } else {
            const R shx = Sy * Hz - Sz * Hy, shy = Sz * Hx - Sx * Hz, shz = Sx * Hy - Sy * Hx;
            Hpx = Hx + F.c_damp * shx; Hpy = Hy + F.c_damp * shy; Hpz = Hz + F.c_damp * shz;
        }
        const R HL2 = Hpx * Hpx + Hpy * Hpy + Hpz * Hpz;
        if (HL2 > (R)0) {
            const R iHL = fs_rsqrt(HL2);
            const R HL = HL2 * iHL;
            // half rotation angle; in FP32 small angles by their Taylor
            // series (|th| <= 0.1: truncation below 1e-10, under FP32
            // rounding), else (and always in FP64) sine and cosine
            const R th = F.c_rot * HL;
            R sn, cs;
            if (sizeof(R) == 4 && fabs(th) <= (R)0.1) {
                const R t2 = th * th;
                sn = th * (1.0f - t2 * (1.0f / 6.0f) * (1.0f - t2 * (1.0f / 20.0f) * (1.0f - t2 * (1.0f / 42.0f))));
                cs = 1.0f - t2 * 0.5f * (1.0f - t2 * (1.0f / 12.0f) * (1.0f - t2 * (1.0f / 30.0f) * (1.0f - t2 * (1.0f / 56.0f))));
            } else {
                fs_sincos(th, &sn, &cs);
            }
            const R qw = cs, qx = sn * Hpx * iHL, qy = sn * Hpy * iHL, qz = sn * Hpz * iHL;
            const R tw = -qx * Sx - qy * Sy - qz * Sz;
            const R tx = qw * Sx + qy * Sz - qz * Sy;
            const R ty = qw * Sy + qz * Sx - qx * Sz;
            const R tz = qw * Sz + qx * Sy - qy * Sx;
            nx_ = -tw * qx + qw * tx - ty * qz + tz * qy;
            ny_ = -tw * qy + qw * ty - tz * qx + tx * qz;
            nz_ = -tw * qz + qw * tz - tx * qy + ty * qx;
        } else { nx_ = Sx; ny_ = Sy; nz_ = Sz; }
    }
    if (F.renorm) {
        const R mm = nx_ * nx_ + ny_ * ny_ + nz_ * nz_;
        if (mm != (R)0) {
            const R inv = F.ms * fs_rsqrt(mm);
            nx_ *= inv; ny_ *= inv; nz_ *= inv;
        }
    }
    rx = nx_; ry = ny_; rz = nz_;
    if (F.status && !(isfinite(nx_) && isfinite(ny_) && isfinite(nz_))) atomicOr(F.status, 1u);
}

template <int LT, bool EXS, bool ANI, bool TH, bool ADD, typename R = float>
__device__ __forceinline__ void fused_site_v(const FastKT<R>& F, int NX, int NY, int NZ, int x, int y, int z, int i,
                                             const R* __restrict__ sx, const R* __restrict__ sy,
                                             const R* __restrict__ sz, R Ax, R Ay, R Az, R& rx, R& ry, R& rz,
                                             const float3* pre = nullptr)
{
    const GlobalSpins<R> g{{sx, sy, sz}};
    fused_site_ld<LT, EXS, ANI, TH, ADD, R>(F, NX, NY, NZ, x, y, z, i, g, Ax, Ay, Az, rx, ry, rz, pre);
}

