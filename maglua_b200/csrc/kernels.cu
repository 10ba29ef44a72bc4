// kernels.cu -- sm_100a kernels of the spin-dynamics step.
//
//   k_fused_step     one pass: Exchange + Anisotropy (generic/uniaxial/cubic)
//                    + Thermal (Philox or injected normals) + Zeeman + materialised
//                    slot arrays (the dipole field) -> LLG (Cartesian or Quaternion)
//                    -> renormalised spins written to the other spin buffer.
//   k_eval_terms     the same field evaluation written to a slot (materialise).
//   k_llg            stand-alone LLG over slot arrays (general from/dmdt/to).
//   k_conv_fx/yz/ix  dipole convolution: R2C along x; per-kx 2D FFT over (y,z)
//                    with the per-k tensor multiply fused; C2R along x.
//   k_tensor_*       FP64 interaction-tensor setup and its FP64 FFT.
//   k_netmoment_*    FP64 reductions.
//
// Reference semantics are cited per device function (paths relative to the
// reference project, M/ = src/modules/).
#include "device.cuh"
#include "fused.cuh"
#include "kparams.h"
#include "launch.h"

#include <cuda_runtime.h>
#include <math.h>

#include <algorithm>
#include <stdint.h>
#include <stdio.h>

// ------------------------------------------------------------ helpers
template <typename R>
struct V3 {
    R x, y, z;
};
template <typename R> __device__ __forceinline__ V3<R> v3(R a, R b, R c) { V3<R> v; v.x = a; v.y = b; v.z = c; return v; }
template <typename R> __device__ __forceinline__ V3<R> add3(V3<R> a, V3<R> b) { return v3<R>(a.x + b.x, a.y + b.y, a.z + b.z); }
template <typename R> __device__ __forceinline__ V3<R> sub3(V3<R> a, V3<R> b) { return v3<R>(a.x - b.x, a.y - b.y, a.z - b.z); }
template <typename R> __device__ __forceinline__ V3<R> scl3(R a, V3<R> b) { return v3<R>(a * b.x, a * b.y, a * b.z); }
template <typename R> __device__ __forceinline__ V3<R> cross3(V3<R> a, V3<R> b)
{
    return v3<R>(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
template <typename R> __device__ __forceinline__ R ldr(const void* p, int i) { return __ldg(static_cast<const R*>(p) + i); }
template <typename R> __device__ __forceinline__ R ms_at(const SysK& s, int i) { return s.ms_uniform ? (R)s.ms_u : ldr<R>(s.ms, i); }
template <typename R> __device__ __forceinline__ R alpha_at(const SysK& s, int i) { return s.site_alpha ? ldr<R>(s.site_alpha, i) : (R)s.alpha; }
template <typename R> __device__ __forceinline__ R gamma_at(const SysK& s, int i) { return s.site_gamma ? ldr<R>(s.site_gamma, i) : (R)s.gamma; }
template <typename R> __device__ __forceinline__ V3<R> spin_at(const SysK& s, int i)
{
    return v3<R>(ldr<R>(s.x, i), ldr<R>(s.y, i), ldr<R>(s.z, i));
}
template <typename R> __device__ __forceinline__ R rsq(R v);
template <> __device__ __forceinline__ float rsq<float>(float v) { return sqrtf(v); }
template <> __device__ __forceinline__ double rsq<double>(double v) { return sqrt(v); }
__device__ __forceinline__ void sincos_r(float v, float* s, float* c) { sincosf(v, s, c); }
__device__ __forceinline__ void sincos_r(double v, double* s, double* c) { sincos(v, s, c); }

// ------------------------------------------------------------ field terms
// Exchange: h_t += J s_f / (m_f m_t) (normalised) or J s_f / m_f, only for
// m_f != 0 (M/cpu/exchange/spinoperationexchange.cpp:134-213).
template <typename R>
__device__ __forceinline__ V3<R> ex_term(const ExchangeK& e, const SysK& s, int i, R mt)
{
    V3<R> h = v3<R>(0, 0, 0);
    if (e.mode == EX_STENCIL) {
        const int ix = i % s.nx;
        const int iy = (i / s.nx) % s.ny;
        const int iz = i / (s.nx * s.ny);
        const int nxy = s.nx * s.ny;
#pragma unroll
        for (int d = 0; d < 6; d++) {
            const R J = (R)e.J[d];
            if (J == (R)0) continue;
            const int ax = d >> 1;
            const int sg = (d & 1) ? -1 : 1;
            int c = ax == 0 ? ix : (ax == 1 ? iy : iz);
            const int n = ax == 0 ? s.nx : (ax == 1 ? s.ny : s.nz);
            c += sg;
            if (c < 0 || c >= n) {
                if (!e.pbc[ax]) continue;
                c = c < 0 ? c + n : c - n;
            }
            const int f = ax == 0 ? (i - ix + c) : (ax == 1 ? (i + (c - iy) * s.nx) : (i + (c - iz) * nxy));
            const R mf = ms_at<R>(s, f);
            if (mf != (R)0) {
                const V3<R> sf = spin_at<R>(s, f);
                const R w = J / (e.normalize ? mf * mt : mf);   // one division per neighbour
                h = add3(h, v3<R>(sf.x * w, sf.y * w, sf.z * w));
            }
        }
    } else if (e.mode == EX_CSR) {
        const int p0 = __ldg(e.ptr + i), p1 = __ldg(e.ptr + i + 1);
        for (int p = p0; p < p1; p++) {
            const int f = __ldg(e.col + p);
            const R J = (R)__ldg(e.val + p);
            const R mf = ms_at<R>(s, f);
            if (mf != (R)0) {
                const V3<R> sf = spin_at<R>(s, f);
                const R den = e.normalize ? mf * mt : mf;
                h = add3(h, v3<R>(sf.x * J / den, sf.y * J / den, sf.z * J / den));
            }
        }
    }
    return h;
}

// Anisotropy: H = 2K (s.n)/ms^2 n for ms > 0
// (M/cpu/anisotropy/spinoperationanisotropy.cpp:247-283).
template <typename R>
__device__ __forceinline__ V3<R> ani_one(V3<R> sp, R ms, R n0, R n1, R n2, R K)
{
    const R sda = sp.x * n0 + sp.y * n1 + sp.z * n2;
    const R v = (R)2 * K * sda / (ms * ms);
    return v3<R>(n0 * v, n1 * v, n2 * v);
}
template <typename R>
__device__ __forceinline__ V3<R> ani_term(const AniK& a, V3<R> sp, R ms, int i)
{
    V3<R> h = v3<R>(0, 0, 0);
    if (!(ms > (R)0)) return h;
    if (a.mode == ANI_UNIFORM) return ani_one<R>(sp, ms, (R)a.axis[0], (R)a.axis[1], (R)a.axis[2], (R)a.K);
    if (a.mode == ANI_CSR) {
        const int p0 = __ldg(a.ptr + i), p1 = __ldg(a.ptr + i + 1);
        for (int p = p0; p < p1; p++)
            h = add3(h, ani_one<R>(sp, ms, (R)__ldg(a.axes + 3 * p), (R)__ldg(a.axes + 3 * p + 1),
                                   (R)__ldg(a.axes + 3 * p + 2), (R)__ldg(a.Ks + p)));
    }
    return h;
}

// Uniaxial: [2K1 u + 4K2 u^3] n with u = s.n of the unit spin; quirk keeps
// the reference's sz*nx (..._uniaxial.cpp:250-298, :287).
template <typename R>
__device__ __forceinline__ V3<R> uni_one(V3<R> u3, R n0, R n1, R n2, R K1, R K2, int quirk)
{
    const R u = u3.x * n0 + u3.y * n1 + u3.z * (quirk ? n0 : n2);
    const R mag = (R)2 * K1 * u + (R)4 * K2 * (u * u * u);
    return v3<R>(n0 * mag, n1 * mag, n2 * mag);
}
template <typename R>
__device__ __forceinline__ V3<R> uni_term(const UniK& a, V3<R> sp, R ms, int i)
{
    V3<R> h = v3<R>(0, 0, 0);
    if (!(ms > (R)0) || a.mode == ANI_NONE) return h;
    const V3<R> u = v3<R>(sp.x / ms, sp.y / ms, sp.z / ms);
    if (a.mode == ANI_UNIFORM)
        return uni_one<R>(u, (R)a.axis[0], (R)a.axis[1], (R)a.axis[2], (R)a.K1, (R)a.K2, a.quirk);
    const int p0 = __ldg(a.ptr + i), p1 = __ldg(a.ptr + i + 1);
    for (int p = p0; p < p1; p++)
        h = add3(h, uni_one<R>(u, (R)__ldg(a.axes + 3 * p), (R)__ldg(a.axes + 3 * p + 1), (R)__ldg(a.axes + 3 * p + 2),
                               (R)__ldg(a.K12 + 2 * p), (R)__ldg(a.K12 + 2 * p + 1), a.quirk));
    return h;
}

// Cubic (..._cubic.cpp:308-390): cubic_field (fused.cuh) on a V3.
template <typename R>
__device__ __forceinline__ V3<R> cub_one(V3<R> s, const R* n, const R* K, int quirk)
{
    V3<R> h;
    cubic_field<R>(s.x, s.y, s.z, n, K, quirk, h.x, h.y, h.z);
    return h;
}
template <typename R>
__device__ __forceinline__ V3<R> cub_term(const CubK& a, V3<R> sp, R ms, int i)
{
    V3<R> h = v3<R>(0, 0, 0);
    if (!(ms > (R)0) || a.mode == ANI_NONE) return h;
    const V3<R> u = v3<R>(sp.x / ms, sp.y / ms, sp.z / ms);
    R n[9], K[3];
    if (a.mode == ANI_UNIFORM) {
#pragma unroll
        for (int q = 0; q < 9; q++) n[q] = (R)a.axes[q];
#pragma unroll
        for (int q = 0; q < 3; q++) K[q] = (R)a.K[q];
        return cub_one<R>(u, n, K, a.quirk);
    }
    const int p0 = __ldg(a.ptr + i), p1 = __ldg(a.ptr + i + 1);
    for (int p = p0; p < p1; p++) {
#pragma unroll
        for (int q = 0; q < 9; q++) n[q] = (R)__ldg(a.axs + 9 * p + q);
#pragma unroll
        for (int q = 0; q < 3; q++) K[q] = (R)__ldg(a.Ks + 3 * p + q);
        h = add3(h, cub_one<R>(u, n, K, a.quirk));
    }
    return h;
}

// Thermal: sigma = sqrt(2 alpha T scale / (ms dt gamma)) times N(0,1) per
// component, zero where ms == 0, T == 0 or gamma <= 0
// (M/cpu/thermal/spinoperationthermal.cpp:135-191).
template <typename R>
__device__ __forceinline__ V3<R> th_term(const ThermalK& t, const SysK& s, R dt_sys, int i, R ms)
{
    V3<R> h = v3<R>(0, 0, 0);
    if (t.mode == TH_NONE || ms == (R)0 || t.T == 0.0) return h;
    const R a = alpha_at<R>(s, i), g = gamma_at<R>(s, i);
    if (!(g > (R)0)) return h;
    const R sc = t.scale ? (R)__ldg(t.scale + i) : (R)1;
    const R sd = rsq<R>(((R)2 * a * (R)t.T * sc) / (ms * dt_sys * g));
    V3<R> n;
    if (t.mode == TH_PHILOX) {
        const uint64_t ctr = t.counter + (t.dctr ? *t.dctr : 0ull);
        const float3 f = philox_normal3(t.seed, ctr, (uint32_t)i, 0x6d6c6232u);
        n = v3<R>((R)f.x, (R)f.y, (R)f.z);
    } else {
        n = v3<R>((R)__ldg(t.nx + i), (R)__ldg(t.ny + i), (R)__ldg(t.nz + i));
    }
    return v3<R>(sd * n.x, sd * n.y, sd * n.z);
}

template <typename R>
struct Fields {
    V3<R> H;
    V3<R> Hth;
};

// Every term of TermsK at site i.  H is the would-be "Total" slot, Hth the
// "Thermal" slot that LLG subtracts (llgcartesian.cpp:160-172).
template <typename R>
__device__ __forceinline__ Fields<R> eval_terms(const TermsK& T, const SysK& s, R dt_sys, int i)
{
    const R ms = ms_at<R>(s, i);
    const V3<R> sp = spin_at<R>(s, i);
    V3<R> H = v3<R>(0, 0, 0);
    V3<R> Hth = v3<R>(0, 0, 0);
    if (T.ex.mode != EX_NONE) H = add3(H, scl3((R)T.ex_gs, ex_term<R>(T.ex, s, i, ms)));
    if (T.ani.mode != ANI_NONE) H = add3(H, ani_term<R>(T.ani, sp, ms, i));
    if (T.uni.mode != ANI_NONE) H = add3(H, uni_term<R>(T.uni, sp, ms, i));
    if (T.cub.mode != ANI_NONE) H = add3(H, cub_term<R>(T.cub, sp, ms, i));
    if (T.th.mode != TH_NONE) { Hth = th_term<R>(T.th, s, dt_sys, i, ms); H = add3(H, Hth); }
    if (T.zee.on) {
        const V3<R> B = T.zee.Bdev ? v3<R>((R)T.zee.Bdev[0], (R)T.zee.Bdev[1], (R)T.zee.Bdev[2])
                                   : v3<R>((R)T.zee.B[0], (R)T.zee.B[1], (R)T.zee.B[2]);
        H = add3(H, B);
    }
    for (int a = 0; a < T.nadd; a++) {
        const V3<R> v = v3<R>(ldr<R>(T.add[a][0], i), ldr<R>(T.add[a][1], i), ldr<R>(T.add[a][2], i));
        const R w = (R)T.addw[a];
        H = add3(H, v3<R>(w * v.x, w * v.y, w * v.z));
        if (T.add_is_thermal[a]) Hth = add3(Hth, v);
    }
    Fields<R> f;
    f.H = H;
    f.Hth = Hth;
    return f;
}

// ------------------------------------------------------------ LLG
// Cartesian Euler step (M/cpu/llg/llgcartesian.cpp:90-278) or quaternion
// rotation (M/cpu/llg/llgquat.cpp:126-378) for one site with ms > 0.
// S: from-spin, M: dmdt-spin, H: Total, Hth: Thermal.
template <typename R>
__device__ __forceinline__ V3<R> llg_site(const LlgK& L, V3<R> S, V3<R> M, V3<R> H, V3<R> Hth, R ms, R a, R g)
{
    const R dt = (R)L.dt, p = (R)L.precess, d = (R)L.damp;
    if (L.type == LLG_CART) {
        if (L.dt_zero) return S;
        const R gaa = g / ((R)1 + a * a);
        if (L.thermal_only_first_term) {
            const V3<R> h = sub3(H, Hth);
            const V3<R> Mh = cross3(M, h);
            const V3<R> MMH = cross3(M, Mh);
            const V3<R> MH = cross3(M, H);
            const V3<R> dM = sub3(scl3(p * -gaa, MH), scl3(d * (a / ms) * gaa, MMH));
            return add3(S, scl3(dt, dM));
        }
        const V3<R> MH = cross3(M, H);
        const V3<R> MMH = cross3(M, MH);
        const V3<R> dM = sub3(scl3(-gaa, MH), scl3((a / ms) * gaa, MMH));
        return add3(S, scl3(dt, dM));
    }
    // quaternion
    const R inv = (R)1 / ms;
    V3<R> Hp;
    if (L.thermal_only_first_term) {
        const V3<R> h = sub3(H, Hth);
        const V3<R> Sh = cross3(M, h);
        Hp = add3(scl3(p, H), scl3(d * a * inv, Sh));
    } else {
        const V3<R> SH = cross3(S, H);
        Hp = add3(H, scl3(a * inv, SH));
    }
    const R HLen = rsq<R>(Hp.x * Hp.x + Hp.y * Hp.y + Hp.z * Hp.z);
    if (!(HLen > (R)0)) return S;
    const R iHLen = (R)1 / HLen;
    const R ra = (R)1 * g * HLen / ((R)1 + a * a);
    R sint, cost;
    sincos_r(((R)0.5) * ra * dt, &sint, &cost);
    // qRot = (cost, sint * Hp/|Hp|); qRes = qRot * (0,S) * conj(qRot)
    const R qw = cost, qx = sint * Hp.x * iHLen, qy = sint * Hp.y * iHLen, qz = sint * Hp.z * iHLen;
    const R tw = -qx * S.x - qy * S.y - qz * S.z;
    const R tx = qw * S.x + qy * S.z - qz * S.y;
    const R ty = qw * S.y + qz * S.x - qx * S.z;
    const R tz = qw * S.z + qx * S.y - qy * S.x;
    const R cx = -qx, cy = -qy, cz = -qz;
    V3<R> r;
    r.x = tw * cx + qw * tx + ty * cz - tz * cy;
    r.y = tw * cy + qw * ty + tz * cx - tx * cz;
    r.z = tw * cz + qw * tz + tx * cy - ty * cx;
    return r;
}

template <typename R>
__device__ __forceinline__ V3<R> renorm(V3<R> v, R ms)
{
    const R mm = v.x * v.x + v.y * v.y + v.z * v.z;
    if (mm != (R)0) {
        const R inv = ms / rsq<R>(mm);
        return v3<R>(v.x * inv, v.y * inv, v.z * inv);
    }
    return v;
}

// ------------------------------------------------------------ kernels
template <typename R>
__global__ void __launch_bounds__(256) k_fused_step(FusedK P, double dt_sys)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.sys.n) return;
    const R ms = ms_at<R>(P.sys, i);
    const V3<R> S = spin_at<R>(P.sys, i);
    V3<R> out = S;
    if (ms > (R)0) {
        const Fields<R> F = eval_terms<R>(P.terms, P.sys, (R)dt_sys, i);
        out = llg_site<R>(P.llg, S, S, F.H, F.Hth, ms, alpha_at<R>(P.sys, i), gamma_at<R>(P.sys, i));
    }
    if (P.llg.renorm) out = renorm<R>(out, ms);
    if (P.llg.status && !(isfinite(out.x) && isfinite(out.y) && isfinite(out.z))) atomicOr(P.llg.status, 1u);
    static_cast<R*>(P.ox)[i] = out.x;
    static_cast<R*>(P.oy)[i] = out.y;
    static_cast<R*>(P.oz)[i] = out.z;
}

// out = (accumulate ? out : 0) + terms
template <typename R>
__global__ void __launch_bounds__(256) k_eval_terms(SysK s, TermsK T, double dt_sys, void* hx_, void* hy_,
                                                    void* hz_, int accumulate)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= s.n) return;
    R* hx = static_cast<R*>(hx_);
    R* hy = static_cast<R*>(hy_);
    R* hz = static_cast<R*>(hz_);
    const Fields<R> F = eval_terms<R>(T, s, (R)dt_sys, i);
    if (accumulate) { hx[i] += F.H.x; hy[i] += F.H.y; hz[i] += F.H.z; }
    else { hx[i] = F.H.x; hy[i] = F.H.y; hz[i] = F.H.z; }
}

// Stand-alone LLG: from (spins+ms), dmdt spins M, Total H, optional Thermal.
// Sites with ms <= 0 keep the destination's current value.
template <typename R>
__global__ void __launch_bounds__(256) k_llg(SysK from, const void* mx, const void* my, const void* mz,
                                             const void* hx, const void* hy, const void* hz,
                                             const void* tx, const void* ty, const void* tz,
                                             const void* dsa, const void* dsg, double da, double dg,
                                             LlgK L, void* ox_, void* oy_, void* oz_)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= from.n) return;
    R* ox = static_cast<R*>(ox_);
    R* oy = static_cast<R*>(oy_);
    R* oz = static_cast<R*>(oz_);
    const R ms = ms_at<R>(from, i);
    V3<R> out = v3<R>(ox[i], oy[i], oz[i]);
    if (L.type == LLG_CART && L.dt_zero) {
        out = spin_at<R>(from, i);
    } else if (ms > (R)0) {
        const V3<R> S = spin_at<R>(from, i);
        const V3<R> M = v3<R>(ldr<R>(mx, i), ldr<R>(my, i), ldr<R>(mz, i));
        const V3<R> H = v3<R>(ldr<R>(hx, i), ldr<R>(hy, i), ldr<R>(hz, i));
        const V3<R> Ht = tx ? v3<R>(ldr<R>(tx, i), ldr<R>(ty, i), ldr<R>(tz, i)) : v3<R>(0, 0, 0);
        const R a = dsa ? ldr<R>(dsa, i) : (R)da, g = dsg ? ldr<R>(dsg, i) : (R)dg;
        out = llg_site<R>(L, S, M, H, Ht, ms, a, g);
    }
    if (L.renorm) out = renorm<R>(out, ms);
    if (L.status && !(isfinite(out.x) && isfinite(out.y) && isfinite(out.z))) atomicOr(L.status, 1u);
    ox[i] = out.x; oy[i] = out.y; oz[i] = out.z;
}

// One step of the device step block: next Thermal counter, swept field.
__global__ void k_advance_step(const DevStep* cur, DevStep* next)
{
    pdl_wait();   // the step's kernels read cur until they complete
    const DevStep c = *cur;
    next->th_counter = c.th_counter + 1ull;
    for (int a = 0; a < 3; a++) {
        next->B[a] = c.B[a] + c.dB[a];
        next->dB[a] = c.dB[a];
    }
}

// FP64 partial sums for netMoment: per block (sum v*m, sum (v*m)^2) x 3.
template <typename R>
__global__ void __launch_bounds__(256) k_netmoment_partial(const void* x_, const void* y_, const void* z_,
                                                           int n, double m, double* part)
{
    const R* x = static_cast<const R*>(x_);
    const R* y = static_cast<const R*>(y_);
    const R* z = static_cast<const R*>(z_);
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double a = (double)x[i] * m, b = (double)y[i] * m, c = (double)z[i] * m;
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
        part[blockIdx.x * 6 + threadIdx.x] = v;
    }
}

// netMoment in one launch: each block writes its six partials as
// k_netmoment_partial does; the last block to finish (a device counter,
// reset for the next launch) reduces them, one warp per quantity in a fixed
// order, and writes the six results to out (pinned host memory the device
// reaches directly) and out_dev.  NMT = 1024 threads per block, so that a
// few blocks keep enough loads in flight (launch_netmoment_one).
constexpr int NMT = 1024;
template <typename R>
__global__ void __launch_bounds__(NMT) k_netmoment_one(const void* x_, const void* y_, const void* z_, int n,
                                                       double m, double* part, unsigned* counter, double* out,
                                                       double* out_dev)
{
    const R* x = static_cast<const R*>(x_);
    const R* y = static_cast<const R*>(y_);
    const R* z = static_cast<const R*>(z_);
    double acc[6] = {0, 0, 0, 0, 0, 0};
    // eight sites per round with their loads issued together (one memory
    // latency per round instead of one per site); sites in increasing order
    const int stride = gridDim.x * blockDim.x;
    constexpr int U = 8;
    for (int i0 = blockIdx.x * blockDim.x + threadIdx.x; i0 < n; i0 += U * stride) {
        R xs[U], ys[U], zs[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int i = i0 + u * stride;
            xs[u] = i < n ? x[i] : (R)0;
            ys[u] = i < n ? y[i] : (R)0;
            zs[u] = i < n ? z[i] : (R)0;
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            if (i0 + u * stride >= n) break;
            const double a = (double)xs[u] * m, b = (double)ys[u] * m, c = (double)zs[u] * m;
            acc[0] += a; acc[1] += b; acc[2] += c;
            acc[3] += a * a; acc[4] += b * b; acc[5] += c * c;
        }
    }
    __shared__ double sh[6][NMT / 32];
    __shared__ bool last;
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
        part[blockIdx.x * 6 + threadIdx.x] = v;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    // warp q sums quantity q: lane l takes blocks l, l + 32, ... in order,
    // then a fixed shuffle tree (deterministic)
    const int nb = gridDim.x;
    if (w < 6) {
        double v = 0;
        for (int b = lane; b < nb; b += 32) v += __ldcg(part + b * 6 + w);
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) {
            out[w] = v;
            out_dev[w] = v;
        }
    }
    // (the host reads the sums after the kernel completes, which orders them)
    if (threadIdx.x == 0) *counter = 0u;
}

namespace mlb {
// side = false (a synchronous read): enough blocks of NMT threads for one
// round of 8 sites each (at most 2 x 148); side = true (a read on its own
// stream next to the following steps, whose kernels take whole SMs): at most
// 16 blocks, so that most SMs stay free for the steps.  part holds nb x 6.
int netmoment_blocks(int n, bool side)
{
    const int full = std::max(1, std::min(2 * 148, (n + 8 * NMT - 1) / (8 * NMT)));
    return side ? std::max(1, std::min(16, (n + NMT - 1) / NMT)) : full;
}

cudaError_t launch_netmoment_one(const void* x, const void* y, const void* z, int n, double m, double* part, int nb,
                                 unsigned* counter, double* out_host, double* out_dev, int rb, cudaStream_t st)
{
    if (rb == 8)
        k_netmoment_one<double><<<nb, NMT, 0, st>>>(x, y, z, n, m, part, counter, out_host, out_dev);
    else
        k_netmoment_one<float><<<nb, NMT, 0, st>>>(x, y, z, n, m, part, counter, out_host, out_dev);
    return cudaGetLastError();
}
} // namespace mlb

// FP64 partial sums of |a - b| per component (SpinSystem::diff,
// spinsystem.cpp:301-307 with dArray::diffSum).
template <typename R>
__global__ void __launch_bounds__(256) k_diff_partial(const void* ax_, const void* ay_, const void* az_,
                                                      const void* bx_, const void* by_, const void* bz_, int n,
                                                      double* part)
{
    const R* a[3] = {static_cast<const R*>(ax_), static_cast<const R*>(ay_), static_cast<const R*>(az_)};
    const R* b[3] = {static_cast<const R*>(bx_), static_cast<const R*>(by_), static_cast<const R*>(bz_)};
    double acc[3] = {0, 0, 0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (int c = 0; c < 3; c++) acc[c] += fabs((double)a[c][i] - (double)b[c][i]);
    __shared__ double sh[3][8];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int q = 0; q < 3; q++) {
        double v = acc[q];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) sh[q][w] = v;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double v = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) v += sh[threadIdx.x][k];
        part[blockIdx.x * 3 + threadIdx.x] = v;
    }
}

// out[q] = sum_b part[b*nq + q]: block q (256 threads), thread t sums
// b = t, t + 256, ... in order, then a fixed shuffle and warp tree
// (deterministic, independent of timing).
__global__ void __launch_bounds__(256) k_partial_final(const double* part, int nb, int nq, double* out)
{
    const int q = blockIdx.x, lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __shared__ double sh[8];
    double v = 0;
    for (int b = threadIdx.x; b < nb; b += 256) v += part[b * nq + q];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) sh[w] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0;
        for (int k = 0; k < 8; k++) s += sh[k];
        out[q] = s;
    }
}

// FP64 sum of s . h over sites (energy-style dot product).
template <typename R>
__global__ void __launch_bounds__(256) k_dot_partial(const void* x_, const void* y_, const void* z_,
                                                     const void* hx_, const void* hy_, const void* hz_,
                                                     int n, double* part)
{
    const R* x = static_cast<const R*>(x_);
    const R* y = static_cast<const R*>(y_);
    const R* z = static_cast<const R*>(z_);
    const R* hx = static_cast<const R*>(hx_);
    const R* hy = static_cast<const R*>(hy_);
    const R* hz = static_cast<const R*>(hz_);
    double acc = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        acc += (double)x[i] * hx[i] + (double)y[i] * hy[i] + (double)z[i] * hz[i];
    __shared__ double sh[8];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double v = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) v += sh[k];
        part[blockIdx.x] = v;
    }
}

// ------------------------------------------------------------ dipole convolution
// Forward x pass: rows (y0..y0+ty) of layer z, three components, zero-padded
// to Px, complex FFT, first Kx bins written to SPEC[kx][c][z][y].
template <typename R>
__global__ void __launch_bounds__(256) k_conv_fx(ConvK c, FftLen Lx, const typename CT<R>::T* tw, const void* sx,
                                                 const void* sy, const void* sz, typename CT<R>::T* spec)
{
    if (c.run_if && *c.run_if == 0) return;
    typedef typename CT<R>::T C;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* smf = reinterpret_cast<C*>(smraw);
    const int y0 = blockIdx.x * c.ty, zz = blockIdx.y;
    const int rows = min(c.ty, c.ny - y0);
    C* A = smf;
    C* B = smf + c.ty * c.Px;
    LineGeo g;
    g.nlines = rows; g.lpg = 1 << 30; g.gstride = 0; g.ls = c.Px; g.es = 1; g.line_fast = 0;
    for (int comp = 0; comp < 3; comp++) {
        const R* src = static_cast<const R*>(comp == 0 ? sx : (comp == 1 ? sy : sz));
        for (int t = threadIdx.x; t < rows * c.Px; t += blockDim.x) {
            const int r = t / c.Px, x = t % c.Px;
            const R v = x < c.nx ? __ldg(src + ((size_t)zz * c.ny + y0 + r) * c.nx + x) : (R)0;
            A[r * c.Px + x] = cmk<C>(v, (R)0);
        }
        __syncthreads();
        const C* Rl = c.Px > 1 ? cta_fft<C>(A, B, g, Lx, tw, -1) : A;
        for (int t = threadIdx.x; t < c.Kx * rows; t += blockDim.x) {
            const int kx = t / rows, r = t % rows;
            spec[(((size_t)kx * 3 + comp) * c.nz + zz) * c.ny + y0 + r] = Rl[r * c.Px + kx];
        }
        __syncthreads();
    }
}

// Per-kx (y,z) plane: forward FFT in y then z (zero padded), tensor
// multiply, inverse z then y, write back the data rows.
template <typename R>
__global__ void __launch_bounds__(512) k_conv_yz(ConvK c, FftLen Ly, FftLen Lz, const typename CT<R>::T* tw,
                                                 typename CT<R>::T* spec, const R* ten6, const typename CT<R>::T* ten9)
{
    if (c.run_if && *c.run_if == 0) return;
    typedef typename CT<R>::T C;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* smf = reinterpret_cast<C*>(smraw);
    const int kx = blockIdx.x;
    const int PP = c.Py * c.Pz;
    C* A = smf;
    C* B = smf + 3 * PP;
    for (int t = threadIdx.x; t < 6 * PP; t += blockDim.x) smf[t] = cmk<C>((R)0, (R)0);
    __syncthreads();
    C* sp = spec + (size_t)kx * 3 * c.nz * c.ny;
    const int NZY = c.nz * c.ny;
    for (int t = threadIdx.x; t < 3 * NZY; t += blockDim.x) {
        const int comp = t / NZY, rem = t % NZY, z = rem / c.ny, y = rem % c.ny;
        A[comp * PP + z * c.Py + y] = sp[t];
    }
    __syncthreads();
    LineGeo gy; gy.nlines = 3 * c.nz; gy.lpg = c.nz; gy.gstride = PP; gy.ls = c.Py; gy.es = 1; gy.line_fast = 0;
    LineGeo gz; gz.nlines = 3 * c.Py; gz.lpg = c.Py; gz.gstride = PP; gz.ls = 1; gz.es = c.Py; gz.line_fast = 1;
    C* cur = A;
    C* oth = B;
    if (c.Py > 1) { cur = cta_fft<C>(cur, oth, gy, Ly, tw, -1); oth = cur == A ? B : A; }
    if (c.Pz > 1) { cur = cta_fft<C>(cur, oth, gz, Lz, tw, -1); oth = cur == A ? B : A; }
    const R gg = (R)c.g;
    if (!c.general) {
        const R* T = ten6 + (size_t)kx * PP * 6;
        for (int t = threadIdx.x; t < PP; t += blockDim.x) {
            const R t0 = __ldg(T + 6 * t), t1 = __ldg(T + 6 * t + 1), t2 = __ldg(T + 6 * t + 2);
            const R t3 = __ldg(T + 6 * t + 3), t4 = __ldg(T + 6 * t + 4), t5 = __ldg(T + 6 * t + 5);
            const C s0 = cur[t], s1 = cur[PP + t], s2 = cur[2 * PP + t];
            cur[t] = cmk<C>(gg * (t0 * s0.x + t1 * s1.x + t2 * s2.x), gg * (t0 * s0.y + t1 * s1.y + t2 * s2.y));
            cur[PP + t] = cmk<C>(gg * (t1 * s0.x + t3 * s1.x + t4 * s2.x), gg * (t1 * s0.y + t3 * s1.y + t4 * s2.y));
            cur[2 * PP + t] = cmk<C>(gg * (t2 * s0.x + t4 * s1.x + t5 * s2.x), gg * (t2 * s0.y + t4 * s1.y + t5 * s2.y));
        }
    } else {
        const C* T = ten9 + (size_t)kx * PP * 9;
        for (int t = threadIdx.x; t < PP; t += blockDim.x) {
            const C s[3] = {cur[t], cur[PP + t], cur[2 * PP + t]};
#pragma unroll
            for (int a = 0; a < 3; a++) {
                C acc = cmk<C>((R)0, (R)0);
#pragma unroll
                for (int b = 0; b < 3; b++) acc = cadd(acc, cmul(T[9 * t + 3 * a + b], s[b]));
                cur[a * PP + t] = cmk<C>(gg * acc.x, gg * acc.y);
            }
        }
    }
    __syncthreads();
    if (c.Pz > 1) { cur = cta_fft<C>(cur, oth, gz, Lz, tw, +1); oth = cur == A ? B : A; }
    if (c.Py > 1) { cur = cta_fft<C>(cur, oth, gy, Ly, tw, +1); oth = cur == A ? B : A; }
    for (int t = threadIdx.x; t < 3 * NZY; t += blockDim.x) {
        const int comp = t / NZY, rem = t % NZY, z = rem / c.ny, y = rem % c.ny;
        sp[t] = cur[comp * PP + z * c.Py + y];
    }
}

// Inverse x pass: Hermitian completion, complex inverse FFT, real part of
// the first nx points written to the field slot.
template <typename R>
__global__ void __launch_bounds__(256) k_conv_ix(ConvK c, FftLen Lx, const typename CT<R>::T* tw, const typename CT<R>::T* spec,
                                                 void* hx, void* hy, void* hz)
{
    if (c.run_if && *c.run_if == 0) return;
    typedef typename CT<R>::T C;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* smf = reinterpret_cast<C*>(smraw);
    const int y0 = blockIdx.x * c.ty, zz = blockIdx.y;
    const int rows = min(c.ty, c.ny - y0);
    C* A = smf;
    C* B = smf + c.ty * c.Px;
    LineGeo g;
    g.nlines = rows; g.lpg = 1 << 30; g.gstride = 0; g.ls = c.Px; g.es = 1; g.line_fast = 0;
    const int nh = c.Px - c.Kx;
    for (int comp = 0; comp < 3; comp++) {
        R* dst = static_cast<R*>(comp == 0 ? hx : (comp == 1 ? hy : hz));
        for (int t = threadIdx.x; t < c.Kx * rows; t += blockDim.x) {
            const int kx = t / rows, r = t % rows;
            A[r * c.Px + kx] = spec[(((size_t)kx * 3 + comp) * c.nz + zz) * c.ny + y0 + r];
        }
        __syncthreads();
        for (int t = threadIdx.x; t < rows * nh; t += blockDim.x) {
            const int r = t / nh, k = c.Kx + t % nh;
            A[r * c.Px + k] = cconj(A[r * c.Px + c.Px - k]);
        }
        __syncthreads();
        const C* Rl = c.Px > 1 ? cta_fft<C>(A, B, g, Lx, tw, +1) : A;
        for (int t = threadIdx.x; t < rows * c.nx; t += blockDim.x) {
            const int r = t / c.nx, x = t % c.nx;
            dst[((size_t)zz * c.ny + y0 + r) * c.nx + x] = Rl[r * c.Px + x].x;
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------ FP64 tensor setup
// Closed-form element, dipolesupport.cpp:32-70 (written without fused
// multiply-adds so the sums match a plain C evaluation bit for bit).
__device__ __forceinline__ void gamma_dip_d(double rx, double ry, double rz, double* g6)
{
    const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(rx, rx), __dmul_rn(ry, ry)), __dmul_rn(rz, rz));
    const double r = __dsqrt_rn(r2);
    if (r < 1E-40) { for (int q = 0; q < 6; q++) g6[q] = 0; return; }
    const double ir = __ddiv_rn(1.0, r);
    const double ir3 = __dmul_rn(__dmul_rn(ir, ir), ir);
    const double ir5 = __dmul_rn(__dmul_rn(ir3, ir), ir);
    g6[0] = -__dsub_rn(ir3, __dmul_rn(__dmul_rn(__dmul_rn(3.0, rx), rx), ir5));
    g6[1] = -(-__dmul_rn(__dmul_rn(__dmul_rn(3.0, rx), ry), ir5));
    g6[2] = -(-__dmul_rn(__dmul_rn(__dmul_rn(3.0, rx), rz), ir5));
    g6[3] = -__dsub_rn(ir3, __dmul_rn(__dmul_rn(__dmul_rn(3.0, ry), ry), ir5));
    g6[4] = -(-__dmul_rn(__dmul_rn(__dmul_rn(3.0, ry), rz), ir5));
    g6[5] = -__dsub_rn(ir3, __dmul_rn(__dmul_rn(__dmul_rn(3.0, rz), rz), ir5));
}

__device__ __forceinline__ long long fdiv_floor(long long a, long long b)
{
    long long q = a / b;
    if ((a % b != 0) && ((a < 0) != (b < 0))) q--;
    return q;
}

// Periodic-in-plane lattice sum for element (i, j, k), getWAB/getWAB_range
// (dipolesupport.cpp:71-240) with the image ranges narrowed to the ones that
// pass the box tests (same terms, same order).  The z offset is written at
// padded index (zsign*k mod Pz): zsign = -1 reproduces the reference's
// source-minus-target layer convention (spinoperationlongrange.cpp:377-384),
// +1 gives the physical target-minus-source one.
__global__ void k_tensor_lattice(int nx, int ny, int nz, int G, int lim0, int limx, int limy,
                                 double A0, double A1, double A2, double B0, double B1, double B2,
                                 double C0, double C1, double C2, int Px, int Py, int Pz, int zsign,
                                 double2* W)
{
    const long long ne = (long long)nx * ny * (2 * nz - 1);
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    const int i = (int)(e % nx);
    const int j = (int)((e / nx) % ny);
    const int k = (int)(e / ((long long)nx * ny)) - (nz - 1);
    double acc[6] = {0, 0, 0, 0, 0, 0};
    const long long R = lim0;
    if (llabs((long long)k) <= R) {
        long long xlo = -(G - 1), xhi = G - 1, ylo = -(G - 1), yhi = G - 1;
        long long a = -fdiv_floor((long long)limx + i, nx), b = fdiv_floor((long long)limx - i, nx);
        if (a > xlo) xlo = a;
        if (b < xhi) xhi = b;
        a = -fdiv_floor((long long)limy + j, ny);
        b = fdiv_floor((long long)limy - j, ny);
        if (a > ylo) ylo = a;
        if (b < yhi) yhi = b;
        const double RR = __dmul_rn((double)R, (double)R);
        for (long long X = xlo; X <= xhi; X++) {
            const long long xx = X * nx + i;
            for (long long Y = ylo; Y <= yhi; Y++) {
                const long long yy = Y * ny + j;
                const long long zz = k;
                const double d2 = __dadd_rn(__dadd_rn(__dmul_rn((double)xx, (double)xx), __dmul_rn((double)yy, (double)yy)),
                                            __dmul_rn((double)zz, (double)zz));
                if (d2 <= RR) {
                    const double fx = (double)xx, fy = (double)yy, fz = (double)zz;
                    const double rx = __dadd_rn(__dadd_rn(__dmul_rn(fx, A0), __dmul_rn(fy, B0)), __dmul_rn(fz, C0));
                    const double ry = __dadd_rn(__dadd_rn(__dmul_rn(fx, A1), __dmul_rn(fy, B1)), __dmul_rn(fz, C1));
                    const double rz = __dadd_rn(__dadd_rn(__dmul_rn(fx, A2), __dmul_rn(fy, B2)), __dmul_rn(fz, C2));
                    double g6[6];
                    gamma_dip_d(rx, ry, rz, g6);
#pragma unroll
                    for (int q = 0; q < 6; q++) acc[q] = __dadd_rn(acc[q], g6[q]);
                }
            }
        }
    }
    int zi = (zsign * k) % Pz;
    if (zi < 0) zi += Pz;
    const size_t plane = (size_t)Px * Py * Pz;
    const size_t off = ((size_t)zi * Py + j) * Px + i;
    for (int q = 0; q < 6; q++) W[q * plane + off] = make_double2(acc[q], 0.0);
}

// The Dipole tensor of truncation math.huge (M/cpu/dipole/dipolesupport.cpp:
// 771-835): the images of each element summed ring by ring, rings of lstep
// lattices (getWAB with smin = q lstep, smax = smin + lstep: for smin = 0 the
// full square |X|, |Y| <= lstep - 1, else the square ring between), nrings
// rings, each ring's sum added to the element's running total in ring
// order.  (The reference's extrapolation never reports convergence -- its
// C side reads a second return value its Lua function does not give -- so
// its result is this sum over its maxiter = 1000 rings of 5 lattices.)  One
// warp per element: the lanes split each ring's images, a shuffle tree
// gives the ring's sum, lane 0 keeps the total.  FP64 throughout.
__global__ void k_tensor_rings(int nx, int ny, int nz, int nrings, int lstep, double A0, double A1, double A2,
                               double B0, double B1, double B2, double C0, double C1, double C2, int Px, int Py,
                               int Pz, int zsign, double2* W)
{
    const long long ne = (long long)nx * ny * (2 * nz - 1);
    const long long e = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (e >= ne) return;   // whole warps leave together
    const int i = (int)(e % nx);
    const int j = (int)((e / nx) % ny);
    const int k = (int)(e / ((long long)nx * ny)) - (nz - 1);
    double tot[6] = {0, 0, 0, 0, 0, 0};
    for (int q = 0; q < nrings; q++) {
        const int mn = q * lstep, mx = mn + lstep;
        double acc[6] = {0, 0, 0, 0, 0, 0};
        // the ring as 2 full-width bands (|Y| >= mn) and 2 side bands (|Y| < mn)
        const int nrect = mn == 0 ? 1 : 4;
        for (int r = 0; r < nrect; r++) {
            int ax, bx, ay, by;
            if (mn == 0) { ax = -(mx - 1); bx = mx - 1; ay = -(mx - 1); by = mx - 1; }
            else if (r == 0) { ax = -(mx - 1); bx = mx - 1; ay = mn; by = mx - 1; }
            else if (r == 1) { ax = -(mx - 1); bx = mx - 1; ay = -(mx - 1); by = -mn; }
            else if (r == 2) { ax = -(mx - 1); bx = -mn; ay = -(mn - 1); by = mn - 1; }
            else { ax = mn; bx = mx - 1; ay = -(mn - 1); by = mn - 1; }
            // lanes stride along the band's long side, each walks the short side
            const bool xlong = (bx - ax) >= (by - ay);
            const int l0 = xlong ? ax : ay, l1 = xlong ? bx : by;
            const int s0 = xlong ? ay : ax, s1 = xlong ? by : bx;
            for (int u = l0 + lane; u <= l1; u += 32) {
                for (int v = s0; v <= s1; v++) {
                    const long long X = xlong ? u : v, Y = xlong ? v : u;
                    const double fx = (double)(X * nx + i), fy = (double)(Y * ny + j), fz = (double)k;
                    const double rx = __dadd_rn(__dadd_rn(__dmul_rn(fx, A0), __dmul_rn(fy, B0)), __dmul_rn(fz, C0));
                    const double ry = __dadd_rn(__dadd_rn(__dmul_rn(fx, A1), __dmul_rn(fy, B1)), __dmul_rn(fz, C1));
                    const double rz = __dadd_rn(__dadd_rn(__dmul_rn(fx, A2), __dmul_rn(fy, B2)), __dmul_rn(fz, C2));
                    double g6[6];
                    gamma_dip_d(rx, ry, rz, g6);
#pragma unroll
                    for (int c = 0; c < 6; c++) acc[c] += g6[c];
                }
            }
        }
#pragma unroll
        for (int c = 0; c < 6; c++) {
            double v = acc[c];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            tot[c] += v;   // meaningful in lane 0
        }
    }
    if (lane != 0) return;
    int zi = (zsign * k) % Pz;
    if (zi < 0) zi += Pz;
    const size_t plane = (size_t)Px * Py * Pz;
    const size_t off = ((size_t)zi * Py + j) * Px + i;
    for (int c = 0; c < 6; c++) W[c * plane + off] = make_double2(tot[c], 0.0);
}

// Also stores the raw (unpadded) reference tensor for inspection:
// out[q][k+nz-1][j][i] like the reference's XX..ZZ arrays.
__global__ void k_tensor_extract_ref(int nx, int ny, int nz, int Px, int Py, int Pz, int zsign,
                                     const double2* W, double* out)
{
    const long long ne = (long long)nx * ny * (2 * nz - 1);
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    const int i = (int)(e % nx);
    const int j = (int)((e / nx) % ny);
    const int k = (int)(e / ((long long)nx * ny)) - (nz - 1);
    int zi = (zsign * k) % Pz;
    if (zi < 0) zi += Pz;
    const size_t plane = (size_t)Px * Py * Pz;
    const size_t off = ((size_t)zi * Py + j) * Px + i;
    for (int q = 0; q < 6; q++) out[q * ne + e] = W[q * plane + off].x;
}

// Open boundaries: Gamma(d) for |dx|<nx, |dy|<ny, |dz|<nz, no images,
// placed at (d mod P).
__global__ void k_tensor_open(int nx, int ny, int nz, double A0, double A1, double A2, double B0,
                              double B1, double B2, double C0, double C1, double C2, int Px, int Py,
                              int Pz, double2* W)
{
    const long long ex = 2 * nx - 1, ey = 2 * ny - 1, ez = 2 * nz - 1;
    const long long ne = ex * ey * ez;
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    const int dx = (int)(e % ex) - (nx - 1);
    const int dy = (int)((e / ex) % ey) - (ny - 1);
    const int dz = (int)(e / (ex * ey)) - (nz - 1);
    const double fx = dx, fy = dy, fz = dz;
    const double rx = __dadd_rn(__dadd_rn(__dmul_rn(fx, A0), __dmul_rn(fy, B0)), __dmul_rn(fz, C0));
    const double ry = __dadd_rn(__dadd_rn(__dmul_rn(fx, A1), __dmul_rn(fy, B1)), __dmul_rn(fz, C1));
    const double rz = __dadd_rn(__dadd_rn(__dmul_rn(fx, A2), __dmul_rn(fy, B2)), __dmul_rn(fz, C2));
    double g6[6];
    gamma_dip_d(rx, ry, rz, g6);
    const int xi = (dx % Px + Px) % Px, yi = (dy % Py + Py) % Py, zi = (dz % Pz + Pz) % Pz;
    const size_t plane = (size_t)Px * Py * Pz;
    const size_t off = ((size_t)zi * Py + yi) * Px + xi;
    for (int q = 0; q < 6; q++) W[q * plane + off] = make_double2(g6[q], 0.0);
}

// One FFT line per CTA of a complex FP64 (or FP32) volume; the line along
// axis ax of component q.  Used for the one-off tensor transforms.
template <typename C>
__global__ void k_fft_lines(C* data, int Px, int Py, int Pz, int ax, FftLen L, const C* tw, int sign)
{
    extern __shared__ unsigned char smraw[];
    C* A = reinterpret_cast<C*>(smraw);
    C* B = A + L.n;
    const long long line = blockIdx.x;
    const int q = blockIdx.y;
    long long base;
    int es;
    if (ax == 0) { base = line * Px; es = 1; }
    else if (ax == 1) { const long long zz = line / Px, xx = line % Px; base = zz * Px * Py + xx; es = Px; }
    else { base = line; es = Px * Py; }
    C* d = data + (size_t)q * Px * Py * Pz + base;
    for (int t = threadIdx.x; t < L.n; t += blockDim.x) A[t] = d[(size_t)t * es];
    __syncthreads();
    LineGeo g;
    g.nlines = 1; g.lpg = 1; g.gstride = 0; g.ls = 0; g.es = 1; g.line_fast = 0;
    const C* R = L.n > 1 ? cta_fft<C>(A, B, g, L, tw, sign) : A;
    for (int t = threadIdx.x; t < L.n; t += blockDim.x) d[(size_t)t * es] = R[t];
}

// Real symmetric tensor: TEN6[kx][kz][ky][q] = Re W_q(kx,ky,kz) in the
// state precision R (kmaj: TEN6[kx][ky][kz][q], the split-pass layout).
template <typename R>
__global__ void k_tensor_pack6(const double2* W, int Px, int Py, int Pz, int Kx, R* ten6, double* maxim, int kmaj)
{
    const long long total = (long long)Kx * Py * Pz;
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= total) return;
    const int kx = (int)(e / ((long long)Py * Pz));
    const int rem = (int)(e % ((long long)Py * Pz));
    const int kz = rem / Py, ky = rem % Py;
    const size_t plane = (size_t)Px * Py * Pz;
    const size_t off = ((size_t)kz * Py + ky) * Px + kx;
    const size_t o = kmaj ? ((size_t)kx * Py + ky) * Pz + kz : (size_t)e;
    double mi = 0;
    for (int q = 0; q < 6; q++) {
        const double2 v = W[q * plane + off];
        ten6[o * 6 + q] = (R)v.x;
        mi = fmax(mi, fabs(v.y));
    }
    if (maxim) {
        unsigned long long* p = reinterpret_cast<unsigned long long*>(maxim);
        atomicMax(p, (unsigned long long)__double_as_longlong(mi));
    }
}

// General 9-component complex tensor: TEN9[kx][kz][ky][q] (kmaj:
// TEN9[kx][ky][kz][q]).
template <typename R>
__global__ void k_tensor_pack9(const double2* W, int Px, int Py, int Pz, int Kx, typename CT<R>::T* ten9, int kmaj)
{
    const long long total = (long long)Kx * Py * Pz;
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= total) return;
    const int kx = (int)(e / ((long long)Py * Pz));
    const int rem = (int)(e % ((long long)Py * Pz));
    const int kz = rem / Py, ky = rem % Py;
    const size_t plane = (size_t)Px * Py * Pz;
    const size_t off = ((size_t)kz * Py + ky) * Px + kx;
    const size_t o = kmaj ? ((size_t)kx * Py + ky) * Pz + kz : (size_t)e;
    for (int q = 0; q < 9; q++) {
        const double2 v = W[q * plane + off];
        ten9[o * 9 + q] = cmk<typename CT<R>::T>((R)v.x, (R)v.y);
    }
}

// ------------------------------------------------------------ LongRange2D
// Layer-pair convolution, periodic in x and y (spinoperationlongrange2d.cpp:
// 430-530), between the x passes of the dipole convolution (k_conv_fx,
// k_conv_ix with Px = nx):
//   k_lr2d_ffty  one CTA per kx: the y transforms of the 3 nz spectrum rows
//                (comp, z) in shared memory, in place (sign -1 forward, +1
//                inverse);
//   k_lr2d_mix   CTA (kx, LR2D_KB consecutive ky): for each ky, destination
//                layer d and component a,
//                  H_a[d] = dst[d] * sum_s src[s] sum_b Q[kx][ky][s][d][ab] M_b[s]
//                (Q: the 2D transforms over nx ny of the arrays set for
//                (s, d), divided by nx ny -- the reference's apply reads its
//                tensors [s][d]).  Each CTA reads and writes only its own ky
//                columns, so the mixing runs in place; many CTAs per kx keep
//                the tensor stream (9 nz^2 complex per k-point) near the
//                HBM roofline.
constexpr int LR2D_KB = 8;

template <typename R>
__global__ void __launch_bounds__(512) k_lr2d_ffty(ConvK c, FftLen Ly, const typename CT<R>::T* tw,
                                                   typename CT<R>::T* spec, int sign)
{
    typedef typename CT<R>::T C;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* smf = reinterpret_cast<C*>(smraw);
    const int kx = blockIdx.x, ny = c.ny;
    const int NL = 3 * c.nz;
    C* A = smf;
    C* B = smf + (size_t)NL * ny;
    C* sp = spec + (size_t)kx * NL * ny;
    for (int t = threadIdx.x; t < NL * ny; t += blockDim.x) A[t] = sp[t];
    __syncthreads();
    LineGeo g;
    g.nlines = NL; g.lpg = 1 << 30; g.gstride = 0; g.ls = ny; g.es = 1; g.line_fast = 0;
    const C* cur = cta_fft<C>(A, B, g, Ly, tw, sign);
    for (int t = threadIdx.x; t < NL * ny; t += blockDim.x) sp[t] = cur[t];
}

// The mixing on the split layout S2[kx][ky][comp][z] (FP32 power-of-two
// ny, after k_sy_fast): a CTA's KB k-points are one contiguous block.
// NZS > 0: the layer count known at compile time, so that the source loop
// unrolls and each thread's tensor loads are all in flight together.
template <int NZS>
__global__ void __launch_bounds__(256) k_lr2d_mix_s2(ConvK c, float2* s2, const float2* Q, LR2DScale sc)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    const int nz = NZS > 0 ? NZS : c.nz;
    float2* Mk = reinterpret_cast<float2*>(smraw);   // [j][b][s]
    float2* Hk = Mk + (size_t)3 * nz * LR2D_KB;        // [j][a][d]
    const int kx = blockIdx.x, ky0 = blockIdx.y * LR2D_KB, ny = c.ny;
    const int nk = min(LR2D_KB, ny - ky0);
    const int NL = 3 * nz;
    pdl_wait();
    float2* base = s2 + ((size_t)kx * ny + ky0) * NL;
    for (int t = threadIdx.x; t < NL * nk; t += blockDim.x) Mk[t] = base[t];
    __syncthreads();
    const float2* Qk = Q + ((size_t)kx * ny + ky0) * nz * nz * 9;
    for (int t = threadIdx.x; t < NL * nk; t += blockDim.x) {
        const int a = t % 3, rest = t / 3, d = rest % nz, j = rest / nz;
        float2 acc = make_float2(0.f, 0.f);
#pragma unroll
        for (int s = 0; s < nz; s++) {
            const float2* q = Qk + (((size_t)j * nz + s) * nz + d) * 9 + 3 * a;
            const float w = (float)sc.src[s];
#pragma unroll
            for (int b = 0; b < 3; b++) {
                const float2 m = Mk[(size_t)j * NL + b * nz + s];
                const float2 qq = __ldcs(q + b);   // read once: evict first, S2 stays in L2
                acc = cadd(acc, cmul(make_float2(w * qq.x, w * qq.y), m));
            }
        }
        const float wd = (float)sc.dst[d];
        Hk[(size_t)j * NL + a * nz + d] = make_float2(wd * acc.x, wd * acc.y);
    }
    __syncthreads();
    pdl_trigger();
    for (int t = threadIdx.x; t < NL * nk; t += blockDim.x) base[t] = Hk[t];
}

template <typename R>
__global__ void __launch_bounds__(256) k_lr2d_mix(ConvK c, typename CT<R>::T* spec, const typename CT<R>::T* Q,
                                                  LR2DScale sc)
{
    typedef typename CT<R>::T C;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* Mk = reinterpret_cast<C*>(smraw);          // [b nz + s][LR2D_KB]: the CTA's spectrum columns
    C* Hk = Mk + (size_t)3 * c.nz * LR2D_KB;      // [a nz + d][LR2D_KB]: its output
    const int kx = blockIdx.x, ky0 = blockIdx.y * LR2D_KB, ny = c.ny, nz = c.nz;
    const int nk = min(LR2D_KB, ny - ky0);
    const int NL = 3 * nz;
    C* sp = spec + (size_t)kx * NL * ny + ky0;
    for (int t = threadIdx.x; t < NL * LR2D_KB; t += blockDim.x) {
        const int line = t / LR2D_KB, j = t % LR2D_KB;
        if (j < nk) Mk[t] = sp[(size_t)line * ny + j];
    }
    __syncthreads();
    const C* Qk = Q + ((size_t)kx * ny + ky0) * nz * nz * 9;
    for (int t = threadIdx.x; t < NL * nk; t += blockDim.x) {
        const int a = t % 3, rest = t / 3, d = rest % nz, j = rest / nz;
        C acc = cmk<C>((R)0, (R)0);
        for (int s = 0; s < nz; s++) {
            const C* q = Qk + (((size_t)j * nz + s) * nz + d) * 9 + 3 * a;
            const R w = (R)sc.src[s];
#pragma unroll
            for (int b = 0; b < 3; b++) {
                const C m = Mk[((size_t)b * nz + s) * LR2D_KB + j];
                const C qq = q[b];
                acc = cadd(acc, cmul(cmk<C>(w * qq.x, w * qq.y), m));
            }
        }
        const R wd = (R)sc.dst[d];
        Hk[((size_t)a * nz + d) * LR2D_KB + j] = cmk<C>(wd * acc.x, wd * acc.y);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < NL * LR2D_KB; t += blockDim.x) {
        const int line = t / LR2D_KB, j = t % LR2D_KB;
        if (j < nk) sp[(size_t)line * ny + j] = Hk[t];
    }
}

// ------------------------------------------------------------ split (y,z) passes
// For (y,z) planes larger than one CTA's shared memory (a 256^3 open cube
// pads to 512 x 512 planes): the plane pass of k_conv_yz done as three
// passes through S2[kx][ky][comp][z] (data layers z < nz only).
//   k_split_y   CTA (kx, comp, SPLIT_ZB data layers): y FFT of the layers'
//               rows (zero-padded to Py), stored ky-major in S2;
//   k_split_z   CTA (kx, ky): z FFT of the three components' columns
//               (zero-padded to Pz), tensor multiply (ky-major tensor),
//               inverse z FFT, data layers back to S2;
//   k_split_yi  CTA (kx, comp, SPLIT_ZB layers): inverse y FFT, data rows to
//               SPEC[kx][comp][z][y].
// The arithmetic per element is that of k_conv_yz: same FFTs, same multiply.
constexpr int SPLIT_ZB = 8;

template <typename R>
__global__ void __launch_bounds__(256) k_split_y(ConvK c, FftLen Ly, const typename CT<R>::T* tw,
                                                 const typename CT<R>::T* spec, typename CT<R>::T* s2)
{
    if (c.run_if && *c.run_if == 0) return;
    typedef typename CT<R>::T C;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* A = reinterpret_cast<C*>(smraw);
    C* B = A + SPLIT_ZB * c.Py;
    const int kx = blockIdx.x, comp = blockIdx.y, z0 = blockIdx.z * SPLIT_ZB;
    const int nl = min(SPLIT_ZB, c.nz - z0);
    const C* src = spec + (((size_t)kx * 3 + comp) * c.nz + z0) * c.ny;
    for (int t = threadIdx.x; t < nl * c.Py; t += blockDim.x) {
        const int l = t / c.Py, y = t % c.Py;
        A[t] = y < c.ny ? src[(size_t)l * c.ny + y] : cmk<C>((R)0, (R)0);
    }
    __syncthreads();
    LineGeo g;
    g.nlines = nl; g.lpg = 1 << 30; g.gstride = 0; g.ls = c.Py; g.es = 1; g.line_fast = 0;
    const C* Rl = c.Py > 1 ? cta_fft<C>(A, B, g, Ly, tw, -1) : A;
    for (int t = threadIdx.x; t < nl * c.Py; t += blockDim.x) {
        const int l = t % nl, ky = t / nl;
        s2[(((size_t)kx * c.Py + ky) * 3 + comp) * c.nz + z0 + l] = Rl[l * c.Py + ky];
    }
}

template <typename R>
__global__ void __launch_bounds__(256) k_split_z(ConvK c, FftLen Lz, const typename CT<R>::T* tw,
                                                 typename CT<R>::T* s2, const R* ten6, const typename CT<R>::T* ten9)
{
    if (c.run_if && *c.run_if == 0) return;
    typedef typename CT<R>::T C;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* A = reinterpret_cast<C*>(smraw);
    C* B = A + 3 * c.Pz;
    const int kx = blockIdx.x, ky = blockIdx.y;
    const int Pz = c.Pz;
    C* col = s2 + ((size_t)kx * c.Py + ky) * 3 * c.nz;
    for (int t = threadIdx.x; t < 3 * Pz; t += blockDim.x) {
        const int comp = t / Pz, z = t % Pz;
        A[t] = z < c.nz ? col[comp * c.nz + z] : cmk<C>((R)0, (R)0);
    }
    __syncthreads();
    LineGeo g;
    g.nlines = 3; g.lpg = 1 << 30; g.gstride = 0; g.ls = Pz; g.es = 1; g.line_fast = 0;
    C* cur = A;
    C* oth = B;
    if (Pz > 1) { cur = cta_fft<C>(cur, oth, g, Lz, tw, -1); oth = cur == A ? B : A; }
    const R gg = (R)c.g;
    const size_t tb = ((size_t)kx * c.Py + ky) * Pz;
    if (!c.general) {
        for (int t = threadIdx.x; t < Pz; t += blockDim.x) {
            const R* T = ten6 + (tb + t) * 6;
            const R t0 = __ldg(T), t1 = __ldg(T + 1), t2 = __ldg(T + 2);
            const R t3 = __ldg(T + 3), t4 = __ldg(T + 4), t5 = __ldg(T + 5);
            const C s0 = cur[t], s1 = cur[Pz + t], s2v = cur[2 * Pz + t];
            cur[t] = cmk<C>(gg * (t0 * s0.x + t1 * s1.x + t2 * s2v.x), gg * (t0 * s0.y + t1 * s1.y + t2 * s2v.y));
            cur[Pz + t] = cmk<C>(gg * (t1 * s0.x + t3 * s1.x + t4 * s2v.x), gg * (t1 * s0.y + t3 * s1.y + t4 * s2v.y));
            cur[2 * Pz + t] =
                cmk<C>(gg * (t2 * s0.x + t4 * s1.x + t5 * s2v.x), gg * (t2 * s0.y + t4 * s1.y + t5 * s2v.y));
        }
    } else {
        for (int t = threadIdx.x; t < Pz; t += blockDim.x) {
            const C* T = ten9 + (tb + t) * 9;
            const C s[3] = {cur[t], cur[Pz + t], cur[2 * Pz + t]};
#pragma unroll
            for (int a = 0; a < 3; a++) {
                C acc = cmk<C>((R)0, (R)0);
#pragma unroll
                for (int b = 0; b < 3; b++) acc = cadd(acc, cmul(T[3 * a + b], s[b]));
                cur[a * Pz + t] = cmk<C>(gg * acc.x, gg * acc.y);
            }
        }
    }
    __syncthreads();
    if (Pz > 1) { cur = cta_fft<C>(cur, oth, g, Lz, tw, +1); }
    for (int t = threadIdx.x; t < 3 * c.nz; t += blockDim.x) {
        const int comp = t / c.nz, z = t % c.nz;
        col[t] = cur[comp * Pz + z];
    }
}

template <typename R>
__global__ void __launch_bounds__(256) k_split_yi(ConvK c, FftLen Ly, const typename CT<R>::T* tw,
                                                  const typename CT<R>::T* s2, typename CT<R>::T* spec)
{
    if (c.run_if && *c.run_if == 0) return;
    typedef typename CT<R>::T C;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* A = reinterpret_cast<C*>(smraw);
    C* B = A + SPLIT_ZB * c.Py;
    const int kx = blockIdx.x, comp = blockIdx.y, z0 = blockIdx.z * SPLIT_ZB;
    const int nl = min(SPLIT_ZB, c.nz - z0);
    for (int t = threadIdx.x; t < nl * c.Py; t += blockDim.x) {
        const int l = t % nl, ky = t / nl;
        A[l * c.Py + ky] = s2[(((size_t)kx * c.Py + ky) * 3 + comp) * c.nz + z0 + l];
    }
    __syncthreads();
    LineGeo g;
    g.nlines = nl; g.lpg = 1 << 30; g.gstride = 0; g.ls = c.Py; g.es = 1; g.line_fast = 0;
    const C* Rl = c.Py > 1 ? cta_fft<C>(A, B, g, Ly, tw, +1) : A;
    C* dst = spec + (((size_t)kx * 3 + comp) * c.nz + z0) * c.ny;
    for (int t = threadIdx.x; t < nl * c.ny; t += blockDim.x) {
        const int l = t / c.ny, y = t % c.ny;
        dst[(size_t)l * c.ny + y] = Rl[l * c.Py + y];
    }
}

// ------------------------------------------------------------ launchers
#include <map>
#include <string>
#include <vector>

namespace mlb {

// Opt-in per-kernel timing: launchers bracket their kernels with CUDA
// events on the launching stream while profiling is on (never inside a
// graph capture); prof_end() sums elapsed times per kernel name.
namespace {
struct ProfRec {
    const char* name;
    cudaEvent_t a, b;
};
bool g_prof = false;
std::vector<ProfRec> g_recs;
std::vector<cudaEvent_t> g_pool;
std::vector<ProfCaptured>* g_sink = nullptr;
} // namespace

void prof_set_capture_sink(std::vector<ProfCaptured>* sink) { g_sink = sink; }

int prof_active(cudaStream_t st)
{
    cudaStreamCaptureStatus cs;
    if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) return 0;
    if (cs != cudaStreamCaptureStatusNone) return g_sink ? 2 : 0;
    return g_prof ? 1 : 0;
}

void prof_push_captured(const char* name, cudaEvent_t a, cudaEvent_t b)
{
    if (g_sink) g_sink->push_back({name, a, b});
}

cudaEvent_t prof_event()
{
    if (!g_pool.empty()) {
        cudaEvent_t e = g_pool.back();
        g_pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}

void prof_push(const char* name, cudaEvent_t a, cudaEvent_t b) { g_recs.push_back({name, a, b}); }

void prof_begin()
{
    g_prof = true;
    g_recs.clear();
}

int prof_end(int cap, char* names, double* ms, int* launches)
{
    std::map<std::string, std::pair<double, int>> agg;
    std::vector<std::string> order;
    for (ProfRec& r : g_recs) {
        cudaEventSynchronize(r.b);
        float t = 0.f;
        cudaEventElapsedTime(&t, r.a, r.b);
        if (!agg.count(r.name)) order.push_back(r.name);
        agg[r.name].first += t;
        agg[r.name].second += 1;
        g_pool.push_back(r.a);
        g_pool.push_back(r.b);
    }
    g_recs.clear();
    g_prof = false;
    int k = 0;
    for (const std::string& nm : order) {
        if (k >= cap) break;
        snprintf(names + 48 * k, 48, "%s", nm.c_str());
        ms[k] = agg[nm].first;
        launches[k] = agg[nm].second;
        k++;
    }
    return k;
}

static inline unsigned blocks_for(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

cudaError_t launch_fused(const FusedK& P, double dt_sys, int rb, cudaStream_t st)
{
    if (P.sys.n == 0) return cudaSuccess;
    Prof pf("k_fused_step", st);
    if (rb == 8) k_fused_step<double><<<blocks_for(P.sys.n, 256), 256, 0, st>>>(P, dt_sys);
    else k_fused_step<float><<<blocks_for(P.sys.n, 256), 256, 0, st>>>(P, dt_sys);
    return cudaGetLastError();
}

cudaError_t launch_eval(const SysK& s, const TermsK& T, double dt_sys, void* const h[3], int acc, int rb,
                        cudaStream_t st)
{
    if (s.n == 0) return cudaSuccess;
    Prof pf("k_eval_terms", st);
    if (rb == 8) k_eval_terms<double><<<blocks_for(s.n, 256), 256, 0, st>>>(s, T, dt_sys, h[0], h[1], h[2], acc);
    else k_eval_terms<float><<<blocks_for(s.n, 256), 256, 0, st>>>(s, T, dt_sys, h[0], h[1], h[2], acc);
    return cudaGetLastError();
}

cudaError_t launch_llg(const SysK& from, const void* const m[3], const void* const H[3], const void* const Ht[3],
                       const void* dsa, const void* dsg, double da, double dg, const LlgK& L,
                       void* const out[3], int rb, cudaStream_t st)
{
    if (from.n == 0) return cudaSuccess;
    Prof pf("k_llg", st);
    if (rb == 8)
        k_llg<double><<<blocks_for(from.n, 256), 256, 0, st>>>(from, m[0], m[1], m[2], H[0], H[1], H[2], Ht[0],
                                                               Ht[1], Ht[2], dsa, dsg, da, dg, L, out[0], out[1],
                                                               out[2]);
    else
        k_llg<float><<<blocks_for(from.n, 256), 256, 0, st>>>(from, m[0], m[1], m[2], H[0], H[1], H[2], Ht[0],
                                                              Ht[1], Ht[2], dsa, dsg, da, dg, L, out[0], out[1],
                                                              out[2]);
    return cudaGetLastError();
}

cudaError_t launch_advance_step(const DevStep* cur, DevStep* next, cudaStream_t st)
{
    return launch_pdl(k_advance_step, dim3(1), dim3(1), 0, st, cur, next);
}

cudaError_t launch_partial_final(const double* part, int nb, int nq, double* out, cudaStream_t st)
{
    k_partial_final<<<nq, 256, 0, st>>>(part, nb, nq, out);
    return cudaGetLastError();
}

cudaError_t launch_netmoment(const void* x, const void* y, const void* z, int n, double m, double* part, int nb,
                             double* out, int rb, cudaStream_t st)
{
    if (rb == 8) k_netmoment_partial<double><<<nb, 256, 0, st>>>(x, y, z, n, m, part);
    else k_netmoment_partial<float><<<nb, 256, 0, st>>>(x, y, z, n, m, part);
    k_partial_final<<<6, 256, 0, st>>>(part, nb, 6, out);
    return cudaGetLastError();
}

cudaError_t launch_diff(const void* const a[3], const void* const b[3], int n, double* part, int nb, double* out,
                        int rb, cudaStream_t st)
{
    if (rb == 8) k_diff_partial<double><<<nb, 256, 0, st>>>(a[0], a[1], a[2], b[0], b[1], b[2], n, part);
    else k_diff_partial<float><<<nb, 256, 0, st>>>(a[0], a[1], a[2], b[0], b[1], b[2], n, part);
    k_partial_final<<<3, 256, 0, st>>>(part, nb, 3, out);
    return cudaGetLastError();
}

cudaError_t launch_dot(const void* const s[3], const void* const h[3], int n, double* part, int nb, double* out,
                       int rb, cudaStream_t st)
{
    if (rb == 8) k_dot_partial<double><<<nb, 256, 0, st>>>(s[0], s[1], s[2], h[0], h[1], h[2], n, part);
    else k_dot_partial<float><<<nb, 256, 0, st>>>(s[0], s[1], s[2], h[0], h[1], h[2], n, part);
    k_partial_final<<<1, 256, 0, st>>>(part, nb, 1, out);
    return cudaGetLastError();
}

size_t conv_x_smem(const ConvK& c, int rb) { return (size_t)2 * c.ty * c.Px * 2 * rb; }
size_t conv_yz_smem(const ConvK& c, int rb) { return (size_t)6 * c.Py * c.Pz * 2 * rb; }

template <typename K>
static cudaError_t max_smem(K kern)
{
    return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
}

cudaError_t conv_configure()
{
    cudaError_t e;
    if ((e = max_smem(k_conv_yz<float>)) != cudaSuccess) return e;
    if ((e = max_smem(k_conv_yz<double>)) != cudaSuccess) return e;
    if ((e = max_smem(k_conv_fx<float>)) != cudaSuccess) return e;
    if ((e = max_smem(k_conv_fx<double>)) != cudaSuccess) return e;
    if ((e = max_smem(k_conv_ix<float>)) != cudaSuccess) return e;
    if ((e = max_smem(k_conv_ix<double>)) != cudaSuccess) return e;
    if ((e = max_smem(k_split_y<float>)) || (e = max_smem(k_split_y<double>)) || (e = max_smem(k_split_yi<float>)) ||
        (e = max_smem(k_split_yi<double>)) || (e = max_smem(k_split_z<float>)) || (e = max_smem(k_split_z<double>)))
        return e;
    if ((e = max_smem(k_lr2d_mix_s2<0>)) || (e = max_smem(k_lr2d_mix_s2<4>)) || (e = max_smem(k_lr2d_mix_s2<8>)) ||
        (e = max_smem(k_lr2d_mix_s2<16>)) || (e = max_smem(k_lr2d_ffty<float>)) || (e = max_smem(k_lr2d_ffty<double>)) ||
        (e = max_smem(k_lr2d_mix<float>)) || (e = max_smem(k_lr2d_mix<double>)))
        return e;
    return max_smem(k_fft_lines<double2>);
}

template <typename R>
static void conv_generic(const ConvK& c, const FftLen& Lx, const FftLen& Ly, const FftLen& Lz, const void* tw_,
                         const void* const s[3], void* spec_, const void* ten6, const void* ten9, void* const h[3],
                         cudaStream_t st)
{
    typedef typename CT<R>::T C;
    const C* tw = static_cast<const C*>(tw_);
    C* spec = static_cast<C*>(spec_);
    dim3 gx(blocks_for(c.ny, c.ty), c.nz);
    const FftLen L3[3] = {Lx, Ly, Lz};
    // FP64 state with a power-of-two x length: the fast x passes in double
    const bool fx64 = sizeof(R) == 8 && x_fast_ok_f64(c);
    const double* sd[3] = {static_cast<const double*>(s[0]), static_cast<const double*>(s[1]),
                           static_cast<const double*>(s[2])};
    double* hd[3] = {static_cast<double*>(h[0]), static_cast<double*>(h[1]), static_cast<double*>(h[2])};
    if (fx64) {
        launch_x_pass_f64(c, L3, static_cast<const double2*>(tw_), sd, static_cast<double2*>(spec_), hd, true, st);
    } else {
        Prof pf("k_conv_fx", st);
        k_conv_fx<R><<<gx, 256, conv_x_smem(c, sizeof(R)), st>>>(c, Lx, tw, s[0], s[1], s[2], spec);
    }
    if (c.split) {
        if (sizeof(R) == 8 && split_fast_ok_f64(c))
            launch_split_fast_f64(c, L3, static_cast<const double2*>(tw_), static_cast<double2*>(spec_),
                                  static_cast<const double*>(ten6), st);
        else
            launch_conv_split_yz(c, Ly, Lz, tw_, spec_, ten6, ten9, (int)sizeof(R), st);
    } else {
        Prof pf("k_conv_yz", st);
        k_conv_yz<R><<<c.Kx, 512, conv_yz_smem(c, sizeof(R)), st>>>(c, Ly, Lz, tw, spec, static_cast<const R*>(ten6),
                                                                    static_cast<const C*>(ten9));
    }
    if (fx64) {
        launch_x_pass_f64(c, L3, static_cast<const double2*>(tw_), sd, static_cast<double2*>(spec_), hd, false, st);
    } else {
        Prof pf("k_conv_ix", st);
        k_conv_ix<R><<<gx, 256, conv_x_smem(c, sizeof(R)), st>>>(c, Lx, tw, spec, h[0], h[1], h[2]);
    }
}

cudaError_t launch_conv(const ConvK& c, const FftLen& Lx, const FftLen& Ly, const FftLen& Lz, const void* tw,
                        const void* const s[3], void* spec, const void* ten6, const void* ten9, void* const h[3],
                        int rb, cudaStream_t st)
{
    if (rb == 8) conv_generic<double>(c, Lx, Ly, Lz, tw, s, spec, ten6, ten9, h, st);
    else conv_generic<float>(c, Lx, Ly, Lz, tw, s, spec, ten6, ten9, h, st);
    return cudaGetLastError();
}

cudaError_t launch_tensor_lattice(int nx, int ny, int nz, const int gmax[4], const double ABC[9], int Px,
                                  int Py, int Pz, int zsign, double2* W, cudaStream_t st)
{
    const long long ne = (long long)nx * ny * (2 * nz - 1);
    const int lim0 = gmax[0];
    const int limx = gmax[2] < gmax[0] ? gmax[2] : gmax[0];
    const int limy = gmax[3] < gmax[0] ? gmax[3] : gmax[0];
    k_tensor_lattice<<<blocks_for(ne, 128), 128, 0, st>>>(nx, ny, nz, gmax[0], lim0, limx, limy, ABC[0], ABC[1],
                                                          ABC[2], ABC[3], ABC[4], ABC[5], ABC[6], ABC[7], ABC[8],
                                                          Px, Py, Pz, zsign, W);
    return cudaGetLastError();
}

cudaError_t launch_tensor_rings(int nx, int ny, int nz, int nrings, int lstep, const double ABC[9], int Px, int Py,
                                int Pz, int zsign, double2* W, cudaStream_t st)
{
    const long long ne = (long long)nx * ny * (2 * nz - 1);
    k_tensor_rings<<<blocks_for(ne * 32, 256), 256, 0, st>>>(nx, ny, nz, nrings, lstep, ABC[0], ABC[1], ABC[2], ABC[3],
                                                              ABC[4], ABC[5], ABC[6], ABC[7], ABC[8], Px, Py, Pz,
                                                              zsign, W);
    return cudaGetLastError();
}

cudaError_t launch_tensor_extract_ref(int nx, int ny, int nz, int Px, int Py, int Pz, int zsign,
                                      const double2* W, double* out, cudaStream_t st)
{
    const long long ne = (long long)nx * ny * (2 * nz - 1);
    k_tensor_extract_ref<<<blocks_for(ne, 256), 256, 0, st>>>(nx, ny, nz, Px, Py, Pz, zsign, W, out);
    return cudaGetLastError();
}

cudaError_t launch_tensor_open(int nx, int ny, int nz, const double ABC[9], int Px, int Py, int Pz,
                               double2* W, cudaStream_t st)
{
    const long long ne = (long long)(2 * nx - 1) * (2 * ny - 1) * (2 * nz - 1);
    k_tensor_open<<<blocks_for(ne, 256), 256, 0, st>>>(nx, ny, nz, ABC[0], ABC[1], ABC[2], ABC[3], ABC[4],
                                                       ABC[5], ABC[6], ABC[7], ABC[8], Px, Py, Pz, W);
    return cudaGetLastError();
}

cudaError_t launch_fft3d_d(double2* W, int ncomp, int Px, int Py, int Pz, const FftLen L[3],
                           const double2* tw, int sign, cudaStream_t st)
{
    const int P[3] = {Px, Py, Pz};
    for (int ax = 0; ax < 3; ax++) {
        if (P[ax] == 1) continue;
        const long long nlines = (long long)Px * Py * Pz / P[ax];
        dim3 g((unsigned)nlines, ncomp);
        const size_t sm = (size_t)2 * P[ax] * sizeof(double2);
        k_fft_lines<double2><<<g, 128, sm, st>>>(W, Px, Py, Pz, ax, L[ax], tw, sign);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// LongRange2D tensor: Q[kx][ky][s][d][ab] = W_{(s d ab)}(kx, ky) / (nx ny) for
// the layer pairs p0 .. p0 + np - 1 (p = s nz + d), W holding their
// transforms [(p - p0) 9 + ab][ky][kx] over the full x length.
template <typename R>
__global__ void k_lr2d_pack(const double2* W, int nx, int ny, int nz, int Kx, int p0, int np,
                            typename CT<R>::T* Q)
{
    const long long total = (long long)Kx * ny * np * 9;
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= total) return;
    const int ab = (int)(e % 9);
    long long r = e / 9;
    const int pl = (int)(r % np);
    r /= np;
    const int ky = (int)(r % ny), kx = (int)(r / ny);
    const double inv = 1.0 / ((double)nx * ny);
    const double2 v = W[((size_t)pl * 9 + ab) * nx * ny + (size_t)ky * nx + kx];
    const size_t o = (((size_t)kx * ny + ky) * nz * nz + p0 + pl) * 9 + ab;
    Q[o] = cmk<typename CT<R>::T>((R)(v.x * inv), (R)(v.y * inv));
}

cudaError_t launch_lr2d_pack(const double2* W, int nx, int ny, int nz, int p0, int np, void* Q, int rb,
                             cudaStream_t st)
{
    const int Kx = nx / 2 + 1;
    const long long total = (long long)Kx * ny * np * 9;
    if (rb == 8)
        k_lr2d_pack<double><<<blocks_for(total, 256), 256, 0, st>>>(W, nx, ny, nz, Kx, p0, np, static_cast<double2*>(Q));
    else
        k_lr2d_pack<float><<<blocks_for(total, 256), 256, 0, st>>>(W, nx, ny, nz, Kx, p0, np, static_cast<float2*>(Q));
    return cudaGetLastError();
}

size_t lr2d_smem(const ConvK& c, int rb) { return (size_t)6 * c.nz * c.ny * 2 * rb; }

// x passes: the FP32 power-of-two kernels of conv_fast.cu where they apply
// (x_fast_ok), else the generic mixed-radix ones
template <typename R>
static void lr2d_t(const ConvK& c, const FftLen L[3], const void* tw_, const void* const s[3], void* spec_,
                   const void* Q, const LR2DScale& sc, void* const h[3], cudaStream_t st)
{
    typedef typename CT<R>::T C;
    const C* tw = static_cast<const C*>(tw_);
    C* spec = static_cast<C*>(spec_);
    dim3 gx(blocks_for(c.ny, c.ty), c.nz);
    const bool fast = sizeof(R) == 4 && x_fast_ok(c);
    const float* sf[3] = {static_cast<const float*>(s[0]), static_cast<const float*>(s[1]),
                          static_cast<const float*>(s[2])};
    float* hf[3] = {static_cast<float*>(h[0]), static_cast<float*>(h[1]), static_cast<float*>(h[2])};
    if (fast) {
        launch_x_pass_fast(c, L, reinterpret_cast<const float2*>(tw), sf, reinterpret_cast<float2*>(spec), hf, true,
                           st);
    } else {
        Prof pf("k_conv_fx", st);
        k_conv_fx<R><<<gx, 256, conv_x_smem(c, sizeof(R)), st>>>(c, L[0], tw, s[0], s[1], s[2], spec);
    }
    if (fast && split_y_fast_ok(c) && c.spec2) {
        // register y transforms through S2 and the mixing on that layout
        float2* sp2 = reinterpret_cast<float2*>(spec);
        launch_split_y_fast(c, L, reinterpret_cast<const float2*>(tw), sp2, true, st);
        {
            Prof pf("k_lr2d_mix", st);
            const size_t sm = (size_t)6 * c.nz * LR2D_KB * sizeof(float2);
            auto kern = c.nz == 8 ? k_lr2d_mix_s2<8> : c.nz == 4 ? k_lr2d_mix_s2<4> :
                        c.nz == 16 ? k_lr2d_mix_s2<16> : k_lr2d_mix_s2<0>;
            // one thread per (k-point, component, layer) item, whole warps
            const int nt = std::min(256, (3 * c.nz * LR2D_KB + 31) / 32 * 32);
            launch_pdl(kern, dim3(c.Kx, (c.ny + LR2D_KB - 1) / LR2D_KB), dim3(nt), sm, st, c,
                       static_cast<float2*>(c.spec2), reinterpret_cast<const float2*>(Q), sc);
        }
        launch_split_y_fast(c, L, reinterpret_cast<const float2*>(tw), sp2, false, st);
        launch_x_pass_fast(c, L, reinterpret_cast<const float2*>(tw), sf, sp2, hf, false, st);
        return;
    }
    if (c.ny > 1) {
        Prof pf("k_lr2d_ffty", st);
        k_lr2d_ffty<R><<<c.Kx, 512, lr2d_smem(c, sizeof(R)), st>>>(c, L[1], tw, spec, -1);
    }
    {
        Prof pf("k_lr2d_mix", st);
        const size_t sm = (size_t)6 * c.nz * LR2D_KB * sizeof(C);
        k_lr2d_mix<R><<<dim3(c.Kx, (c.ny + LR2D_KB - 1) / LR2D_KB), 256, sm, st>>>(c, spec, static_cast<const C*>(Q),
                                                                                    sc);
    }
    if (c.ny > 1) {
        Prof pf("k_lr2d_ffty", st);
        k_lr2d_ffty<R><<<c.Kx, 512, lr2d_smem(c, sizeof(R)), st>>>(c, L[1], tw, spec, +1);
    }
    if (fast) {
        launch_x_pass_fast(c, L, reinterpret_cast<const float2*>(tw), sf, reinterpret_cast<float2*>(spec), hf, false,
                           st);
    } else {
        Prof pf("k_conv_ix", st);
        k_conv_ix<R><<<gx, 256, conv_x_smem(c, sizeof(R)), st>>>(c, L[0], tw, spec, h[0], h[1], h[2]);
    }
}

cudaError_t launch_lr2d(const ConvK& c, const FftLen L[3], const void* tw, const void* const s[3], void* spec,
                        const void* Q, const LR2DScale& sc, void* const h[3], int rb, cudaStream_t st)
{
    if (rb == 8) lr2d_t<double>(c, L, tw, s, spec, Q, sc, h, st);
    else lr2d_t<float>(c, L, tw, s, spec, Q, sc, h, st);
    return cudaGetLastError();
}

// Largest |W|, and the largest deviations from the parities T(kx, -ky, kz)
// = s_y(q) T(kx, ky, kz) and T(kx, ky, -kz) = s_z(q) T(kx, ky, kz) of the
// real parts of the six transformed components (XY, YZ odd in ky; XZ, YZ
// odd in kz), as the bits of non-negative doubles.
__global__ void k_tensor_symcheck(const double2* W, int Px, int Py, int Pz, int Kx, unsigned long long* out)
{
    const long long total = (long long)6 * Kx * Py * Pz;
    unsigned long long m[3] = {0ull, 0ull, 0ull};
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int q = (int)(e % 6);
        long long r = e / 6;
        const int kx = (int)(r % Kx);
        r /= Kx;
        const int ky = (int)(r % Py), kz = (int)(r / Py);
        const size_t plane = (size_t)Px * Py * Pz;
        const double2* Wq = W + q * plane;
        const double v = Wq[((size_t)kz * Py + ky) * Px + kx].x;
        const double vy = Wq[((size_t)kz * Py + (Py - ky) % Py) * Px + kx].x;
        const double vz = Wq[((size_t)((Pz - kz) % Pz) * Py + ky) * Px + kx].x;
        const double sy = (q == 1 || q == 4) ? -1.0 : 1.0;
        const double sz = (q == 2 || q == 4) ? -1.0 : 1.0;
        // non-negative doubles order as their bit patterns
        m[0] = max(m[0], (unsigned long long)__double_as_longlong(fabs(v)));
        m[1] = max(m[1], (unsigned long long)__double_as_longlong(fabs(vy - sy * v)));
        m[2] = max(m[2], (unsigned long long)__double_as_longlong(fabs(vz - sz * v)));
    }
    for (int k = 0; k < 3; k++) {
        unsigned long long x = m[k];
        for (int o = 16; o > 0; o >>= 1) x = max(x, __shfl_xor_sync(0xffffffffu, x, o));
        if ((threadIdx.x & 31) == 0 && x) atomicMax(out + k, x);
    }
}

// Quarter tensor TEN6Q[kx][ky <= Py/2][kz <= Pz/2][q] = Re W_q in FP32.
// Quarter tensor (ky <= Py/2, kz <= Pz/2): ky-major TEN[kx][ky][kz][6] for the
// split passes, or (zmaj) TEN[kx][kz][ky][6] with the per-kx stride padded to
// a multiple of four floats for the single-CTA-plane (y,z) kernel.
__global__ void k_tensor_pack6q(const double2* W, int Px, int Py, int Pz, int Kx, float* ten, int zmaj)
{
    const int Qy = Py / 2 + 1, Qz = Pz / 2 + 1;
    const long long total = (long long)Kx * Qy * Qz;
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= total) return;
    int kx, ky, kz;
    size_t o;
    if (zmaj) {
        ky = (int)(e % Qy);
        const long long r = e / Qy;
        kz = (int)(r % Qz);
        kx = (int)(r / Qz);
        const size_t ks = ((size_t)Qz * Qy * 6 + 3) & ~(size_t)3;
        o = (size_t)kx * ks + ((size_t)kz * Qy + ky) * 6;
    } else {
        kz = (int)(e % Qz);
        const long long r = e / Qz;
        ky = (int)(r % Qy);
        kx = (int)(r / Qy);
        o = (size_t)e * 6;
    }
    const size_t plane = (size_t)Px * Py * Pz;
    const size_t off = ((size_t)kz * Py + ky) * Px + kx;
    for (int q = 0; q < 6; q++) ten[o + q] = (float)W[q * plane + off].x;
}

cudaError_t launch_tensor_symcheck(const double2* W, int Px, int Py, int Pz, int Kx, unsigned long long* out3,
                                   cudaStream_t st)
{
    const long long total = (long long)6 * Kx * Py * Pz;
    const long long nb = std::min<long long>(blocks_for(total, 256), 148LL * 8);
    k_tensor_symcheck<<<(unsigned)nb, 256, 0, st>>>(W, Px, Py, Pz, Kx, out3);
    return cudaGetLastError();
}

cudaError_t launch_tensor_pack6q(const double2* W, int Px, int Py, int Pz, int Kx, float* ten, int zmaj,
                                cudaStream_t st)
{
    const long long total = (long long)Kx * (Py / 2 + 1) * (Pz / 2 + 1);
    k_tensor_pack6q<<<blocks_for(total, 256), 256, 0, st>>>(W, Px, Py, Pz, Kx, ten, zmaj);
    return cudaGetLastError();
}

cudaError_t launch_tensor_pack6(const double2* W, int Px, int Py, int Pz, int Kx, void* ten6, double* maxim,
                                int rb, int kmaj, cudaStream_t st)
{
    const long long total = (long long)Kx * Py * Pz;
    if (rb == 8)
        k_tensor_pack6<double><<<blocks_for(total, 256), 256, 0, st>>>(W, Px, Py, Pz, Kx, static_cast<double*>(ten6),
                                                                       maxim, kmaj);
    else
        k_tensor_pack6<float><<<blocks_for(total, 256), 256, 0, st>>>(W, Px, Py, Pz, Kx, static_cast<float*>(ten6),
                                                                      maxim, kmaj);
    return cudaGetLastError();
}

cudaError_t launch_tensor_pack9(const double2* W, int Px, int Py, int Pz, int Kx, void* ten9, int rb, int kmaj,
                                cudaStream_t st)
{
    const long long total = (long long)Kx * Py * Pz;
    if (rb == 8)
        k_tensor_pack9<double><<<blocks_for(total, 256), 256, 0, st>>>(W, Px, Py, Pz, Kx, static_cast<double2*>(ten9),
                                                                       kmaj);
    else
        k_tensor_pack9<float><<<blocks_for(total, 256), 256, 0, st>>>(W, Px, Py, Pz, Kx, static_cast<float2*>(ten9),
                                                                      kmaj);
    return cudaGetLastError();
}

size_t split_smem(const ConvK& c, int rb)
{
    const size_t cb = (size_t)2 * rb;
    return std::max((size_t)2 * SPLIT_ZB * c.Py * cb, (size_t)6 * c.Pz * cb);
}

template <typename R>
static void split_t(const ConvK& c, const FftLen& Ly, const FftLen& Lz, const void* tw_, void* spec_,
                    const void* ten6, const void* ten9, cudaStream_t st)
{
    typedef typename CT<R>::T C;
    const C* tw = static_cast<const C*>(tw_);
    C* spec = static_cast<C*>(spec_);
    C* s2 = static_cast<C*>(c.spec2);
    const size_t cb = 2 * sizeof(R);
    dim3 gy(c.Kx, 3, (c.nz + SPLIT_ZB - 1) / SPLIT_ZB);
    const size_t smy = (size_t)2 * SPLIT_ZB * c.Py * cb;
    k_split_y<R><<<gy, 256, smy, st>>>(c, Ly, tw, spec, s2);
    k_split_z<R><<<dim3(c.Kx, c.Py), 256, (size_t)6 * c.Pz * cb, st>>>(c, Lz, tw, s2, static_cast<const R*>(ten6),
                                                                       static_cast<const C*>(ten9));
    k_split_yi<R><<<gy, 256, smy, st>>>(c, Ly, tw, s2, spec);
}

cudaError_t launch_conv_split_yz(const ConvK& c, const FftLen& Ly, const FftLen& Lz, const void* tw, void* spec,
                                 const void* ten6, const void* ten9, int rb, cudaStream_t st)
{
    Prof pf("k_conv_yz_split", st);
    if (rb == 8) split_t<double>(c, Ly, Lz, tw, spec, ten6, ten9, st);
    else split_t<float>(c, Ly, Lz, tw, spec, ten6, ten9, st);
    return cudaGetLastError();
}

} // namespace mlb
