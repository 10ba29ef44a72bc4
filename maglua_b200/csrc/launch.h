// launch.h -- host-callable launchers for the kernels in kernels.cu.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include "device.cuh"
#include "kparams.h"

#include <vector>

namespace mlb {
// Launch with programmatic stream serialization: the kernel's CTAs may be
// scheduled before the previous kernel of the stream has finished (they
// wait in pdl_wait()), which hides the launch latency between the kernels
// of a step.
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                              Args... args)
{
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg;
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
}

// Kernel timing: 1 = eager profiling (mlb_profile_begin/end), 2 = event
// nodes inside a graph being captured for a plan with timing, 0 = off.
struct ProfCaptured {
    const char* name;
    cudaEvent_t a, b;
};
int prof_active(cudaStream_t st);
cudaEvent_t prof_event();
void prof_push(const char* name, cudaEvent_t a, cudaEvent_t b);
void prof_push_captured(const char* name, cudaEvent_t a, cudaEvent_t b);
void prof_set_capture_sink(std::vector<ProfCaptured>* sink);
// Scope timer used around kernel launches.
struct Prof {
    int mode;
    const char* name;
    cudaStream_t st;
    cudaEvent_t a = nullptr;
    Prof(const char* n, cudaStream_t s) : mode(prof_active(s)), name(n), st(s)
    {
        if (mode == 1) { a = prof_event(); cudaEventRecord(a, st); }
        else if (mode == 2) { cudaEventCreate(&a); cudaEventRecordWithFlags(a, st, cudaEventRecordExternal); }
    }
    ~Prof()
    {
        if (mode == 0) return;
        cudaEvent_t b;
        if (mode == 1) { b = prof_event(); cudaEventRecord(b, st); prof_push(name, a, b); }
        else { cudaEventCreate(&b); cudaEventRecordWithFlags(b, st, cudaEventRecordExternal); prof_push_captured(name, a, b); }
    }
};
cudaError_t fftreg_init();
cudaError_t conv_fast_configure();
bool conv_fast_ok(const ConvK& c);
// the 256-wide single-CTA-plane (y,z) kernel runs this pass (it can read a quarter tensor)
bool yz_col3_ok(const ConvK& c);
// FP32 x passes alone (power-of-two periodic x, 16..512): the forward
// transform of the spins to SPEC (fwd) or the inverse to the field h.
bool x_fast_ok(const ConvK& c);
// The fast x passes for FP64 state (power-of-two Px 16..512).
bool x_fast_ok_f64(const ConvK& c);
cudaError_t launch_x_pass_f64(const ConvK& c, const FftLen L[3], const double2* tw, const double* s[3],
                              double2* spec, double* h[3], bool fwd, cudaStream_t st);
// The register split (y,z) passes for FP64 state (power-of-two planes, real
// tensor).
bool split_fast_ok_f64(const ConvK& c);
cudaError_t launch_split_fast_f64(const ConvK& c, const FftLen L[3], const double2* tw, double2* spec,
                                  const double* ten6, cudaStream_t st);
// The FP32 split y passes alone: SPEC -> S2 (c.spec2) forward, S2 -> SPEC
// inverse, power-of-two Py 32..512.
bool split_y_fast_ok(const ConvK& c);
cudaError_t launch_split_y_fast(const ConvK& c, const FftLen L[3], const float2* tw, float2* spec, bool fwd,
                                cudaStream_t st);
cudaError_t launch_x_pass_fast(const ConvK& c, const FftLen L[3], const float2* tw, const float* s[3], float2* spec,
                               float* h[3], bool fwd, cudaStream_t st);
cudaError_t launch_conv_fast(const ConvK& c, const FftLen L[3], const float2* tw, const float* s[3], float2* spec,
                             const float* ten6, float* h[3], cudaStream_t st);
// The (y,z) pass, optionally preceded by the forward x pass, without the
// inverse x pass: the fused x pass (launch_xstep) completes the step.
cudaError_t launch_conv_fast_fyz(const ConvK& c, const FftLen L[3], const float2* tw, const float* s[3], float2* spec,
                                 const float* ten6, bool with_fx, cudaStream_t st);
cudaError_t launch_conv_fast_ix(const ConvK& c, const FftLen L[3], const float2* tw, float2* spec, float* h[3],
                                cudaStream_t st);
bool xstep_ok(const ConvK& c, const FastK& F);
// Inverse x pass + fused step (+ forward x pass of the new spins when fwd).
cudaError_t launch_xstep(const ConvK& c, const FftLen L[3], const float2* tw, float2* spec, const FastK& F,
                         bool fwd, const float* s[3], float* h[3], float* o[3], cudaStream_t st);
cudaError_t launch_fused_fast(const FastK& F, const float* s[3], const float* a[3], float* o[3], cudaStream_t st);
// the same for FP64 state (constants in double)
cudaError_t launch_fused_fast_f64(const FastKT<double>& F, const double* s[3], const double* a[3], double* o[3],
                                  cudaStream_t st);
cudaError_t launch_fused_ens(const FastK& F, const EnsLaunch& E, const float* s[3], const float* a[3], float* o[3],
                             cudaStream_t st);
cudaError_t launch_ens_moments(const int4* rinfo, int nrep, const float* s[3], double* out, cudaStream_t st);
void prof_begin();
int prof_end(int cap, char* names, double* ms, int* launches);
// Generic kernels: rb = bytes per real of the state arrays (4 or 8).
cudaError_t launch_fused(const FusedK& P, double dt_sys, int rb, cudaStream_t st);
cudaError_t launch_eval(const SysK& s, const TermsK& T, double dt_sys, void* const h[3], int acc, int rb,
                        cudaStream_t st);
cudaError_t launch_llg(const SysK& from, const void* const m[3], const void* const H[3], const void* const Ht[3],
                       const void* dsa, const void* dsg, double da, double dg, const LlgK& L,
                       void* const out[3], int rb, cudaStream_t st);
cudaError_t launch_advance_step(const DevStep* cur, DevStep* next, cudaStream_t st);
cudaError_t launch_partial_final(const double* part, int nb, int nq, double* out, cudaStream_t st);
// netMoment as one launch (partials, then the last block's fixed-order
// final sums into pinned host memory and out_dev); counter starts at 0.
// blocks of a netMoment read of n sites: a synchronous read, or one on a side stream
int netmoment_blocks(int n, bool side);
cudaError_t launch_netmoment_one(const void* x, const void* y, const void* z, int n, double m, double* part, int nb,
                                 unsigned* counter, double* out_host, double* out_dev, int rb, cudaStream_t st);
cudaError_t launch_netmoment(const void* x, const void* y, const void* z, int n, double m, double* part, int nb,
                             double* out, int rb, cudaStream_t st);
cudaError_t launch_dot(const void* const s[3], const void* const h[3], int n, double* part, int nb, double* out,
                       int rb, cudaStream_t st);
cudaError_t launch_diff(const void* const a[3], const void* const b[3], int n, double* part, int nb, double* out,
                        int rb, cudaStream_t st);
size_t conv_x_smem(const ConvK& c, int rb);
size_t conv_yz_smem(const ConvK& c, int rb);
cudaError_t conv_configure();
cudaError_t launch_conv(const ConvK& c, const FftLen& Lx, const FftLen& Ly, const FftLen& Lz, const void* tw,
                        const void* const s[3], void* spec, const void* ten6, const void* ten9, void* const h[3],
                        int rb, cudaStream_t st);
cudaError_t launch_tensor_lattice(int nx, int ny, int nz, const int gmax[4], const double ABC[9], int Px,
                                  int Py, int Pz, int zsign, double2* W, cudaStream_t st);
cudaError_t launch_tensor_rings(int nx, int ny, int nz, int nrings, int lstep, const double ABC[9], int Px, int Py,
                                int Pz, int zsign, double2* W, cudaStream_t st);
cudaError_t launch_tensor_extract_ref(int nx, int ny, int nz, int Px, int Py, int Pz, int zsign,
                                      const double2* W, double* out, cudaStream_t st);
cudaError_t launch_tensor_open(int nx, int ny, int nz, const double ABC[9], int Px, int Py, int Pz,
                               double2* W, cudaStream_t st);
// LongRange2D: x passes around the y transforms and the layer mixing
// (k_lr2d_ffty, k_lr2d_mix); the
// tensor spectrum Q[kx][ky][s][d][9] packed from FP64 transforms of the
// layer pairs p0 .. p0 + np - 1.
size_t lr2d_smem(const ConvK& c, int rb);
cudaError_t launch_lr2d(const ConvK& c, const FftLen L[3], const void* tw, const void* const s[3], void* spec,
                        const void* Q, const LR2DScale& sc, void* const h[3], int rb, cudaStream_t st);
cudaError_t launch_lr2d_pack(const double2* W, int nx, int ny, int nz, int p0, int np, void* Q, int rb,
                             cudaStream_t st);
cudaError_t launch_fft3d_d(double2* W, int ncomp, int Px, int Py, int Pz, const FftLen L[3],
                           const double2* tw, int sign, cudaStream_t st);
// Parity check of the FP64 transformed six-component tensor (out3: max |W|,
// largest ky- and kz-parity deviations, as double bits; zero them first)
// and the FP32 quarter tensor of the split passes (ConvK::quarter).
cudaError_t launch_tensor_symcheck(const double2* W, int Px, int Py, int Pz, int Kx, unsigned long long* out3,
                                   cudaStream_t st);
cudaError_t launch_tensor_pack6q(const double2* W, int Px, int Py, int Pz, int Kx, float* ten, int zmaj,
                                cudaStream_t st);
cudaError_t launch_tensor_pack6(const double2* W, int Px, int Py, int Pz, int Kx, void* ten6, double* maxim,
                                int rb, int kmaj, cudaStream_t st);
cudaError_t launch_tensor_pack9(const double2* W, int Px, int Py, int Pz, int Kx, void* ten9, int rb, int kmaj,
                                cudaStream_t st);
// Split (y,z) passes for planes larger than shared memory (c.split, c.spec2).
size_t split_smem(const ConvK& c, int rb);
cudaError_t launch_conv_split_yz(const ConvK& c, const FftLen& Ly, const FftLen& Lz, const void* tw, void* spec,
                                 const void* ten6, const void* ten9, int rb, cudaStream_t st);
// Learned surrogate (surrogate.cu).
size_t sur_out_smem(int CP, int rad);
// CTAs of the surrogate output kernel (one per 128 x-sites of a block of rows): its residual partials
int sur_out_ctas(int nx, int ny);
size_t sur_gw_smem(int C, int rad);
size_t sur_ydft_smem(const SurK& k);
cudaError_t sur_configure();
cudaError_t launch_sur_xdft(const SurK& k, const float* const a[3], const float* const b[3],
                            const __nv_bfloat16* F, float2* Xp, uint4* Xb, int* err, cudaStream_t st);
cudaError_t launch_sur_ydft(const SurK& k, const float2* Xp, const float2* twy, const float2* R, float2* Yh,
                            float2* Zh, unsigned int* cnt, cudaStream_t st);
cudaError_t launch_sur_zrows(const SurK& k, const float2* Zh, const float2* twy, uint8_t* Zb, cudaStream_t st);
// mode 0: out = h0 + ratio * dH (the surrogate's field; per-CTA residual
// sums to part); mode 1: out = dH.
cudaError_t launch_sur_out(const SurK& k, const uint4* Xb, const float* const h0[3], float* const out[3],
                           const uint8_t* Wc, const uint8_t* Fc, const uint8_t* Zb, SurDev* dev, double* part,
                           int* err, int mode, cudaStream_t st);
cudaError_t launch_sur_snapshot(SurDev* d, int n, const float* const m[3], const float* const h[3],
                                float* const sm[3], float* const sh[3], cudaStream_t st);
// End of a step: residual check of a surrogate step (np per-CTA sums), schedule
cudaError_t launch_sur_advance(SurDev* d, const double* part, int np, cudaStream_t st);
cudaError_t launch_sur_loss(int n, const float* const P[3], const float* const X[3], const float* const H0[3],
                            float* const G[3], double* part, int nb, double* out, cudaStream_t st);
cudaError_t launch_sur_grad_w(const SurK& k, const float* const a[3], const float* const b[3],
                              const float* const g[3], float* part, float* gw, cudaStream_t st);
cudaError_t launch_sur_grad_r(const SurK& k, const float2* Gh, const float2* Xh, float2* dR, cudaStream_t st);
cudaError_t launch_sur_adam(float* w, float* r, const float* gw, const float* gr, float* mw, float* vw, float* mr,
                            float* vr, uint8_t* wc, const double* sums, float lr, int step, int nw, int nr, int C,
                            int CP, cudaStream_t st);
} // namespace mlb
