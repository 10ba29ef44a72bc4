// ref_cuda_shim.cu -- TEST INFRASTRUCTURE ONLY (part of the oracle).
//
// C-ABI entry points over the reference's own FP64 CUDA kernels, which
// oracle/Makefile compiles unchanged from the reference tree together with
// this file into oracle/_ref/libref_cuda.so.  The reference declares them
// with C++ linkage (M/ = src/modules/):
//   cuda_llg_quat_apply    M/cuda/llg_cuda/llgquat.cu:283 (llgquat.hpp)
//   cuda_llg_cart_apply_N  M/cuda/llg_cuda/llgcartesian.cu:133 (llgcartesian.hpp)
//   cuda_anisotropy_N      M/cuda/anisotropy_cuda/spinoperationanisotropy.cu:50
//   cuda_thermal           M/cuda/thermal_cuda/spinoperationthermal.cu:77
// The prototypes below restate those declarations so that this file links
// against them; each wrapper launches on the legacy default stream (as the
// reference does), synchronises and returns the CUDA error code (0 = ok).
// Every pointer argument is a device pointer; the `_N` forms take device
// arrays of n device pointers, as the reference's batched calls do.
// Only tests/ load this library, to pin the oracle and the product against
// the reference's own arithmetic; nothing in the product links it.
#include <cuda_runtime.h>

void cuda_llg_quat_apply(const int nx, const int ny, const int nz, double* dsx, double* dsy, double* dsz, double* dms,
                         double* ssx, double* ssy, double* ssz, double* sms, double* ddx, double* ddy, double* ddz,
                         double* dds, double* htx, double* hty, double* htz, double* dhx, double* dhy, double* dhz,
                         double* ws1, double* ws2, double* ws3, double* ws4, const double dt, const double alpha,
                         const double* d_alpha, const double gamma, const double* d_gamma, int thermalOnlyFirstTerm);

void cuda_llg_cart_apply_N(int nx, int ny, int nz, double** dsx, double** dsy, double** dsz, double** dms,
                           double** ssx, double** ssy, double** ssz, double** sms, double** ddx, double** ddy,
                           double** ddz, double** dds, double** htx, double** hty, double** htz, double** dhx,
                           double** dhy, double** dhz, double* dt, double** d_alpha_N, double* d_alpha,
                           double** d_gamma_N, double* d_gamma, int thermalOnlyFirstTerm, int disableRenormalization,
                           const int n);

void cuda_anisotropy_N(const double global_scale, const double** d_sx_N, const double** d_sy_N,
                       const double** d_sz_N, const double* d_nx, const double* d_ny, const double* d_nz,
                       const double* d_k, double** d_hx_N, double** d_hy_N, double** d_hz_N, const int nxyz,
                       const int n);

void cuda_thermal(const float* d_rng6, const int i, double temperature, double* d_hx, double* d_hy, double* d_hz,
                  double* d_ms, double* d_scale, const int n, const double dt, const double alpha,
                  const double* d_alpha, const double gamma, const double* d_gamma);

static int finish()
{
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaGetLastError();
    return (int)e;
}

extern "C" {

// to = quaternion LLG step of `from` driven by dmdt's spins and fields
// (s: x, y, z, ms arrays; ht: the thermal slot or NULLs; h: the total
// field); ws: four scratch arrays of nxyz doubles.
int ref_llg_quat_apply(int nx, int ny, int nz, double* const to[4], double* const from[4], double* const dmdt[4],
                       double* const ht[3], double* const h[3], double* const ws[4], double dt, double alpha,
                       const double* site_alpha, double gamma, const double* site_gamma, int thermal_only_first_term)
{
    cuda_llg_quat_apply(nx, ny, nz, to[0], to[1], to[2], to[3], from[0], from[1], from[2], from[3], dmdt[0], dmdt[1],
                        dmdt[2], dmdt[3], ht[0], ht[1], ht[2], h[0], h[1], h[2], ws[0], ws[1], ws[2], ws[3], dt,
                        alpha, site_alpha, gamma, site_gamma, thermal_only_first_term);
    return finish();
}

// Batched Cartesian LLG: each argument p[k] is a device array of n device
// pointers (replica j's array at index j); dt, alpha, gamma are device
// arrays of n doubles; alpha_n / gamma_n device arrays of n pointers
// (NULL entries: the replica's uniform value).
int ref_llg_cart_apply_n(int nx, int ny, int nz, double** const to[4], double** const from[4],
                         double** const dmdt[4], double** const ht[3], double** const h[3], double* dt,
                         double** alpha_n, double* alpha, double** gamma_n, double* gamma,
                         int thermal_only_first_term, int disable_renormalization, int n)
{
    cuda_llg_cart_apply_N(nx, ny, nz, to[0], to[1], to[2], to[3], from[0], from[1], from[2], from[3], dmdt[0],
                          dmdt[1], dmdt[2], dmdt[3], ht[0], ht[1], ht[2], h[0], h[1], h[2], dt, alpha_n, alpha,
                          gamma_n, gamma, thermal_only_first_term, disable_renormalization, n);
    return finish();
}

// Anisotropy field of n replicas (device arrays of n pointers) from per-site
// axis components and strengths (nxyz each).
int ref_anisotropy_n(double global_scale, const double** sx, const double** sy, const double** sz, const double* ax,
                     const double* ay, const double* az, const double* k, double** hx, double** hy, double** hz,
                     int nxyz, int n)
{
    cuda_anisotropy_N(global_scale, sx, sy, sz, ax, ay, az, k, hx, hy, hz, nxyz, n);
    return finish();
}

// Thermal field from six FP32 normals per site (half = 0: the first three,
// 1: the second three).
int ref_thermal(const float* rng6, int half, double temperature, double* hx, double* hy, double* hz, double* ms,
                double* scale, int nxyz, double dt, double alpha, const double* site_alpha, double gamma,
                const double* site_gamma)
{
    cuda_thermal(rng6, half, temperature, hx, hy, hz, ms, scale, nxyz, dt, alpha, site_alpha, gamma, site_gamma);
    return finish();
}

} // extern "C"
