// ewald.cu -- DipoleEwald3D (M/cpu/ewald3d/ewald3d.cpp): the dipolar
// interaction tensor of a periodic lattice by Ewald summation in FP64, the
// tensor source of LongRange3D (make_tensor.lua).
//
// Geometry (ewald3d.cpp:76-104): supercell vectors u_i = d_i a_i, volume
// vu = |u1 . (u2 x u3)|, reciprocal vectors b_i = 2 pi (u_j x u_k) / vu.
// Element G_ab(r) (ewald3d.cpp:221-358): the sum over the (2N+1)^3 integer
// triples (n, m, k) of a real-space term at r + n u1 + m u2 + k u3 and a
// reciprocal-space term at Q = n b1 + m b2 + k b3, with the r = 0 forms of
// both (no self term), real and reciprocal parts accumulated separately in
// the order n, m, k.  The real/reciprocal split eta is the golden-section
// minimum of |the N -> N + 1 shell of G_xx(a1)| (ewald3d.cpp:109-218), found
// on the host once per geometry.
//
// The per-element sum runs on the host for single elements and on the GPU,
// one warp per lattice site and all nine components at once, for whole
// lattices (the loop of make_tensor.lua).
#include "../../include/mlb200.h"

#include <cuda_runtime.h>
#include <math.h>

#include <algorithm>
#include <new>
#include <string>
#include <vector>

namespace mlb {
void set_last_error(const std::string& msg);
}

namespace {

struct EwaldGeo {
    double u[3][3];   // supercell vectors
    double b[3][3];   // reciprocal vectors
    double vu;        // supercell volume
};

__host__ __device__ inline double ew_dot(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// One (n, m, k) term: real_part and recip_part of G_ab at r (ewald3d.cpp:
// 221-328).
__host__ __device__ inline void ew_term(const EwaldGeo& g, int alpha, int beta, const double* r, double eta, int n,
                                        int m, int k, double& real_part, double& recip_part)
{
    const double eta2 = eta * eta;
    const double delta = alpha == beta ? 1.0 : 0.0;
    double Q[3], R[3];
    for (int i = 0; i < 3; i++) Q[i] = n * g.b[0][i] + m * g.b[1][i] + k * g.b[2][i];
    const bool r0 = ew_dot(r, r) == 0;
    if (r0) {
        for (int i = 0; i < 3; i++) R[i] = n * g.u[0][i] + m * g.u[1][i] + k * g.u[2][i];
    } else {
        for (int i = 0; i < 3; i++) R[i] = n * g.u[0][i] + m * g.u[1][i] + k * g.u[2][i] + r[i];
    }
    const double Q2 = ew_dot(Q, Q);
    const double Q1 = sqrt(Q2);
    if (Q1 > 0) {
        if (r0)
            recip_part = -4.0 * M_PI * exp(-Q2 / (4.0 * eta2)) * (Q2 * delta - 3 * Q[alpha] * Q[beta]) / (3.0 * g.vu * Q2);
        else
            recip_part = 4.0 * M_PI * Q[alpha] * Q[beta] * cos(ew_dot(r, Q)) * exp(-Q2 / (4.0 * eta2)) / (Q2 * g.vu);
    } else {
        recip_part = 0;
    }
    const double Rab = R[alpha] * R[beta];
    const double R2 = ew_dot(R, R);
    const double R1 = sqrt(R2);
    const double R4 = R2 * R2;
    const double R5 = R4 * R1;
    const double sqrtpi = 1.772453850905516027;
    if (R1 > 0) {
        if (r0)
            real_part = (R2 * delta - 3.0 * R[alpha] * R[beta]) *
                        (2.0 * eta * exp(-R2 * eta2) * (3.0 + 2.0 * R2 * eta2) / (3.0 * R4 * sqrtpi) + erfc(R1 * eta) / R5);
        else
            real_part = 2.0 * eta * exp(-eta2 * R2) * (R2 * delta - 3.0 * Rab - 2.0 * eta2 * Rab * R2) / (sqrtpi * R4) +
                        (R2 * delta - 3.0 * Rab) * erfc(eta * R1) / R5;
    } else {
        real_part = 0;
    }
}

__host__ __device__ inline double ew_element(const EwaldGeo& g, int alpha, int beta, const double* r, double eta,
                                             int N)
{
    double tq = 0, tr = 0, pr, pq;
    for (int n = -N; n <= N; n++)
        for (int m = -N; m <= N; m++)
            for (int k = -N; k <= N; k++) {
                ew_term(g, alpha, beta, r, eta, n, m, k, pr, pq);
                tr += pr;
                tq += pq;
            }
    return tq + tr;
}

// G(N + 1) - G(N) by its surface shell (ewald3d.cpp:361-422).
double ew_next_shell(const EwaldGeo& g, int alpha, int beta, const double* r, double eta, int N)
{
    double tq = 0, tr = 0, r1, q1, r2, q2;
    const int M = N + 1;
    for (int n = -M; n <= M; n++)
        for (int m = -M; m <= M; m++) {
            ew_term(g, alpha, beta, r, eta, n, m, M, r1, q1);
            ew_term(g, alpha, beta, r, eta, n, m, -M, r2, q2);
            tr += r1; tq += q1; tr += r2; tq += q2;
        }
    for (int n = -M; n <= M; n++)
        for (int k = -N; k <= N; k++) {
            ew_term(g, alpha, beta, r, eta, n, M, k, r1, q1);
            ew_term(g, alpha, beta, r, eta, n, -M, k, r2, q2);
            tr += r1; tq += q1; tr += r2; tq += q2;
        }
    for (int m = -N; m <= N; m++)
        for (int k = -N; k <= N; k++) {
            ew_term(g, alpha, beta, r, eta, M, m, k, r1, q1);
            ew_term(g, alpha, beta, r, eta, -M, m, k, r2, q2);
            tr += r1; tq += q1; tr += r2; tq += q2;
        }
    return tq + tr;
}

// The whole lattice: one warp per site r.  A term's exponentials, erfc and
// cosine do not depend on the component, so each lane evaluates them once
// per (n, m, k) for all nine components; the 32 lanes take every 32nd
// triple and the real and reciprocal partial sums meet in a shuffle tree.
// The result equals the per-element sum up to rounding (the order of the
// additions and the component factors taken as products with reciprocals):
// G_ab and G_ba come out equal here.
constexpr int EW_SITES_PER_CTA = 8;

__global__ void __launch_bounds__(32 * EW_SITES_PER_CTA)
k_ewald_tensor(EwaldGeo g, double a1x, double a1y, double a1z, double a2x, double a2y, double a2z, double a3x,
               double a3y, double a3z, double eta, int N, int nx, int ny, int nz, double* out)
{
    const long long n = (long long)nx * ny * nz;
    const long long i = (long long)blockIdx.x * EW_SITES_PER_CTA + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= n) return;   // whole warps leave together
    const int x = (int)(i % nx), y = (int)((i / nx) % ny), z = (int)(i / ((long long)nx * ny));
    const double r[3] = {x * a1x + y * a2x + z * a3x, x * a1y + y * a2y + z * a3y, x * a1z + y * a2z + z * a3z};
    const bool r0 = ew_dot(r, r) == 0;
    const double eta2 = eta * eta;
    const double sqrtpi = 1.772453850905516027;
    const double inv4eta2 = 1.0 / (4.0 * eta2);
    // six independent components xx, xy, xz, yy, yz, zz
    double tr[6] = {0, 0, 0, 0, 0, 0}, tq[6] = {0, 0, 0, 0, 0, 0};
    const int S = 2 * N + 1;
    const int terms = S * S * S;
    for (int t = lane; t < terms; t += 32) {
        const int nn = t / (S * S) - N, mm = (t / S) % S - N, kk = t % S - N;
        double Q[3], R[3];
        for (int c = 0; c < 3; c++) Q[c] = nn * g.b[0][c] + mm * g.b[1][c] + kk * g.b[2][c];
        for (int c = 0; c < 3; c++) R[c] = nn * g.u[0][c] + mm * g.u[1][c] + kk * g.u[2][c] + (r0 ? 0.0 : r[c]);
        const double Q2 = ew_dot(Q, Q);
        if (Q2 > 0) {
            const double ex = exp(-Q2 * inv4eta2);
            if (r0) {
                // -4 pi e (Q2 delta - 3 Qa Qb) / (3 vu Q2)
                const double f = -4.0 * M_PI * ex / (3.0 * g.vu * Q2);
                tq[0] += f * (Q2 - 3 * Q[0] * Q[0]);
                tq[1] += f * (-3 * Q[0] * Q[1]);
                tq[2] += f * (-3 * Q[0] * Q[2]);
                tq[3] += f * (Q2 - 3 * Q[1] * Q[1]);
                tq[4] += f * (-3 * Q[1] * Q[2]);
                tq[5] += f * (Q2 - 3 * Q[2] * Q[2]);
            } else {
                // 4 pi Qa Qb cos(r.Q) e / (Q2 vu)
                const double f = 4.0 * M_PI * cos(ew_dot(r, Q)) * ex / (Q2 * g.vu);
                tq[0] += f * Q[0] * Q[0];
                tq[1] += f * Q[0] * Q[1];
                tq[2] += f * Q[0] * Q[2];
                tq[3] += f * Q[1] * Q[1];
                tq[4] += f * Q[1] * Q[2];
                tq[5] += f * Q[2] * Q[2];
            }
        }
        const double R2 = ew_dot(R, R);
        if (R2 > 0) {
            const double R1 = sqrt(R2);
            const double R4 = R2 * R2;
            const double R5 = R4 * R1;
            const double ex = exp(-eta2 * R2);
            const double ec = erfc(eta * R1) / R5;
            if (r0) {
                // (R2 delta - 3 Ra Rb) (2 eta e (3 + 2 R2 eta2) / (3 R4 sqrt(pi)) + erfc / R5)
                const double f = 2.0 * eta * ex * (3.0 + 2.0 * R2 * eta2) / (3.0 * R4 * sqrtpi) + ec;
                tr[0] += (R2 - 3.0 * R[0] * R[0]) * f;
                tr[1] += (-3.0 * R[0] * R[1]) * f;
                tr[2] += (-3.0 * R[0] * R[2]) * f;
                tr[3] += (R2 - 3.0 * R[1] * R[1]) * f;
                tr[4] += (-3.0 * R[1] * R[2]) * f;
                tr[5] += (R2 - 3.0 * R[2] * R[2]) * f;
            } else {
                // 2 eta e (R2 delta - 3 Rab - 2 eta2 Rab R2) / (sqrt(pi) R4) + (R2 delta - 3 Rab) erfc / R5
                const double A = 2.0 * eta * ex / (sqrtpi * R4);
                const double w = 3.0 + 2.0 * eta2 * R2;
                const double Rab[6] = {R[0] * R[0], R[0] * R[1], R[0] * R[2], R[1] * R[1], R[1] * R[2], R[2] * R[2]};
                const double dl[6] = {R2, 0.0, 0.0, R2, 0.0, R2};
#pragma unroll
                for (int q = 0; q < 6; q++) tr[q] += A * (dl[q] - w * Rab[q]) + (dl[q] - 3.0 * Rab[q]) * ec;
            }
        }
    }
#pragma unroll
    for (int q = 0; q < 6; q++) {
        double a = tr[q], b = tq[q];
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, o);
            b += __shfl_xor_sync(0xffffffffu, b, o);
        }
        tr[q] = a;
        tq[q] = b;
    }
    if (lane == 0) {
        double G[6];
#pragma unroll
        for (int q = 0; q < 6; q++) G[q] = tq[q] + tr[q];
        out[0 * n + i] = G[0];   // xx
        out[1 * n + i] = G[1];   // xy
        out[2 * n + i] = G[2];   // xz
        out[3 * n + i] = G[1];   // yx
        out[4 * n + i] = G[3];   // yy
        out[5 * n + i] = G[4];   // yz
        out[6 * n + i] = G[2];   // zx
        out[7 * n + i] = G[4];   // zy
        out[8 * n + i] = G[5];   // zz
    }
}

} // namespace

struct mlb_ewald3d {
    int d[3] = {1, 1, 1};
    double a[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    int nsites = 10;
    double tau = 1e-3;
    double eta = 0.5;
    bool good_eta = false;
    EwaldGeo g{};
};

namespace {

struct EwErr {
    int code;
    std::string msg;
};

template <class F>
int ew_guard(F&& f)
{
    try {
        f();
        return MLB_OK;
    } catch (EwErr& e) {
        mlb::set_last_error(e.msg);
        return e.code;
    } catch (std::bad_alloc&) {
        mlb::set_last_error("host allocation failed");
        return MLB_ENOMEM;
    }
}

void ew_support(mlb_ewald3d* e)
{
    EwaldGeo& g = e->g;
    for (int i = 0; i < 3; i++)
        for (int c = 0; c < 3; c++) g.u[i][c] = e->d[i] * e->a[i][c];
    auto cross = [](double* o, const double* p, const double* q) {
        o[0] = p[1] * q[2] - p[2] * q[1];
        o[1] = p[2] * q[0] - p[0] * q[2];
        o[2] = p[0] * q[1] - p[1] * q[0];
    };
    double c23[3], c31[3], c12[3];
    cross(c23, g.u[1], g.u[2]);
    cross(c31, g.u[2], g.u[0]);
    cross(c12, g.u[0], g.u[1]);
    g.vu = fabs(ew_dot(g.u[0], c23));
    for (int c = 0; c < 3; c++) {
        g.b[0][c] = 2.0 * M_PI * c23[c] / g.vu;
        g.b[1][c] = 2.0 * M_PI * c31[c] / g.vu;
        g.b[2][c] = 2.0 * M_PI * c12[c] / g.vu;
    }
    e->good_eta = false;
}

// Golden-section search of ewald3d.cpp:109-218 (recursion depth 100),
// minimising |ew_next_shell(G_xx, r3, x, N)| over x.
const double kRgr = 0.3819660112501051518;
const double kMinA = 1e-10;

bool ew_search(mlb_ewald3d* e, int depth, const double* r3, double a, double fa, double b, double fb, double c,
               double fc, int N, double tol)
{
    auto F = [&](double x) { return fabs(ew_next_shell(e->g, 0, 0, r3, x, N)); };
    auto done = [&](double x) { return (c - a) < tol * (fabs(b) + fabs(x)); };
    if (depth < 0) return false;
    if (a > kMinA && fa < fb && fb < fc) {
        const double x = c + kRgr * (c - b);
        return ew_search(e, depth - 1, r3, b, fb, c, fc, x, F(x), N, tol);
    }
    if (fa > fb && fb > fc) {
        const double x = a - kRgr * (b - a);
        return ew_search(e, depth - 1, r3, x, F(x), a, fa, b, fb, N, tol);
    }
    if ((c - b) > (b - a)) {
        const double x = b + kRgr * (c - b);
        if (done(x)) { e->eta = (c + a) * 0.5; return true; }
        const double fx = F(x);
        if (fx < fb) return ew_search(e, depth - 1, r3, b, fb, x, fx, c, fc, N, tol);
        return ew_search(e, depth - 1, r3, a, fa, b, fb, x, fx, N, tol);
    }
    const double x = b - kRgr * (b - a);
    if (done(x)) { e->eta = (c + a) * 0.5; return true; }
    const double fx = F(x);
    if (fx < fb) return ew_search(e, depth - 1, r3, a, fa, x, fx, b, fb, N, tol);
    return ew_search(e, depth - 1, r3, x, fx, b, fb, c, fc, N, tol);
}

// findEta as calcTensorElement calls it (ewald3d.cpp:30, 48): at r = a1,
// with the object's tau passed where the shell count goes (so the shell
// count is the integer part of tau) and the default tolerance 1e-3.
void ew_need_eta(mlb_ewald3d* e)
{
    if (e->good_eta) return;
    const int N = (int)e->tau;
    const double tol = 1e-3;
    const double a = kMinA, c = 1000, b = a + kRgr * (c - a);
    const double* r3 = e->a[0];
    const double fa = fabs(ew_next_shell(e->g, 0, 0, r3, a, N));
    const double fb = fabs(ew_next_shell(e->g, 0, 0, r3, b, N));
    const double fc = fabs(ew_next_shell(e->g, 0, 0, r3, c, N));
    if (!ew_search(e, 100, r3, a, fa, b, fb, c, fc, N, tol)) {
        char msg[256];
        snprintf(msg, sizeof(msg),
                 "Failed to calculate real/reciprocal partition point (eta) for series limits. Try a different tau "
                 "value for a tolerance (current tau = %f)",
                 e->tau);
        throw EwErr{MLB_ESTATE, msg};
    }
    e->good_eta = true;
}

void ew_check_ab(int ab)
{
    if (ab < 0 || ab > 8)
        throw EwErr{MLB_EINVAL, "first argument of calculateTensorElement must be AB pair: `XX', `XY', ... `ZZ'"};
}

} // namespace

extern "C" {

int mlb_ewald3d_create(int nx, int ny, int nz, mlb_ewald3d** out)
{
    return ew_guard([&] {
        if (!out) throw EwErr{MLB_EINVAL, "null argument"};
        mlb_ewald3d* e = new mlb_ewald3d();
        e->d[0] = nx > 0 ? nx : 1;
        e->d[1] = ny > 0 ? ny : 1;
        e->d[2] = nz > 0 ? nz : 1;
        ew_support(e);
        *out = e;
    });
}

int mlb_ewald3d_destroy(mlb_ewald3d* e)
{
    delete e;
    return MLB_OK;
}

int mlb_ewald3d_set_unit_cell(mlb_ewald3d* e, const double a[3], const double b[3], const double c[3])
{
    return ew_guard([&] {
        if (!e || !a || !b || !c) throw EwErr{MLB_EINVAL, "null argument"};
        const double* v[3] = {a, b, c};
        for (int i = 0; i < 3; i++)
            for (int k = 0; k < 3; k++) e->a[i][k] = v[i][k];
        ew_support(e);
    });
}

int mlb_ewald3d_get_unit_cell(const mlb_ewald3d* e, double abc[9])
{
    if (!e || !abc) return MLB_EINVAL;
    for (int i = 0; i < 3; i++)
        for (int k = 0; k < 3; k++) abc[3 * i + k] = e->a[i][k];
    return MLB_OK;
}

int mlb_ewald3d_set_lattice_size(mlb_ewald3d* e, int nx, int ny, int nz)
{
    return ew_guard([&] {
        if (!e) throw EwErr{MLB_EINVAL, "null argument"};
        e->d[0] = nx > 0 ? nx : 1;
        e->d[1] = ny > 0 ? ny : 1;
        e->d[2] = nz > 0 ? nz : 1;
        ew_support(e);
    });
}

int mlb_ewald3d_get_lattice_size(const mlb_ewald3d* e, int n3[3])
{
    if (!e || !n3) return MLB_EINVAL;
    for (int i = 0; i < 3; i++) n3[i] = e->d[i];
    return MLB_OK;
}

int mlb_ewald3d_set_tau(mlb_ewald3d* e, double tau)
{
    if (!e) return MLB_EINVAL;
    if (tau > 0) { e->tau = tau; e->good_eta = false; }
    return MLB_OK;
}

int mlb_ewald3d_get_tau(const mlb_ewald3d* e, double* tau)
{
    if (!e || !tau) return MLB_EINVAL;
    *tau = e->tau;
    return MLB_OK;
}

int mlb_ewald3d_set_nsites(mlb_ewald3d* e, int n)
{
    if (!e) return MLB_EINVAL;
    if (n > 1) { e->nsites = n; e->good_eta = false; }
    return MLB_OK;
}

int mlb_ewald3d_get_nsites(const mlb_ewald3d* e, int* n)
{
    if (!e || !n) return MLB_EINVAL;
    *n = e->nsites;
    return MLB_OK;
}

int mlb_ewald3d_get_eta(const mlb_ewald3d* e, double* eta)
{
    if (!e || !eta) return MLB_EINVAL;
    *eta = e->eta;
    return MLB_OK;
}

int mlb_ewald3d_get_volume(const mlb_ewald3d* e, double* v)
{
    if (!e || !v) return MLB_EINVAL;
    *v = e->g.vu;
    return MLB_OK;
}

int mlb_ewald3d_element(mlb_ewald3d* e, int ab, const int r3[3], double* out)
{
    return ew_guard([&] {
        if (!e || !r3 || !out) throw EwErr{MLB_EINVAL, "null argument"};
        ew_check_ab(ab);
        ew_need_eta(e);
        double r[3];
        for (int i = 0; i < 3; i++) r[i] = r3[0] * e->a[0][i] + r3[1] * e->a[1][i] + r3[2] * e->a[2][i];
        *out = ew_element(e->g, ab / 3, ab % 3, r, e->eta, e->nsites);
    });
}

int mlb_ewald3d_element_real(mlb_ewald3d* e, int ab, const double r[3], double* out)
{
    return ew_guard([&] {
        if (!e || !r || !out) throw EwErr{MLB_EINVAL, "null argument"};
        ew_check_ab(ab);
        ew_need_eta(e);
        *out = ew_element(e->g, ab / 3, ab % 3, r, e->eta, e->nsites);
    });
}

int mlb_ewald3d_tensor(mlb_ewald3d* e, double* out9)
{
    return ew_guard([&] {
        if (!e || !out9) throw EwErr{MLB_EINVAL, "null argument"};
        ew_need_eta(e);
        const long long n = (long long)e->d[0] * e->d[1] * e->d[2];
        double* dev = nullptr;
        cudaError_t rc = cudaMalloc(&dev, sizeof(double) * 9 * n);
        if (rc != cudaSuccess) throw EwErr{MLB_ENOMEM, std::string("Ewald tensor: ") + cudaGetErrorString(rc)};
        const long long nb = (n + EW_SITES_PER_CTA - 1) / EW_SITES_PER_CTA;
        k_ewald_tensor<<<(unsigned)nb, 32 * EW_SITES_PER_CTA>>>(e->g, e->a[0][0], e->a[0][1], e->a[0][2], e->a[1][0], e->a[1][1], e->a[1][2],
                                    e->a[2][0], e->a[2][1], e->a[2][2], e->eta, e->nsites, e->d[0], e->d[1], e->d[2],
                                    dev);
        rc = cudaGetLastError();
        if (rc == cudaSuccess) rc = cudaMemcpy(out9, dev, sizeof(double) * 9 * n, cudaMemcpyDeviceToHost);
        cudaFree(dev);
        if (rc != cudaSuccess) throw EwErr{MLB_ECUDA, std::string("Ewald tensor: ") + cudaGetErrorString(rc)};
    });
}

} // extern "C"
