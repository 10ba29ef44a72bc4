/*
 * oracle.c -- FP64 CPU restatement of MagLua's spin-dynamics step.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product; see oracle.h).
 * Paths are relative to the reference project; M/ = src/modules/.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <strings.h>

/* ------------------------------------------------------------------ */
/* SpinSystem                                                           */
/* ------------------------------------------------------------------ */

/* SpinSystem constructor + init: M/cpu/core/spinsystem.cpp:29-41, 502-566. */
orc_ss* orc_ss_new(int nx, int ny, int nz)
{
    orc_ss* ss = (orc_ss*)calloc(1, sizeof(orc_ss));
    ss->nx = nx; ss->ny = ny; ss->nz = nz; ss->n = nx * ny * nz;
    ss->x = (double*)calloc(ss->n, sizeof(double));
    ss->y = (double*)calloc(ss->n, sizeof(double));
    ss->z = (double*)calloc(ss->n, sizeof(double));
    ss->ms = (double*)calloc(ss->n, sizeof(double));
    ss->alpha = 1.0; ss->gamma = 1.0; ss->dt = 1.0; ss->time = 0.0;
    orc_ss_slot(ss, "Total"); /* slot 0, spinsystem.cpp:565 */
    return ss;
}

void orc_ss_free(orc_ss* ss)
{
    if (!ss) return;
    free(ss->x); free(ss->y); free(ss->z); free(ss->ms);
    free(ss->site_alpha); free(ss->site_gamma);
    for (int i = 0; i < ss->nslots; i++) { free(ss->hx[i]); free(ss->hy[i]); free(ss->hz[i]); }
    free(ss);
}

void orc_ss_copy(orc_ss* d, const orc_ss* s)
{
    memcpy(d->x, s->x, sizeof(double) * s->n);
    memcpy(d->y, s->y, sizeof(double) * s->n);
    memcpy(d->z, s->z, sizeof(double) * s->n);
    memcpy(d->ms, s->ms, sizeof(double) * s->n);
    d->alpha = s->alpha; d->gamma = s->gamma; d->dt = s->dt; d->time = s->time;
}

/* getSlot: case-insensitive name lookup, spinsystem.cpp:889-905. */
int orc_ss_find_slot(const orc_ss* ss, const char* name)
{
    for (int i = 0; i < ss->nslots; i++)
        if (strcasecmp(ss->names[i], name) == 0) return i;
    return -1;
}

/* register_slot_name + ensureSlotExists (zeroed arrays), spinsystem.cpp:603-667. */
int orc_ss_slot(orc_ss* ss, const char* name)
{
    int s = orc_ss_find_slot(ss, name);
    if (s >= 0) return s;
    if (ss->nslots >= ORC_MAX_SLOTS) return -1;
    s = ss->nslots++;
    strncpy(ss->names[s], name, ORC_SLOT_NAME - 1);
    ss->hx[s] = (double*)calloc(ss->n, sizeof(double));
    ss->hy[s] = (double*)calloc(ss->n, sizeof(double));
    ss->hz[s] = (double*)calloc(ss->n, sizeof(double));
    ss->used[s] = 0;
    return s;
}

double* orc_ss_field(orc_ss* ss, const char* name, int comp)
{
    int s = orc_ss_slot(ss, name);
    if (s < 0) return NULL;
    return comp == 0 ? ss->hx[s] : (comp == 1 ? ss->hy[s] : ss->hz[s]);
}

/* SpinSystem::set(i, sx, sy, sz): the length becomes |s|, spinsystem.cpp:1090-1098. */
void orc_ss_set_spin(orc_ss* ss, int i, double sx, double sy, double sz)
{
    ss->x[i] = sx; ss->y[i] = sy; ss->z[i] = sz;
    ss->ms[i] = sqrt(sx * sx + sy * sy + sz * sz);
}

static void set_site(double** dst, const double* src, int n)
{
    free(*dst); *dst = NULL;
    if (src) { *dst = (double*)malloc(sizeof(double) * n); memcpy(*dst, src, sizeof(double) * n); }
}
void orc_ss_set_site_alpha(orc_ss* ss, const double* a) { set_site(&ss->site_alpha, a, ss->n); }
void orc_ss_set_site_gamma(orc_ss* ss, const double* g) { set_site(&ss->site_gamma, g, ss->n); }

/* zeroFields: zero every slot and mark it unused, spinsystem.cpp:968-980. */
void orc_ss_reset_fields(orc_ss* ss)
{
    for (int s = 0; s < ss->nslots; s++) {
        ss->used[s] = 0;
        memset(ss->hx[s], 0, sizeof(double) * ss->n);
        memset(ss->hy[s], 0, sizeof(double) * ss->n);
        memset(ss->hz[s], 0, sizeof(double) * ss->n);
    }
}

/* sumFields: Total = sum over used slots != Total in slot order, each as
 * Total = 1*Total + 1*slot (pairwiseScaleAdd), spinsystem.cpp:853-871. */
void orc_ss_sum_fields(orc_ss* ss)
{
    const int T = orc_ss_slot(ss, "Total");
    double* H[3] = {ss->hx[T], ss->hy[T], ss->hz[T]};
    for (int c = 0; c < 3; c++) {
        memset(H[c], 0, sizeof(double) * ss->n);
        for (int s = 1; s < ss->nslots; s++) {
            if (s == T || !ss->used[s]) continue;
            const double* src = c == 0 ? ss->hx[s] : (c == 1 ? ss->hy[s] : ss->hz[s]);
            for (int i = 0; i < ss->n; i++) H[c][i] = 1.0 * H[c][i] + 1.0 * src[i];
        }
    }
}

/* Lua sumFieldsCustom: dest = sum_k w_k * src_k over used sources,
 * M/cpu/core/spinsystem_luafuncs.lua:298-323 (pairwiseScaleAdd(factor, src, dest)). */
void orc_ss_sum_fields_weighted(orc_ss* ss, const char* dest, int nsrc,
                                const char* const* src, const double* w)
{
    const int D = orc_ss_slot(ss, dest);
    memset(ss->hx[D], 0, sizeof(double) * ss->n);
    memset(ss->hy[D], 0, sizeof(double) * ss->n);
    memset(ss->hz[D], 0, sizeof(double) * ss->n);
    for (int k = 0; k < nsrc; k++) {
        int s = orc_ss_find_slot(ss, src[k]);
        if (s < 0 || !ss->used[s]) continue;
        for (int i = 0; i < ss->n; i++) {
            ss->hx[D][i] = w[k] * ss->hx[s][i] + ss->hx[D][i];
            ss->hy[D][i] = w[k] * ss->hy[s][i] + ss->hy[D][i];
            ss->hz[D][i] = w[k] * ss->hz[s][i] + ss->hz[D][i];
        }
    }
}

/* netMoment (Lua), spinsystem_luafuncs.lua:17-54: per component sum(v*m),
 * sum((v*m)^2), then the two vector lengths. */
void orc_ss_netmoment(const orc_ss* ss, double m, double out[8])
{
    const double* v[3] = {ss->x, ss->y, ss->z};
    for (int c = 0; c < 3; c++) {
        double s1 = 0, s2 = 0;
        for (int i = 0; i < ss->n; i++) { double a = v[c][i] * m; s1 += a; s2 += a * a; }
        out[c] = s1; out[c + 4] = s2;
    }
    out[3] = sqrt(out[0] * out[0] + out[1] * out[1] + out[2] * out[2]);
    out[7] = sqrt(out[4] * out[4] + out[5] * out[5] + out[6] * out[6]);
}

/* ------------------------------------------------------------------ */
/* Mersenne Twister (64-bit unsigned long storage, 32-bit masked values) */
/* ------------------------------------------------------------------ */
#define MT_N 624
#define MT_M 397
static unsigned long long mt_twist(unsigned long long m, unsigned long long s0, unsigned long long s1)
{
    /* twist = m ^ (mixBits(s0,s1) >> 1) ^ magic(s1), mersennetwister.h:141-150 */
    unsigned long long mix = (s0 & 0x80000000ULL) | (s1 & 0x7fffffffULL);
    return m ^ (mix >> 1) ^ ((s1 & 1ULL) ? 0x9908b0dfULL : 0ULL);
}

/* initialize, mersennetwister.h:177-190 */
static void mt_initialize(orc_mt* mt, unsigned long long seed)
{
    mt->state[0] = seed & 0xffffffffULL;
    for (int i = 1; i < MT_N; i++)
        mt->state[i] = (1812433253ULL * (mt->state[i - 1] ^ (mt->state[i - 1] >> 30)) + (unsigned long long)i) & 0xffffffffULL;
}

/* reload, mersennetwister.h:192-205 */
static void mt_reload(orc_mt* mt)
{
    unsigned long long* s = mt->state;
    int i = 0;
    for (; i < MT_N - MT_M; i++) s[i] = mt_twist(s[i + MT_M], s[i], s[i + 1]);
    for (; i < MT_N - 1; i++) s[i] = mt_twist(s[i + MT_M - MT_N], s[i], s[i + 1]);
    s[MT_N - 1] = mt_twist(s[MT_M - 1], s[MT_N - 1], s[0]);
    mt->left = MT_N; mt->pnext = 0;
}

/* seed(oneSeed) = initialize + reload, mersennetwister.h:207-212 */
void orc_mt_seed(orc_mt* mt, unsigned long long seed) { mt_initialize(mt, seed); mt_reload(mt); }

/* seed(bigSeed, len), mersennetwister.h:214-245 (used only for the
 * published init_by_array known-answer test). */
void orc_mt_seed_array(orc_mt* mt, const unsigned long long* key, int len)
{
    mt_initialize(mt, 19650218ULL);
    unsigned long long* s = mt->state;
    int i = 1, j = 0;
    int k = MT_N > len ? MT_N : len;
    for (; k; --k) {
        s[i] = s[i] ^ ((s[i - 1] ^ (s[i - 1] >> 30)) * 1664525ULL);
        s[i] += (key[j] & 0xffffffffULL) + (unsigned long long)j;
        s[i] &= 0xffffffffULL;
        ++i; ++j;
        if (i >= MT_N) { s[0] = s[MT_N - 1]; i = 1; }
        if (j >= len) j = 0;
    }
    for (k = MT_N - 1; k; --k) {
        s[i] = s[i] ^ ((s[i - 1] ^ (s[i - 1] >> 30)) * 1566083941ULL);
        s[i] -= (unsigned long long)i;
        s[i] &= 0xffffffffULL;
        ++i;
        if (i >= MT_N) { s[0] = s[MT_N - 1]; i = 1; }
    }
    s[0] = 0x80000000ULL;
    mt_reload(mt);
}

/* randInt with tempering, mersennetwister.h:281-294 */
unsigned long long orc_mt_randint(orc_mt* mt)
{
    if (mt->left == 0) mt_reload(mt);
    --mt->left;
    unsigned long long s1 = mt->state[mt->pnext++];
    s1 ^= (s1 >> 11);
    s1 ^= (s1 << 7) & 0x9d2c5680ULL;
    s1 ^= (s1 << 15) & 0xefc60000ULL;
    return s1 ^ (s1 >> 18);
}

/* rand(): [0,1], mersennetwister.h:317-318 */
double orc_mt_rand(orc_mt* mt) { return (double)orc_mt_randint(mt) * (1.0 / 4294967295.0); }

/* MTRand::randNorm overrides RNG::randNorm: polar Box-Muller that keeps
 * only x*s of each accepted pair, mersennetwister.h:340-352. */
double orc_mt_randnorm(orc_mt* mt, double mean, double stddev)
{
    double x, y, r;
    do {
        x = 2.0 * orc_mt_rand(mt) - 1.0;
        y = 2.0 * orc_mt_rand(mt) - 1.0;
        r = x * x + y * y;
    } while (r >= 1.0 || r == 0.0);
    double s = sqrt(-2.0 * log(r) / r);
    return mean + x * s * stddev;
}

/* ------------------------------------------------------------------ */
/* Field operators                                                      */
/* ------------------------------------------------------------------ */

static int mark_slot_used(orc_ss* ss, const char* name)
{
    /* SpinOperation::markSlotUsed, spinoperation.cpp:238-245 */
    int s = orc_ss_slot(ss, name);
    ss->used[s] = 1;
    return s;
}

/* Exchange::apply, M/cpu/exchange/spinoperationexchange.cpp:134-213.
 * Adds into the slot (no zeroing); three passes, one per component. */
void orc_exchange_apply(orc_ss* ss, const int* from, const int* to, const double* J,
                        int npath, int normalize, double gscale)
{
    int s = mark_slot_used(ss, "Exchange");
    double* h[3] = {ss->hx[s], ss->hy[s], ss->hz[s]};
    const double* v[3] = {ss->x, ss->y, ss->z};
    const double* mm = ss->ms;
    for (int c = 0; c < 3; c++) {
        for (int p = 0; p < npath; p++) {
            const int t = to[p], f = from[p];
            const double st = J[p];
            if (mm[f]) {
                if (normalize) h[c][t] += v[c][f] * st * gscale / (mm[f] * mm[t]);
                else           h[c][t] += v[c][f] * st * gscale / mm[f];
            }
        }
    }
}

/* Anisotropy::apply, M/cpu/anisotropy/spinoperationanisotropy.cpp:247-283.
 * Axis stored normalised by l_add (:367-410). */
void orc_anisotropy_apply(orc_ss* ss, const int* site, const double* axis, const double* K,
                          int nops, double gscale)
{
    int s = mark_slot_used(ss, "Anisotropy");
    double *hx = ss->hx[s], *hy = ss->hy[s], *hz = ss->hz[s];
    memset(hx, 0, sizeof(double) * ss->n);
    memset(hy, 0, sizeof(double) * ss->n);
    memset(hz, 0, sizeof(double) * ss->n);
    for (int j = 0; j < nops; j++) {
        const int i = site[j];
        const double ms = ss->ms[i];
        if (ms > 0) {
            const double* a = axis + 3 * j;
            const double sda = ss->x[i] * a[0] + ss->y[i] * a[1] + ss->z[i] * a[2];
            const double v = 2.0 * K[j] * sda / (ms * ms);
            hx[i] += a[0] * v * gscale;
            hy[i] += a[1] * v * gscale;
            hz[i] += a[2] * v * gscale;
        }
    }
}

/* AnisotropyUniaxial::addAnisotropy scales the axis by 1/dot(a,a) (not
 * 1/|a|), spinoperationanisotropy_uniaxial.cpp:158-179. */
void orc_uniaxial_axis(const double* a, double out[3])
{
    out[0] = a[0]; out[1] = a[1]; out[2] = a[2];
    const double len = a[0] * a[0] + a[1] * a[1] + a[2] * a[2];
    if (len > 0) { out[0] *= 1.0 / len; out[1] *= 1.0 / len; out[2] *= 1.0 / len; }
}

/* AnisotropyUniaxial::apply, ..._uniaxial.cpp:250-298.  quirk=1 keeps the
 * reference's s.n = sx*nx + sy*ny + sz*nx (:287); quirk=0 uses sz*nz. */
void orc_anisotropy_uniaxial_apply(orc_ss* ss, const int* site, const double* axis,
                                   const double* K1, const double* K2, int nops,
                                   double gscale, int quirk)
{
    int s = mark_slot_used(ss, "UniaxialAnisotropy");
    double *hx = ss->hx[s], *hy = ss->hy[s], *hz = ss->hz[s];
    memset(hx, 0, sizeof(double) * ss->n);
    memset(hy, 0, sizeof(double) * ss->n);
    memset(hz, 0, sizeof(double) * ss->n);
    for (int j = 0; j < nops; j++) {
        const int i = site[j];
        const double ms = ss->ms[i];
        if (ms > 0) {
            const double sx = ss->x[i] / ms, sy = ss->y[i] / ms, sz = ss->z[i] / ms;
            const double nx = axis[3 * j], ny = axis[3 * j + 1], nz = axis[3 * j + 2];
            const double sda = sx * nx + sy * ny + sz * (quirk ? nx : nz);
            const double sda3 = sda * sda * sda;
            const double mag = 2.0 * K1[j] * sda + 4.0 * K2[j] * sda3;
            hx[i] += nx * mag * gscale;
            hy[i] += ny * mag * gscale;
            hz[i] += nz * mag * gscale;
        }
    }
}

static double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static void cross3(const double* a, const double* b, double* c)
{
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

/* AnisotropyCubic::addAnisotropy axis construction,
 * spinoperationanisotropy_cubic.cpp:180-236.  Returns nonzero on the
 * reference's error cases (zero length 1, colinear 2). */
int orc_cubic_axes(const double* a1_in, const double* a2_in, double out[9])
{
    double a1[3] = {a1_in[0], a1_in[1], a1_in[2]}, a2[3] = {a2_in[0], a2_in[1], a2_in[2]};
    if (dot3(a1, a1) == 0 || dot3(a2, a2) == 0) return 1;
    double s1 = 1.0 / sqrt(dot3(a1, a1));
    a1[0] *= s1; a1[1] *= s1; a1[2] *= s1;
    double s2 = 1.0 / sqrt(dot3(a2, a2));
    a2[0] *= s2; a2[1] *= s2; a2[2] *= s2;
    if (fabs(dot3(a1, a2)) == 1) return 2;
    double a3[3];
    cross3(a1, a2, a3);
    double s3 = 1.0 / sqrt(dot3(a3, a3));
    a3[0] *= s3; a3[1] *= s3; a3[2] *= s3;
    if (dot3(a1, a2) != 0) {
        double p[3], d = dot3(a1, a2);
        p[0] = a1[0] * d; p[1] = a1[1] * d; p[2] = a1[2] * d;
        a2[0] = a2[0] + -1 * p[0]; a2[1] = a2[1] + -1 * p[1]; a2[2] = a2[2] + -1 * p[2];
    }
    memcpy(out, a1, sizeof(a1));
    memcpy(out + 3, a2, sizeof(a2));
    cross3(out, out + 3, out + 6);
    for (int i = 0; i < 3; i++) {
        const double len = dot3(out + 3 * i, out + 3 * i);
        if (len > 0) { double sc = 1.0 / len; out[3 * i] *= sc; out[3 * i + 1] *= sc; out[3 * i + 2] *= sc; }
    }
    return 0;
}

/* AnisotropyCubic::apply, spinoperationanisotropy_cubic.cpp:308-390.
 * quirk=1 keeps the (n2s2 + n3s3) typo of the first K1 term (:372-374). */
void orc_anisotropy_cubic_apply(orc_ss* ss, const int* site, const double* axes,
                                const double* K, int nops, double gscale, int quirk)
{
    int s = mark_slot_used(ss, "CubicAnisotropy");
    double *hx = ss->hx[s], *hy = ss->hy[s], *hz = ss->hz[s];
    memset(hx, 0, sizeof(double) * ss->n);
    memset(hy, 0, sizeof(double) * ss->n);
    memset(hz, 0, sizeof(double) * ss->n);
    for (int j = 0; j < nops; j++) {
        const int i = site[j];
        const double ms = ss->ms[i];
        if (!(ms > 0)) continue;
        const double sx = ss->x[i] / ms, sy = ss->y[i] / ms, sz = ss->z[i] / ms;
        const double* n = axes + 9 * j;
        const double n1x = n[0], n1y = n[1], n1z = n[2];
        const double n2x = n[3], n2y = n[4], n2z = n[5];
        const double n3x = n[6], n3y = n[7], n3z = n[8];
        const double K1 = K[3 * j], K2 = K[3 * j + 1], K3 = K[3 * j + 2];
        const double n1s = n1x * sx + n1y * sy + n1z * sz;
        const double n2s = n2x * sx + n2y * sy + n2z * sz;
        const double n3s = n3x * sx + n3y * sy + n3z * sz;
        const double n1s2 = n1s * n1s, n2s2 = n2s * n2s, n3s2 = n3s * n3s;
        const double n1s3 = n1s2 * n1s, n2s3 = n2s2 * n2s, n3s3 = n3s2 * n3s;
        const double n1s4 = n1s2 * n1s2, n2s4 = n2s2 * n2s2, n3s4 = n3s2 * n3s2;
        const double q = quirk ? n3s3 : n3s2;
        const double t1x = 2.0 * K1 * (n1x * n1s * (n2s2 + q) + n2x * n2s * (n1s2 + n3s2) + n3x * n3s * (n1s2 + n2s2));
        const double t1y = 2.0 * K1 * (n1y * n1s * (n2s2 + q) + n2y * n2s * (n1s2 + n3s2) + n3y * n3s * (n1s2 + n2s2));
        const double t1z = 2.0 * K1 * (n1z * n1s * (n2s2 + q) + n2z * n2s * (n1s2 + n3s2) + n3z * n3s * (n1s2 + n2s2));
        const double t2x = 2.0 * K2 * (n1s * n2s * n3s * (n1x * n2s * n3s + n2x * n1s * n3s + n3x * n1s * n2s));
        const double t2y = 2.0 * K2 * (n1s * n2s * n3s * (n1y * n2s * n3s + n2y * n1s * n3s + n3y * n1s * n2s));
        const double t2z = 2.0 * K2 * (n1s * n2s * n3s * (n1z * n2s * n3s + n2z * n1s * n3s + n3z * n1s * n2s));
        const double t3x = 4.0 * K3 * (n1x * n1s3 * (n2s4 + n3s4) + n2x * n2s3 * (n1s4 + n3s4) + n3x * n3s3 * (n1s4 + n2s4));
        const double t3y = 4.0 * K3 * (n1y * n1s3 * (n2s4 + n3s4) + n2y * n2s3 * (n1s4 + n3s4) + n3y * n3s3 * (n1s4 + n2s4));
        const double t3z = 4.0 * K3 * (n1z * n1s3 * (n2s4 + n3s4) + n2z * n2s3 * (n1s4 + n3s4) + n3z * n3s3 * (n1s4 + n2s4));
        hx[i] += gscale * (t1x + t2x + t3x);
        hy[i] += gscale * (t1y + t2y + t3y);
        hz[i] += gscale * (t1z + t2z + t3z);
    }
}

/* Thermal::apply, M/cpu/thermal/spinoperationthermal.cpp:135-191: the slot
 * is overwritten; sigma = sqrt(2 alpha_i gscale T scale_i / (ms dt gamma_i))
 * with the system dt; normals drawn hx, hy, hz per active site in order. */
static double site_a(const orc_ss* ss, int i) { return ss->site_alpha ? ss->site_alpha[i] : ss->alpha; }
static double site_g(const orc_ss* ss, int i) { return ss->site_gamma ? ss->site_gamma[i] : ss->gamma; }

int orc_thermal_apply(orc_ss* ss, double T, const double* scale, double gscale, orc_mt* rng)
{
    int s = mark_slot_used(ss, "Thermal");
    if (!rng) return -1; /* "Missing RNG" */
    double *hx = ss->hx[s], *hy = ss->hy[s], *hz = ss->hz[s];
    for (int i = 0; i < ss->n; i++) {
        hx[i] = hy[i] = hz[i] = 0;
        if (ss->ms[i] != 0 && T != 0) {
            const double a = site_a(ss, i), g = site_g(ss, i);
            if (g > 0) {
                const double sc = scale ? scale[i] : 1.0;
                const double sd = sqrt((2.0 * a * gscale * T * sc) / (ss->ms[i] * ss->dt * g));
                hx[i] = sd * orc_mt_randnorm(rng, 0, 1);
                hy[i] = sd * orc_mt_randnorm(rng, 0, 1);
                hz[i] = sd * orc_mt_randnorm(rng, 0, 1);
            }
        }
    }
    return 0;
}

/* Draw the normals Thermal::apply would consume, placed per site (zero on
 * sites that draw nothing).  Used to inject the reference stream into the
 * GPU path. */
void orc_thermal_draw(const orc_ss* ss, double T, orc_mt* rng, double* nx, double* ny, double* nz)
{
    for (int i = 0; i < ss->n; i++) {
        nx[i] = ny[i] = nz[i] = 0;
        if (ss->ms[i] != 0 && T != 0 && site_g(ss, i) > 0) {
            nx[i] = orc_mt_randnorm(rng, 0, 1);
            ny[i] = orc_mt_randnorm(rng, 0, 1);
            nz[i] = orc_mt_randnorm(rng, 0, 1);
        }
    }
}

void orc_thermal_apply_noise(orc_ss* ss, double T, const double* scale, double gscale,
                             const double* nx, const double* ny, const double* nz)
{
    int s = mark_slot_used(ss, "Thermal");
    double *hx = ss->hx[s], *hy = ss->hy[s], *hz = ss->hz[s];
    for (int i = 0; i < ss->n; i++) {
        hx[i] = hy[i] = hz[i] = 0;
        if (ss->ms[i] != 0 && T != 0) {
            const double a = site_a(ss, i), g = site_g(ss, i);
            if (g > 0) {
                const double sc = scale ? scale[i] : 1.0;
                const double sd = sqrt((2.0 * a * gscale * T * sc) / (ss->ms[i] * ss->dt * g));
                hx[i] = sd * nx[i]; hy[i] = sd * ny[i]; hz[i] = sd * nz[i];
            }
        }
    }
}

/* AppliedField Lua apply: ensureSlotExists, setAll(B*scale), setSlotUsed,
 * M/cpu/appliedfield/appliedfield_luafuncs.lua:46-60. */
void orc_zeeman_apply(orc_ss* ss, const double B[3], double gscale)
{
    int s = mark_slot_used(ss, "Zeeman");
    for (int i = 0; i < ss->n; i++) {
        ss->hx[s][i] = B[0] * gscale;
        ss->hy[s][i] = B[1] * gscale;
        ss->hz[s][i] = B[2] * gscale;
    }
}

/* ------------------------------------------------------------------ */
/* FFT (FP64, any length: mixed-radix recursion over a twiddle table,   */
/* direct DFT for prime factors)                                         */
/* ------------------------------------------------------------------ */
typedef struct fft_plan { int n; double* tw; double* a; double* b; double* c; } fft_plan;
static fft_plan* g_plans[64];
static int g_nplans;

static fft_plan* get_plan(int n)
{
    for (int i = 0; i < g_nplans; i++) if (g_plans[i]->n == n) return g_plans[i];
    fft_plan* p = (fft_plan*)malloc(sizeof(fft_plan));
    p->n = n;
    p->tw = (double*)malloc(sizeof(double) * 2 * n);
    for (int k = 0; k < n; k++) {
        p->tw[2 * k] = cos(2.0 * M_PI * (double)k / n);
        p->tw[2 * k + 1] = -sin(2.0 * M_PI * (double)k / n);
    }
    p->a = (double*)malloc(sizeof(double) * 2 * n);
    p->b = (double*)malloc(sizeof(double) * 2 * n);
    p->c = (double*)malloc(sizeof(double) * 2 * n);
    if (g_nplans < 64) g_plans[g_nplans++] = p;
    return p;
}

static int smallest_factor(int n)
{
    for (int p = 2; p * p <= n; p++) if (n % p == 0) return p;
    return n;
}

/* out[k] = sum_j in[j*istride] * exp(sign*2*pi*i*j*k/n).  tw holds
 * exp(-2*pi*i*k/N) for the top-level N; sign=+1 uses its conjugate. */
static void fft_rec(const double* in, int istride, double* out, int n, int sign,
                    double* tmp, const double* tw, int N)
{
    if (n == 1) { out[0] = in[0]; out[1] = in[1]; return; }
    const int p = smallest_factor(n);
    const int m = n / p;
    const int step = N / n;
    const double sg = sign < 0 ? 1.0 : -1.0;
    if (p == n) {
        for (int k = 0; k < n; k++) {
            double sr = 0, si = 0;
            for (int j = 0; j < n; j++) {
                const int e = (int)(((long long)j * k) % n) * step;
                const double c = tw[2 * e], s = sg * tw[2 * e + 1];
                const double xr = in[2 * j * istride], xi = in[2 * j * istride + 1];
                sr += xr * c - xi * s;
                si += xr * s + xi * c;
            }
            out[2 * k] = sr; out[2 * k + 1] = si;
        }
        return;
    }
    for (int r = 0; r < p; r++)
        fft_rec(in + 2 * r * istride, istride * p, tmp + 2 * r * m, m, sign, out, tw, N);
    for (int k = 0; k < m; k++) {
        for (int q = 0; q < p; q++) {
            const int kk = k + q * m;
            double sr = tmp[2 * k], si = tmp[2 * k + 1];
            for (int r = 1; r < p; r++) {
                const int e = (int)(((long long)r * kk) % n) * step;
                const double c = tw[2 * e], s = sg * tw[2 * e + 1];
                const double xr = tmp[2 * (r * m + k)], xi = tmp[2 * (r * m + k) + 1];
                sr += xr * c - xi * s;
                si += xr * s + xi * c;
            }
            out[2 * kk] = sr; out[2 * kk + 1] = si;
        }
    }
}

void orc_fft1d(double* data, int n, int stride, int sign)
{
    fft_plan* P = get_plan(n);
    for (int i = 0; i < n; i++) { P->a[2 * i] = data[2 * (size_t)i * stride]; P->a[2 * i + 1] = data[2 * (size_t)i * stride + 1]; }
    fft_rec(P->a, 1, P->b, n, sign, P->c, P->tw, n);
    for (int i = 0; i < n; i++) { data[2 * (size_t)i * stride] = P->b[2 * i]; data[2 * (size_t)i * stride + 1] = P->b[2 * i + 1]; }
}

/* fft2DTo: a 2D transform of every z layer, fourier.cpp:112-126. */
void orc_fft2d_layers(double* d, int nx, int ny, int nz, int sign)
{
    for (int z = 0; z < nz; z++) {
        double* L = d + 2 * (size_t)z * nx * ny;
        for (int y = 0; y < ny; y++) orc_fft1d(L + 2 * (size_t)y * nx, nx, 1, sign);
        for (int x = 0; x < nx; x++) orc_fft1d(L + 2 * x, ny, nx, sign);
    }
}

void orc_fft3d(double* d, int nx, int ny, int nz, int sign)
{
    orc_fft2d_layers(d, nx, ny, nz, sign);
    for (int y = 0; y < ny; y++)
        for (int x = 0; x < nx; x++) orc_fft1d(d + 2 * (x + (size_t)nx * y), nz, nx * ny, sign);
}

/* ------------------------------------------------------------------ */
/* Dipole tensor                                                         */
/* ------------------------------------------------------------------ */

/* gamma_ab_dip = -(delta_ab/r^3 - 3 r_a r_b / r^5), zero for r < 1e-40,
 * M/cpu/dipole/dipolesupport.cpp:32-70. */
static void gamma_dip(double rx, double ry, double rz, double* g6)
{
    double r = sqrt(rx * rx + ry * ry + rz * rz);
    if (r < 1E-40) { g6[0] = g6[1] = g6[2] = g6[3] = g6[4] = g6[5] = 0; return; }
    const double ir = 1.0 / r, ir3 = ir * ir * ir, ir5 = ir3 * ir * ir;
    g6[0] = -1.0 * (ir3 - 3.0 * rx * rx * ir5);
    g6[1] = -1.0 * (-3.0 * rx * ry * ir5);
    g6[2] = -1.0 * (-3.0 * rx * rz * ir5);
    g6[3] = -1.0 * (ir3 - 3.0 * ry * ry * ir5);
    g6[4] = -1.0 * (-3.0 * ry * rz * ir5);
    g6[5] = -1.0 * (ir3 - 3.0 * rz * rz * ir5);
}

static long long floor_div(long long a, long long b)
{
    long long q = a / b;
    if ((a % b != 0) && ((a < 0) != (b < 0))) q--;
    return q;
}

/* getWAB with smin=0 (single range, index 8) and getWAB_range,
 * dipolesupport.cpp:71-240.  Image indices X, Y run over
 * [-(G-1), G-1] in ascending order (X outer), contributing when
 * |X nx + i| <= min(gmax[2], gmax[0]), |Y ny + j| <= min(gmax[3], gmax[0]),
 * |k| <= gmax[0] and the radial test.  The reference's z test reads
 * truemax[4], one element past the gmax[4] array (:80): undefined
 * behaviour that, whenever the stray word is large and positive, puts no
 * limit on |k|; this restatement takes that branch.  Iterating only the
 * X and Y that can pass the box tests visits the same terms in the same
 * order as the reference's full loop. */
static void get_wab(const double* ABC, int nA, int nB, int ix, int iy, int iz,
                    const int* gmax, double* out6)
{
    double acc[6] = {0, 0, 0, 0, 0, 0};
    const int G = gmax[0];
    const long long R = gmax[0];
    if (!(llabs(iz) <= R)) { memset(out6, 0, sizeof(double) * 6); return; }
    const long long limx = gmax[2] < gmax[0] ? gmax[2] : gmax[0];
    const long long limy = gmax[3] < gmax[0] ? gmax[3] : gmax[0];
    long long xlo = -(G - 1), xhi = G - 1, ylo = -(G - 1), yhi = G - 1;
    /* |X nA + ix| <= limx  <=>  (-limx - ix)/nA <= X <= (limx - ix)/nA */
    long long a = -floor_div(limx + ix, nA); /* ceil((-limx-ix)/nA) */
    long long b = floor_div(limx - ix, nA);
    if (a > xlo) xlo = a;
    if (b < xhi) xhi = b;
    a = -floor_div(limy + iy, nB);
    b = floor_div(limy - iy, nB);
    if (a > ylo) ylo = a;
    if (b < yhi) yhi = b;
    for (long long X = xlo; X <= xhi; X++) {
        const long long xx = X * nA + ix;
        for (long long Y = ylo; Y <= yhi; Y++) {
            const long long yy = Y * nB + iy;
            const long long zz = iz;
            if (((double)xx * xx + (double)yy * yy + (double)zz * zz) <= ((double)R * (double)R)) {
                const double rx = ((double)xx) * ABC[0] + ((double)yy) * ABC[3] + ((double)zz) * ABC[6];
                const double ry = ((double)xx) * ABC[1] + ((double)yy) * ABC[4] + ((double)zz) * ABC[7];
                const double rz = ((double)xx) * ABC[2] + ((double)yy) * ABC[5] + ((double)zz) * ABC[8];
                double g6[6];
                gamma_dip(rx, ry, rz, g6);
                for (int q = 0; q < 6; q++) acc[q] += g6[q];
            }
        }
    }
    memcpy(out6, acc, sizeof(acc));
}

/* dipoleLoad element loop k in [-nz+1, nz-1], j, i (dipolesupport.cpp:757-770). */
void orc_dipole_tensor(int nx, int ny, int nz, const int gmax[4], const double ABC[9],
                       double* XX, double* XY, double* XZ, double* YY, double* YZ, double* ZZ)
{
    int c = 0;
    for (int k = -nz + 1; k < nz; k++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                double o[6];
                get_wab(ABC, nx, ny, i, j, k, gmax, o);
                XX[c] = o[0]; XY[c] = o[1]; XZ[c] = o[2];
                YY[c] = o[3]; YZ[c] = o[4]; ZZ[c] = o[5];
                c++;
            }
}

/* getWAB_range over one rectangle of images [ax, bx] x [ay, by] (X outer,
 * Y inner) with the truncation of the math.huge sum, truemax = {1e9, ...}:
 * every box and radial test passes for lattices of fewer than 1e5 sites a
 * side out to 5000 lattices (dipolesupport.cpp:71-128, the z test's
 * truemax[4] taken large as in get_wab). */
static void wab_rect(const double* ABC, int nA, int nB, int ix, int iy, int iz, int ax, int ay, int bx, int by,
                     double* acc)
{
    for (long long X = ax; X <= bx; X++) {
        const long long xx = X * nA + ix;
        for (long long Y = ay; Y <= by; Y++) {
            const long long yy = Y * nB + iy;
            const long long zz = iz;
            const double rx = ((double)xx) * ABC[0] + ((double)yy) * ABC[3] + ((double)zz) * ABC[6];
            const double ry = ((double)xx) * ABC[1] + ((double)yy) * ABC[4] + ((double)zz) * ABC[7];
            const double rz = ((double)xx) * ABC[2] + ((double)yy) * ABC[5] + ((double)zz) * ABC[8];
            double g6[6];
            gamma_dip(rx, ry, rz, g6);
            for (int q = 0; q < 6; q++) acc[q] += g6[q];
        }
    }
}

/* The Dipole tensor of truncation math.huge (dipoleLoad, dipolesupport.cpp:
 * 771-835): per element the images are summed ring by ring, rings of lstep
 * lattices (getWAB with smin = q lstep, smax = smin + lstep: the full square
 * for smin = 0, else its eight rectangles in getWAB's order, :150-232), each
 * ring's sum added to the running total.  The reference asks its Lua
 * extrapolate() for two results where the function returns one, so the
 * convergence flag it reads is nil and the loop always runs its maxiter =
 * 1000 rings of 5 lattices; the result is the last running total.  nrings
 * and lstep are parameters here (1000 and 5 in the reference). */
void orc_dipole_tensor_rings(int nx, int ny, int nz, const double ABC[9], int nrings, int lstep,
                             double* XX, double* XY, double* XZ, double* YY, double* YZ, double* ZZ)
{
    int c = 0;
    for (int k = -nz + 1; k < nz; k++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                double s[6] = {0, 0, 0, 0, 0, 0};
                for (int q = 0; q < nrings; q++) {
                    const int mn = q * lstep, mx = mn + lstep;
                    double t[6] = {0, 0, 0, 0, 0, 0};
                    if (mn == 0) {
                        wab_rect(ABC, nx, ny, i, j, k, -(mx - 1), -(mx - 1), mx - 1, mx - 1, t);
                    } else {
                        const int ax[8] = {-(mx - 1), -mn + 1, mn, -(mx - 1), mn, -(mx - 1), -mn + 1, mn};
                        const int bx[8] = {-mn, mn - 1, mx - 1, -mn, mx - 1, -mn, mn - 1, mx - 1};
                        const int ay[8] = {mn, mn, mn, -(mn - 1), -(mn - 1), -(mx - 1), -(mx - 1), -(mx - 1)};
                        const int by[8] = {mx - 1, mx - 1, mx - 1, mn - 1, mn - 1, -mn, -mn, -mn};
                        for (int r = 0; r < 8; r++) wab_rect(ABC, nx, ny, i, j, k, ax[r], ay[r], bx[r], by[r], t);
                    }
                    for (int a = 0; a < 6; a++) s[a] += t[a];
                }
                XX[c] = s[0]; XY[c] = s[1]; XZ[c] = s[2];
                YY[c] = s[3]; YZ[c] = s[4]; ZZ[c] = s[5];
                c++;
            }
}

/* ------------------------------------------------------------------ */
/* Magnetostatic (deprecated LongRange subclass): prism tensors          */
/* ------------------------------------------------------------------ */
/* Restated from M/cpu/magnetostatics/gamma_ab_v.cpp (after J. Geophys. Res.
 * 98 B6 9551, 1993): the demagnetising tensor N_ab of a rectangular prism
 * (dx, dy, dz) seen from another at offset (X, Y, Z), with the reference's
 * guards (invtan with a zero denominator, phi = asinh(n/d) with 1000 sign(n)
 * for d = 0). */
static double mg_invtan(double num, double den)
{
    if (den == 0) return num > 0 ? M_PI * 0.5 : -M_PI * 0.5;
    return atan(num / den);
}
static double mg_sign(double x) { return x > 0 ? 1.0 : (x < 0 ? -1.0 : 0.0); }
static double mg_phi(double n, double d)
{
    if (n == 0) return 0;
    if (d == 0) return 1000 * mg_sign(n);
    const double p = n / d;
    return log(p + sqrt(1.0 + p * p));
}
static double mg_g(double x, double y, double z)
{
    const double xx = x * x, yy = y * y, zz = z * z;
    const double R = sqrt(xx + yy + zz);
    return (x * y * z) * mg_phi(z, sqrt(xx + yy)) + (y / 6.0) * (3.0 * zz - yy) * mg_phi(x, sqrt(yy + zz)) +
           (x / 6.0) * (3.0 * zz - xx) * mg_phi(y, sqrt(xx + zz)) - (z * zz / 6.0) * mg_invtan(x * y, (z * R)) -
           (z * yy / 2.0) * mg_invtan(x * z, (y * R)) - (z * xx / 2.0) * mg_invtan(y * z, (x * R)) - (x * y * R / 3.0);
}
static double mg_G2(double x, double y, double z) { return mg_g(x, y, z) - mg_g(x, y, 0); }
static double mg_G1(double X, double Y, double Z, double dx, double dy, double dz)
{
    (void)dy;
    return mg_G2(X + dx, Y, Z + dz) - mg_G2(X + dx, Y, Z) - mg_G2(X, Y, Z + dz) + mg_G2(X, Y, Z);
}
static double mg_G0(double X, double Y, double Z, double dx, double dy, double dz)
{
    return mg_G1(X, Y, Z, dx, dy, dz) - mg_G1(X, Y - dy, Z, dx, dy, dz) - mg_G1(X, Y, Z - dz, dx, dy, dz) +
           mg_G1(X, Y - dy, Z - dz, dx, dy, dz);
}
static double mg_f(double x, double y, double z)
{
    const double xx = x * x, yy = y * y, zz = z * z;
    const double R = sqrt(xx + yy + zz);
    return y * 0.5 * (zz - xx) * mg_phi(y, sqrt(xx + zz)) + z * 0.5 * (yy - xx) * mg_phi(z, sqrt(xx + yy)) -
           x * y * z * mg_invtan(y * z, x * R) + (1.0 / 6.0) * (2.0 * xx - yy - zz) * R;
}
static double mg_F2(double X, double Y, double Z) { return mg_f(X, Y, Z) - mg_f(X, 0, Z) - mg_f(X, Y, 0) + mg_f(X, 0, 0); }
static double mg_F1(double X, double Y, double Z, double dx, double dy, double dz)
{
    (void)dx;
    return mg_F2(X, Y, Z) - mg_F2(X, Y - dy, Z) - mg_F2(X, Y, Z - dz) + mg_F2(X, Y - dy, Z - dz);
}
static double mg_F0(double X, double Y, double Z, double dx, double dy, double dz)
{
    return mg_F1(X, Y + dy, Z + dz, dx, dy, dz) - mg_F1(X, Y, Z + dz, dx, dy, dz) - mg_F1(X, Y + dy, Z, dx, dy, dz) +
           mg_F1(X, Y, Z, dx, dy, dz);
}
static double mg_Nxx(double X, double Y, double Z, double dx, double dy, double dz)
{
    const double tau = dx * dy * dz;
    return -1.0 * (1.0 / (4.0 * M_PI * tau)) *
           (2.0 * mg_F0(X, Y, Z, dx, dy, dz) - mg_F0(X + dx, Y, Z, dx, dy, dz) - mg_F0(X - dx, Y, Z, dx, dy, dz));
}
static double mg_Nxy(double X, double Y, double Z, double dx, double dy, double dz)
{
    const double tau = dx * dy * dz;
    return -1.0 * (1.0 / (4.0 * M_PI * tau)) *
           (mg_G0(X, Y, Z, dx, dy, dz) - mg_G0(X - dx, Y, Z, dx, dy, dz) - mg_G0(X, Y + dy, Z, dx, dy, dz) +
            mg_G0(X - dx, Y + dy, Z, dx, dy, dz));
}
/* the six components XX, XY, XZ, YY, YZ, ZZ (gamma_ab_v.cpp:135-188) */
static double mg_gamma_v(int c, double x, double y, double z, const double* p)
{
    switch (c) {
    case 0: return mg_Nxx(x, y, z, p[0], p[1], p[2]);
    case 1: return mg_Nxy(x, y, z, p[0], p[1], p[2]);
    case 2: return mg_Nxy(x, z, y, p[0], p[2], p[1]);
    case 3: return mg_Nxx(y, x, z, p[1], p[0], p[2]);
    case 4: return mg_Nxy(y, z, x, p[1], p[2], p[0]);
    default: return mg_Nxx(z, y, x, p[2], p[1], p[0]);
    }
}
static int mg_equal_tol(double a, double b, double tol)
{
    if (a == 0 && b == 0) return 1;
    if (b == 0 || a == 0) return 0;
    const double t1 = fabs((a - b) / a), t2 = fabs((a - b) / b);
    return t1 < tol && t2 < tol;
}
typedef struct { double x, y, z, r2; } mg_pt;
static int mg_cmp(const void* a, const void* b)
{
    const double u = ((const mg_pt*)a)->r2, v = ((const mg_pt*)b)->r2;
    return u < v ? -1 : (u > v ? 1 : 0);
}

/* magnetostaticsLoad for a finite truncation (magnetostaticssupport.cpp:
 * 799-866 with getGAB, :191-318, smin = 0, and getGAB_range, :81-187): per
 * element the images inside the truncation (the tests of the Dipole sum,
 * truemax[4] taken large) collected in X-outer Y-inner order, sorted by r^2,
 * then per component summed from the nearest out: the prism tensor until the
 * first image where it and the point dipole (DipMagConversion 1/(4 pi) times
 * the prism volume times gamma_dip) agree within tol (relative, both ways),
 * the point dipole from there on.  The crossover restarts for every
 * element. */
void orc_magnetostatic_tensor(int nx, int ny, int nz, const int gmax[4], const double ABC[9], const double prism[3],
                              double tol, double* XX, double* XY, double* XZ, double* YY, double* YZ, double* ZZ)
{
    double* out[6] = {XX, XY, XZ, YY, YZ, ZZ};
    const double volume = prism[0] * prism[1] * prism[2];
    const int G = gmax[0];
    const long long cap = (long long)(2 * G - 1) * (2 * G - 1);
    mg_pt* pts = (mg_pt*)malloc(sizeof(mg_pt) * (size_t)(cap > 0 ? cap : 1));
    int c = 0;
    for (int k = -nz + 1; k < nz; k++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                long long np = 0;
                const int zz = k;
                if (abs(zz) <= gmax[0]) {
                    for (int X = -(G - 1); X <= G - 1; X++) {
                        const int xx = X * nx + i;
                        if (!(abs(xx) <= gmax[2] && abs(xx) <= gmax[0])) continue;
                        for (int Y = -(G - 1); Y <= G - 1; Y++) {
                            const int yy = Y * ny + j;
                            if (!(abs(yy) <= gmax[3] && abs(yy) <= gmax[0])) continue;
                            if (((double)xx * xx + (double)yy * yy + (double)zz * zz) <= ((double)gmax[0] * (double)gmax[0])) {
                                mg_pt q;
                                q.x = ((double)xx) * ABC[0] + ((double)yy) * ABC[3] + ((double)zz) * ABC[6];
                                q.y = ((double)xx) * ABC[1] + ((double)yy) * ABC[4] + ((double)zz) * ABC[7];
                                q.z = ((double)xx) * ABC[2] + ((double)yy) * ABC[5] + ((double)zz) * ABC[8];
                                q.r2 = q.x * q.x + q.y * q.y + q.z * q.z;
                                pts[np++] = q;
                            }
                        }
                    }
                }
                qsort(pts, (size_t)np, sizeof(mg_pt), mg_cmp);
                for (int a = 0; a < 6; a++) {
                    double cross_r2 = 1e10, g = 0;
                    for (long long p = 0; p < np; p++) {
                        double dip = 0, mag;
                        if (tol > 0) {
                            double g6[6];
                            gamma_dip(pts[p].x, pts[p].y, pts[p].z, g6);
                            dip = (1.0 / (M_PI * 4.0)) * volume * g6[a];
                        }
                        if (pts[p].r2 >= cross_r2) {
                            mag = dip;
                        } else {
                            mag = mg_gamma_v(a, pts[p].x, pts[p].y, pts[p].z, prism);
                            if (tol > 0 && mg_equal_tol(mag, dip, tol) && pts[p].r2 > 0 && pts[p].r2 < cross_r2)
                                cross_r2 = pts[p].r2;
                        }
                        g += mag;
                    }
                    out[a][c] = g;
                }
                c++;
            }
    free(pts);
}

/* LongRange context: the tensor transforms of updateData, prescaled by
 * 1/(nx*ny), spinoperationlongrange.cpp:275-312, plus workspaces. */
struct orc_lr {
    int nx, ny, nz;
    double* q[6];
    double* sq[3];
    double* ws;
};

orc_lr* orc_lr_new(int nx, int ny, int nz, double* const T6[6])
{
    orc_lr* c = (orc_lr*)calloc(1, sizeof(orc_lr));
    const int nxy = nx * ny, L = 2 * nz - 1, n = nxy * nz;
    c->nx = nx; c->ny = ny; c->nz = nz;
    for (int a = 0; a < 6; a++) {
        c->q[a] = (double*)calloc((size_t)2 * nxy * L, sizeof(double));
        for (int i = 0; i < nxy * L; i++) c->q[a][2 * i] = T6[a][i];
        orc_fft2d_layers(c->q[a], nx, ny, L, -1);
        for (int i = 0; i < 2 * nxy * L; i++) c->q[a][i] *= 1.0 / ((double)(nx * ny));
    }
    for (int b = 0; b < 3; b++) c->sq[b] = (double*)malloc(sizeof(double) * 2 * (size_t)n);
    c->ws = (double*)malloc(sizeof(double) * 2 * (size_t)n);
    return c;
}

void orc_lr_free(orc_lr* c)
{
    if (!c) return;
    for (int a = 0; a < 6; a++) free(c->q[a]);
    for (int b = 0; b < 3; b++) free(c->sq[b]);
    free(c->ws);
    free(c);
}

/* LongRange::apply, spinoperationlongrange.cpp:354-440.  Tensor layer o
 * holds z offset o-(nz-1) = source - target. */
void orc_lr_apply(orc_lr* c, orc_ss* ss, const char* slot, double g, double gscale)
{
    const int nx = ss->nx, ny = ss->ny, nz = ss->nz, nxy = nx * ny;
    int s = mark_slot_used(ss, slot);
    /* spin transforms (SpinSystem::fft, spinsystem.cpp:936-966) */
    const double* v[3] = {ss->x, ss->y, ss->z};
    for (int b = 0; b < 3; b++) {
        memset(c->sq[b], 0, sizeof(double) * 2 * (size_t)ss->n);
        for (int i = 0; i < ss->n; i++) c->sq[b][2 * i] = v[b][i];
        orc_fft2d_layers(c->sq[b], nx, ny, nz, -1);
    }
    /* H_a(t) = sum_s sum_b Q_ab(s-t+nz-1) S_b(s);
     * HX: XX,XY,XZ  HY: XY,YY,YZ  HZ: XZ,YZ,ZZ */
    const int comp[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
    double* ws = c->ws;
    double* out[3] = {ss->hx[s], ss->hy[s], ss->hz[s]};
    for (int a = 0; a < 3; a++) {
        memset(ws, 0, sizeof(double) * 2 * (size_t)ss->n);
        for (int t = 0; t < nz; t++)
            for (int sl = 0; sl < nz; sl++) {
                const int off = sl - t + nz - 1;
                for (int b = 0; b < 3; b++) {
                    const double* Q = c->q[comp[a][b]] + 2 * (size_t)off * nxy;
                    const double* S = c->sq[b] + 2 * (size_t)sl * nxy;
                    double* D = ws + 2 * (size_t)t * nxy;
                    for (int i = 0; i < nxy; i++) {
                        /* d += s1 * s2 * one (arrayLayerMult_, array_ops.cpp:652-668) */
                        const double qr = Q[2 * i], qi = Q[2 * i + 1];
                        const double sr = S[2 * i], si = S[2 * i + 1];
                        D[2 * i] += qr * sr - qi * si;
                        D[2 * i + 1] += qr * si + qi * sr;
                    }
                }
            }
        orc_fft2d_layers(ws, nx, ny, nz, +1);
        for (int i = 0; i < ss->n; i++) out[a][i] = ws[2 * i];
        for (int i = 0; i < ss->n; i++) out[a][i] *= g * gscale;
    }
}

void orc_longrange_apply(orc_ss* ss, const char* slot, double* const T6[6], double g, double gscale)
{
    orc_lr* c = orc_lr_new(ss->nx, ss->ny, ss->nz, T6);
    orc_lr_apply(c, ss, slot, g, gscale);
    orc_lr_free(c);
}

/* LongRange3D::compile + apply, spinoperationlongrange3d.cpp:331-424. */
void orc_longrange3d_apply(orc_ss* ss, double* const T9[9], double g, double gscale)
{
    const int nx = ss->nx, ny = ss->ny, nz = ss->nz, n = ss->n;
    int s = mark_slot_used(ss, "LongRange3D");
    double* q[9];
    for (int a = 0; a < 9; a++) {
        q[a] = (double*)calloc((size_t)2 * n, sizeof(double));
        for (int i = 0; i < n; i++) q[a][2 * i] = T9[a][i];
        orc_fft3d(q[a], nx, ny, nz, -1);
        for (int i = 0; i < 2 * n; i++) q[a][i] *= 1.0 / ((double)(nx * ny * nz));
    }
    double* sq[3];
    const double* v[3] = {ss->x, ss->y, ss->z};
    for (int c = 0; c < 3; c++) {
        sq[c] = (double*)calloc((size_t)2 * n, sizeof(double));
        for (int i = 0; i < n; i++) sq[c][2 * i] = v[c][i];
        orc_fft3d(sq[c], nx, ny, nz, -1);
    }
    double* ws = (double*)malloc(sizeof(double) * 2 * n);
    double* out[3] = {ss->hx[s], ss->hy[s], ss->hz[s]};
    for (int a = 0; a < 3; a++) {
        memset(ws, 0, sizeof(double) * 2 * n);
        for (int b = 0; b < 3; b++) {
            const double* Q = q[3 * a + b];
            const double* S = sq[b];
            for (int i = 0; i < n; i++) {
                const double qr = Q[2 * i], qi = Q[2 * i + 1], sr = S[2 * i], si = S[2 * i + 1];
                ws[2 * i] += qr * sr - qi * si;
                ws[2 * i + 1] += qr * si + qi * sr;
            }
        }
        orc_fft3d(ws, nx, ny, nz, +1);
        for (int i = 0; i < n; i++) out[a][i] = ws[2 * i] * (g * gscale);
    }
    free(ws);
    for (int a = 0; a < 9; a++) free(q[a]);
    for (int c = 0; c < 3; c++) free(sq[c]);
}

/* Physical direct sum.  p{x,y,z} = 1 applies the minimum-image wrap in
 * that axis (single image), 0 = open. */
void orc_dipole_direct(const orc_ss* ss, const double ABC[9], double g,
                       int px, int py, int pz, double* hx, double* hy, double* hz)
{
    const int nx = ss->nx, ny = ss->ny, nz = ss->nz;
    for (int t = 0; t < ss->n; t++) {
        const int tx = t % nx, ty = (t / nx) % ny, tz = t / (nx * ny);
        double ax = 0, ay = 0, az = 0;
        for (int s = 0; s < ss->n; s++) {
            const int sx = s % nx, sy = (s / nx) % ny, sz = s / (nx * ny);
            int dx = tx - sx, dy = ty - sy, dz = tz - sz;
            if (px) { if (dx > nx / 2) dx -= nx; if (dx < -(nx - 1) / 2) dx += nx; }
            if (py) { if (dy > ny / 2) dy -= ny; if (dy < -(ny - 1) / 2) dy += ny; }
            if (pz) { if (dz > nz / 2) dz -= nz; if (dz < -(nz - 1) / 2) dz += nz; }
            const double rx = dx * ABC[0] + dy * ABC[3] + dz * ABC[6];
            const double ry = dx * ABC[1] + dy * ABC[4] + dz * ABC[7];
            const double rz = dx * ABC[2] + dy * ABC[5] + dz * ABC[8];
            double G[6];
            gamma_dip(rx, ry, rz, G);
            ax += G[0] * ss->x[s] + G[1] * ss->y[s] + G[2] * ss->z[s];
            ay += G[1] * ss->x[s] + G[3] * ss->y[s] + G[4] * ss->z[s];
            az += G[2] * ss->x[s] + G[4] * ss->y[s] + G[5] * ss->z[s];
        }
        hx[t] = g * ax; hy[t] = g * ay; hz[t] = g * az;
    }
}

/* The same open-boundary direct sum at chosen target sites only, over
 * spin arrays given directly (for lattices too large for the O(N^2) form):
 * out[3*q + a] = g * sum_s Gamma(r_t - r_s) m_s for target t = sites[q]. */
void orc_dipole_direct_sites(int nx, int ny, int nz, const double* x, const double* y, const double* z,
                             const double ABC[9], double g, const long long* sites, int nsites, double* out)
{
    const long long n = (long long)nx * ny * nz;
    for (int q = 0; q < nsites; q++) {
        const long long t = sites[q];
        const int tx = (int)(t % nx), ty = (int)((t / nx) % ny), tz = (int)(t / ((long long)nx * ny));
        double ax = 0, ay = 0, az = 0;
        for (long long s = 0; s < n; s++) {
            const int sx = (int)(s % nx), sy = (int)((s / nx) % ny), sz = (int)(s / ((long long)nx * ny));
            const int dx = tx - sx, dy = ty - sy, dz = tz - sz;
            const double rx = dx * ABC[0] + dy * ABC[3] + dz * ABC[6];
            const double ry = dx * ABC[1] + dy * ABC[4] + dz * ABC[7];
            const double rz = dx * ABC[2] + dy * ABC[5] + dz * ABC[8];
            double G[6];
            gamma_dip(rx, ry, rz, G);
            ax += G[0] * x[s] + G[1] * y[s] + G[2] * z[s];
            ay += G[1] * x[s] + G[3] * y[s] + G[4] * z[s];
            az += G[2] * x[s] + G[4] * y[s] + G[5] * z[s];
        }
        out[3 * q] = g * ax; out[3 * q + 1] = g * ay; out[3 * q + 2] = g * az;
    }
}

/* Gamma(r) for every offset d = t - s of an open nx x ny x nz lattice,
 * r = d . ABC (the same kernel as orc_dipole_direct_sites), written as six
 * arrays (XX, XY, XZ, YY, YZ, ZZ) of (2nx-1)(2ny-1)(2nz-1) values at
 * (dx+nx-1) + (2nx-1)*((dy+ny-1) + (2ny-1)*(dz+nz-1)); Gamma(0) = 0.  The
 * open-boundary field is this tensor's linear convolution with the spins. */
void orc_dipole_open_tensor(int nx, int ny, int nz, const double ABC[9], double* out6)
{
    const long long Lx = 2 * nx - 1, Ly = 2 * ny - 1, Lz = 2 * nz - 1, L = Lx * Ly * Lz;
    for (int dz = -(nz - 1); dz <= nz - 1; dz++)
        for (int dy = -(ny - 1); dy <= ny - 1; dy++)
            for (int dx = -(nx - 1); dx <= nx - 1; dx++) {
                const double rx = dx * ABC[0] + dy * ABC[3] + dz * ABC[6];
                const double ry = dx * ABC[1] + dy * ABC[4] + dz * ABC[7];
                const double rz = dx * ABC[2] + dy * ABC[5] + dz * ABC[8];
                double G[6];
                gamma_dip(rx, ry, rz, G);
                const long long o = (dx + nx - 1) + Lx * ((dy + ny - 1) + Ly * (long long)(dz + nz - 1));
                for (int c = 0; c < 6; c++) out6[c * L + o] = G[c];
            }
}

/* ------------------------------------------------------------------ */
/* LLG                                                                  */
/* ------------------------------------------------------------------ */
void orc_llg_default(orc_llg* l)
{
    l->thermal_only_first_term = 1; l->disable_renormalization = 0;
    l->precess_scale = 1; l->damp_scale = 1;
}

#define CROSS(v, a, b) \
    v[0] = a[1] * b[2] - a[2] * b[1]; \
    v[1] = a[2] * b[0] - a[0] * b[2]; \
    v[2] = a[0] * b[1] - a[1] * b[0];

/* renormalisation to ms of the from-system, llgcartesian.cpp:262-277 */
static void renormalize(orc_ss* to, const double* ms)
{
    for (int i = 0; i < to->n; i++) {
        const double mm = to->x[i] * to->x[i] + to->y[i] * to->y[i] + to->z[i] * to->z[i];
        if (mm != 0) {
            const double inv = ms[i] / sqrt(mm);
            to->x[i] *= inv; to->y[i] *= inv; to->z[i] *= inv;
        }
    }
}

/* LLGCartesian::apply, M/cpu/llg/llgcartesian.cpp:90-278. */
void orc_llg_cart_apply(const orc_llg* l, orc_ss* from, double scale, orc_ss* dmdt,
                        orc_ss* to, int advance)
{
    const int SUM = orc_ss_find_slot(dmdt, "Total");
    const int TH = orc_ss_find_slot(dmdt, "Thermal");
    if (SUM < 0) {
        if (advance) to->time = from->time + scale * dmdt->dt;
        return;
    }
    const double* ms = from->ms;
    const double dt = scale * dmdt->dt;
    const int n = from->n;
    /* from and to may alias: keep a copy of the from spins */
    double* sx = (double*)malloc(sizeof(double) * n);
    double* sy = (double*)malloc(sizeof(double) * n);
    double* sz = (double*)malloc(sizeof(double) * n);
    double* msc = (double*)malloc(sizeof(double) * n);
    memcpy(sx, from->x, sizeof(double) * n);
    memcpy(sy, from->y, sizeof(double) * n);
    memcpy(sz, from->z, sizeof(double) * n);
    memcpy(msc, ms, sizeof(double) * n);
    if (dt == 0) {
        memcpy(to->x, sx, sizeof(double) * n);
        memcpy(to->y, sy, sizeof(double) * n);
        memcpy(to->z, sz, sizeof(double) * n);
    } else {
        for (int i = 0; i < n; i++) {
            to->ms[i] = msc[i];
            if (!(msc[i] > 0)) continue;
            double dM[3], M[3], H[3], MH[3], MMH[3];
            M[0] = dmdt->x[i]; M[1] = dmdt->y[i]; M[2] = dmdt->z[i];
            H[0] = dmdt->hx[SUM][i]; H[1] = dmdt->hy[SUM][i]; H[2] = dmdt->hz[SUM][i];
            const double a = site_a(dmdt, i), g = site_g(dmdt, i);
            const double gaa = g / (1.0 + a * a);
            if (l->thermal_only_first_term) {
                double h[3];
                if (TH >= 0) {
                    h[0] = H[0] - dmdt->hx[TH][i];
                    h[1] = H[1] - dmdt->hy[TH][i];
                    h[2] = H[2] - dmdt->hz[TH][i];
                } else { h[0] = H[0]; h[1] = H[1]; h[2] = H[2]; }
                CROSS(MH, M, h);
                CROSS(MMH, M, MH);
                CROSS(MH, M, H);
                for (int c = 0; c < 3; c++)
                    dM[c] = l->precess_scale * -gaa * MH[c] - l->damp_scale * (a / msc[i]) * gaa * MMH[c];
            } else {
                CROSS(MH, M, H);
                CROSS(MMH, M, MH);
                for (int c = 0; c < 3; c++) dM[c] = -gaa * MH[c] - (a / msc[i]) * gaa * MMH[c];
            }
            to->x[i] = (sx[i] + dt * dM[0]);
            to->y[i] = (sy[i] + dt * dM[1]);
            to->z[i] = (sz[i] + dt * dM[2]);
        }
        if (advance) to->time = from->time + dt;
    }
    if (!l->disable_renormalization) renormalize(to, msc);
    free(sx); free(sy); free(sz); free(msc);
}

typedef struct { double w, x, y, z; } quat;
static quat qmult(quat a, quat b)
{
    quat ab;
    ab.w = a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z;
    ab.x = a.w * b.x + b.w * a.x + a.y * b.z - a.z * b.y;
    ab.y = a.w * b.y + b.w * a.y + a.z * b.x - a.x * b.z;
    ab.z = a.w * b.z + b.w * a.z + a.x * b.y - a.y * b.x;
    return ab;
}
static quat qmult_xyz(quat a, quat b)
{
    quat ab;
    ab.x = a.w * b.x + b.w * a.x + a.y * b.z - a.z * b.y;
    ab.y = a.w * b.y + b.w * a.y + a.z * b.x - a.x * b.z;
    ab.z = a.w * b.z + b.w * a.z + a.x * b.y - a.y * b.x;
    ab.w = 0;
    return ab;
}
static quat qconj(quat q) { quat r = {q.w, -1.0 * q.x, -1.0 * q.y, -1.0 * q.z}; return r; }

/* LLGQuaternion::apply, M/cpu/llg/llgquat.cpp:126-378. */
void orc_llg_quat_apply(const orc_llg* l, orc_ss* from, double scale, orc_ss* dmdt,
                        orc_ss* to, int advance)
{
    const int SUM = orc_ss_find_slot(dmdt, "Total");
    const int TH = orc_ss_find_slot(dmdt, "Thermal");
    if (SUM < 0) {
        if (advance) to->time = from->time + dmdt->dt * scale;
        return;
    }
    const int n = from->n;
    const double dt = dmdt->dt * scale;
    double* sx = (double*)malloc(sizeof(double) * n);
    double* sy = (double*)malloc(sizeof(double) * n);
    double* sz = (double*)malloc(sizeof(double) * n);
    double* msc = (double*)malloc(sizeof(double) * n);
    memcpy(sx, from->x, sizeof(double) * n);
    memcpy(sy, from->y, sizeof(double) * n);
    memcpy(sz, from->z, sizeof(double) * n);
    memcpy(msc, from->ms, sizeof(double) * n);
    for (int i = 0; i < n; i++) {
        to->ms[i] = msc[i];
        if (!(msc[i] > 0)) continue;
        double S[3] = {sx[i], sy[i], sz[i]};
        double H[3] = {dmdt->hx[SUM][i], dmdt->hy[SUM][i], dmdt->hz[SUM][i]};
        const double inv = 1.0 / msc[i];
        const double a = site_a(dmdt, i), g = site_g(dmdt, i);
        if (l->thermal_only_first_term) {
            double M[3] = {dmdt->x[i], dmdt->y[i], dmdt->z[i]};
            double h[3], Sh[3];
            if (TH >= 0) {
                h[0] = H[0] - dmdt->hx[TH][i];
                h[1] = H[1] - dmdt->hy[TH][i];
                h[2] = H[2] - dmdt->hz[TH][i];
            } else { h[0] = H[0]; h[1] = H[1]; h[2] = H[2]; }
            CROSS(Sh, M, h);
            for (int j = 0; j < 3; j++) H[j] = l->precess_scale * H[j] + l->damp_scale * a * Sh[j] * inv;
        } else {
            double SH[3];
            CROSS(SH, S, H);
            for (int j = 0; j < 3; j++) H[j] += a * SH[j] * inv;
        }
        const double HLen = sqrt(H[0] * H[0] + H[1] * H[1] + H[2] * H[2]);
        if (HLen > 0) {
            const double iHLen = 1.0 / HLen;
            const double ra = 1.0 * g * HLen / (1.0 + a * a);
            const double cost = cos(0.5 * ra * dt), sint = sin(0.5 * ra * dt);
            quat qRot = {cost, sint * H[0] * iHLen, sint * H[1] * iHLen, sint * H[2] * iHLen};
            quat qVec = {0, S[0], S[1], S[2]};
            quat qRes = qmult_xyz(qmult(qRot, qVec), qconj(qRot));
            to->x[i] = qRes.x; to->y[i] = qRes.y; to->z[i] = qRes.z;
        } else {
            to->x[i] = S[0]; to->y[i] = S[1]; to->z[i] = S[2];
        }
    }
    if (advance) to->time = from->time + dt;
    if (!l->disable_renormalization) renormalize(to, msc);
    free(sx); free(sy); free(sz); free(msc);
}

/* ------------------------------------------------------------------ */
/* Canonical step driver                                                 */
/* ------------------------------------------------------------------ */
void orc_run_steps(orc_ss* ss, const orc_step_cfg* c, int nsteps)
{
    for (int it = 0; it < nsteps; it++) {
        orc_ss_reset_fields(ss);
        if (c->npath) orc_exchange_apply(ss, c->from, c->to, c->J, c->npath, c->ex_normalize, 1.0);
        if (c->nani) orc_anisotropy_apply(ss, c->ani_site, c->ani_axis, c->ani_K, c->nani, 1.0);
        if (c->ncub) orc_anisotropy_cubic_apply(ss, c->cub_site, c->cub_axes, c->cub_K, c->ncub, 1.0, c->cub_quirk);
        if (c->T != 0 && c->rng) orc_thermal_apply(ss, c->T, NULL, 1.0, c->rng);
        if (c->zeeman) orc_zeeman_apply(ss, c->B, 1.0);
        if (c->dipole) orc_lr_apply(c->lr, ss, "Dipole", c->g, 1.0);
        orc_ss_sum_fields(ss);
        if (c->llg_type == 0) orc_llg_cart_apply(&c->llg, ss, 1.0, ss, ss, 1);
        else orc_llg_quat_apply(&c->llg, ss, 1.0, ss, ss, 1);
    }
}
