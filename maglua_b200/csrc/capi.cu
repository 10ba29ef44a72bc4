// capi.cu -- host layer behind include/mlb200.h.
//
// Object model (mirrors MagLua's SpinSystem / SpinOperation / LLG classes):
//   * mlb_system: SoA spins (FP32, or FP64 for systems created with 8-byte
//     reals) in two generations (ping-pong buffers), ms,
//     per-site alpha/gamma, named field slots ("Total" is slot 0).
//   * Field slots are evaluated lazily.  A slot is ZERO, DATA (device arrays
//     hold its value), LAZY (a base -- zero or its arrays -- plus operator terms
//     recorded at apply time against a spin generation) or SUM ("Total" after
//     sumFields, defined by the slots it sums).  Reading a slot, or anything
//     that would invalidate a record, materialises it with k_eval_terms.  When
//     llg:apply(ss) meets a lazily defined "Total", the whole step runs as one
//     fused kernel (field terms + LLG) that writes the other spin buffer.
//   * Dipole / LongRange / LongRange3D run eagerly (FFT convolution pipeline)
//     into DATA slots that the fused kernel reads.
#include "../../include/mlb200.h"
#include "device.cuh"
#include "kparams.h"
#include "launch.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <new>
#include <set>
#include <stdexcept>
#include <string>
#include <strings.h>
#include <vector>
#include <thread>
#include <atomic>
#include <mutex>
#include <cstdlib>
#include <sys/stat.h>

namespace {

thread_local std::string g_err;

struct Err {
    int code;
    std::string msg;
};

#define CK(x)                                                                                  \
    do {                                                                                       \
        cudaError_t e_ = (x);                                                                  \
        if (e_ != cudaSuccess)                                                                 \
            throw Err{e_ == cudaErrorMemoryAllocation ? MLB_ENOMEM : MLB_ECUDA,                \
                      std::string(#x) + ": " + cudaGetErrorString(e_)};                        \
    } while (0)

[[noreturn]] void fail(int code, const std::string& m) { throw Err{code, m}; }

template <class F>
int guard(F&& f)
{
    try {
        f();
        return MLB_OK;
    } catch (Err& e) {
        g_err = e.msg;
        return e.code;
    } catch (std::bad_alloc&) {
        g_err = "host allocation failed";
        return MLB_ENOMEM;
    } catch (std::exception& e) {
        g_err = e.what();
        return MLB_EINVAL;
    } catch (...) {
        g_err = "unknown error";
        return MLB_EINVAL;
    }
}

template <class T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    ~DBuf() { release(); }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    void alloc(size_t k)
    {
        if (k == n && p) return;
        release();
        if (k == 0) return;
        CK(cudaMalloc(&p, k * sizeof(T)));
        n = k;
    }
};

bool name_eq(const std::string& a, const char* b) { return strcasecmp(a.c_str(), b) == 0; }

// ------------------------------------------------------------------ FFT plans
std::vector<int> factorize(int n)
{
    std::vector<int> r;
    while (n % 8 == 0 && n != 16 && n / 8 != 2) { r.push_back(8); n /= 8; }
    while (n % 4 == 0) { r.push_back(4); n /= 4; }
    while (n % 2 == 0) { r.push_back(2); n /= 2; }
    for (int p = 3; p <= 7; p += 2)
        while (n % p == 0) { r.push_back(p); n /= p; }
    for (int p = 11; n > 1; p += 2)
        while (n % p == 0) { r.push_back(p); n /= p; }
    return r;
}

FftLen make_len(int n, int tw_off)
{
    FftLen L;
    memset(&L, 0, sizeof(L));
    L.n = n;
    std::vector<int> r = factorize(n);
    if ((int)r.size() > MLB_FFT_MAX_STAGES) fail(MLB_EUNSUP, "FFT length has too many factors");
    for (int p : r)
        if (p > 32) fail(MLB_EUNSUP, "FFT length " + std::to_string(n) + " has a prime factor above 32");
    L.nst = (int)r.size();
    for (size_t i = 0; i < r.size(); i++) L.radix[i] = r[i];
    L.tw_off = tw_off;
    return L;
}

// padded length for an open axis: the smallest power of two >= m (the
// register-FFT fast path covers powers of two)
int nice_len(int m)
{
    if (m <= 1) return 1;
    int best = 1;
    while (best < m) best *= 2;
    return best;
}

template <class C>
void append_twiddles(std::vector<C>& pool, int n)
{
    for (int k = 0; k < n; k++) {
        const double a = 2.0 * M_PI * (double)k / (double)n;
        C c;
        c.x = (decltype(c.x))std::cos(a);
        c.y = (decltype(c.y))(-std::sin(a));
        pool.push_back(c);
    }
}

// Convolution plan of one operator for one lattice size.
struct ConvPlan {
    ConvK k;
    FftLen L[3];
    int rb = 4;          // bytes per real of the arrays below (state precision)
    DBuf<char> tw;       // complex twiddles per axis
    DBuf<char> spec;     // SPEC[kx][c][z][y] (complex)
    DBuf<char> ten6;     // TEN6[kx][kz][ky][6] (real)
    DBuf<char> ten9;     // TEN9[kx][kz][ky][9] (complex)
    DBuf<char> spec2;    // split passes: S2[kx][ky][c][z] (complex)
    double max_imag = 0; // largest |Im| of the FP64 tensor transform (6-component)
    int device = -1;     // CUDA device the arrays above live on
    // SPEC holds the forward x transform of the spins of the system whose
    // spec_token equals this one (set by the fused x pass; 0 = none)
    unsigned long long spec_token = 0;
};

// LongRange2D / Dipole2D: the per-kx layer-mixing convolution and its
// tensor spectrum Q[kx][ky][s][d][9] (complex, state precision).
struct LR2DPlan {
    ConvK k;
    FftLen L[3];
    int rb = 4;
    DBuf<char> tw;
    DBuf<char> spec;
    DBuf<char> spec2;    // S2[kx][ky][c][z] for the FP32 register y passes
    DBuf<char> Q;
};

} // namespace

// ====================================================================== objects
struct Term {
    mlb_op* op;
    int weight;
    uint64_t counter;
    double B[3];
    double T;
    double gs;
    double dt_sys;
};

enum { ST_ZERO = 0, ST_DATA = 1, ST_LAZY = 2, ST_SUM = 3 };

struct Slot {
    std::string name;
    void* h[3] = {nullptr, nullptr, nullptr};
    bool used = false;
    int state = ST_ZERO;
    bool base_data = false;
    std::vector<Term> terms;
    long long gen = 0;
    std::vector<int> sum_list;
};

struct mlb_system {
    int nx, ny, nz, n;
    int rb = 4;                     // bytes per real of every state array (4 or 8)
    void* sp[2][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};
    int cur = 0;
    long long gen = 0;
    void* ms = nullptr;
    std::vector<double> ms_host;    // ms as stored on the device (rounded to rb)
    bool ms_dirty = true;
    // identifies the moment magnitudes held (device ms and ms_host): equal
    // tokens, equal magnitudes; a new one whenever they are set
    unsigned long long ms_token = 0;
    bool ms_uniform = true;
    double ms_u = 0.0;
    void* sa = nullptr;
    void* sg = nullptr;
    double alpha = 1.0, gamma = 1.0, dt = 1.0, time = 0.0;
    std::vector<Slot> slots;
    cudaStream_t own = nullptr;
    cudaStream_t st = nullptr;
    // device step blocks of captured steps, one per spin-buffer parity: a
    // step with parity q reads dstep[q] and writes the next step's values
    // into dstep[1 - q]
    DevStep* dstep = nullptr;
    DevStep dstep_mirror{};         // what dstep[dstep_cur] holds, when dstep_known
    bool dstep_known = false;
    int dstep_cur = 0;
    // netMoment: reduction + copy to pinned memory captured once per spin
    // buffer (and per length argument m)
    // netMoment: the reduction and its copy to pinned memory captured once per
    // spin buffer q and destination d (0: the synchronous read, 1..4: the
    // slots of mlb_system_netmoment_async, each with an event)
    cudaGraphExec_t nm_exec[2][5] = {};
    double nm_m[2][5] = {};
    double* nm_host = nullptr;      // pinned, 5 x 6 doubles (the device writes them directly)
    double* nm_host_dev = nullptr;  // the device's address of nm_host
    unsigned* nm_counter = nullptr; // blocks done in the current netMoment launch
    unsigned* status = nullptr;     // device status word (bit 0: a step wrote a non-finite spin)
    cudaEvent_t nm_ev[4] = {};
    bool nm_pending[4] = {};
    double* red = nullptr;
    double* redout = nullptr;
    int red_nb = 1;
    // mlb_system_netmoment_async runs on a stream of its own (its own
    // partial sums and counter), concurrently with the next steps; slot k
    // reads spin buffer nm_buf[k] until nm_ev[k], and nm_reading[k] stays set
    // until the system's stream has been made to wait for it before a write
    // of that buffer
    cudaStream_t nm_st = nullptr;
    cudaEvent_t nm_go[4] = {};
    int nm_buf[4] = {};
    bool nm_reading[4] = {};
    double* red_a = nullptr;
    double* redout_a = nullptr;
    unsigned* nm_counter_a = nullptr;
    bool capturing = false;
    bool dry = false;               // replay host bookkeeping without launching
    // a system the library owns and never shows to the caller (Runge-Kutta
    // stages, the adaptive stepper's copies): when its spins are overwritten,
    // the fields of the old spins are dropped instead of settled
    bool internal = false;
    bool last_fused = false;
    mlb_surrogate* sur = nullptr;   // learned surrogate standing in for its operator (surrogate runs)
    // Inside do_step the inverse x pass of a fast-path convolution waits for
    // the LLG update, which runs it fused with the step (launch_xstep).
    bool defer_x = false;
    mlb_op* pend_op = nullptr;      // operator whose inverse x pass is pending
    int pend_si = -1;               // and its slot
    bool cap_carry = false;         // capture: assume SPEC holds the current spins' x transform
    mlb_op* cap_xstep = nullptr;    // capture: the convolution whose x pass the captured step fused
    unsigned long long* cap_tl = nullptr;   // capture: device timeline stamps of a timing plan
    unsigned long long spec_token = 0;   // matches ConvPlan::spec_token while that holds
};

struct mlb_op {
    int kind;
    int nx, ny, nz;
    double gs = 1.0;
    std::string slot;
    bool quirks = true;
    // exchange
    std::vector<int> ef, et;
    std::vector<double> eJ;
    bool normalize = true;
    int ex_pbc[3] = {1, 1, 1};   // setPeriodicXYZ (Exchange::Exchange sets all three)
    bool ex_dirty = true;
    ExchangeK exk{};
    DBuf<int> eptr, ecol;
    DBuf<double> eval;
    // anisotropies: per op site + parameters
    std::vector<int> asite;
    std::vector<double> apar; // generic: axis3,K ; uni: axis3,K1,K2 ; cubic: axes9,K3
    bool a_dirty = true;
    AniK anik{};
    UniK unik{};
    CubK cubk{};
    DBuf<int> aptr;
    DBuf<double> aaxes, aK;
    double gs_compiled = -1;
    // thermal
    double T = 0.0;
    std::vector<double> tscale;
    DBuf<double> dscale;
    bool tscale_dirty = false;
    uint64_t seed = 0;
    uint64_t counter = 0;
    bool inject_pending = false;
    DBuf<double> inj[3];
    // applied field
    double B[3] = {0, 0, 0};
    double dB[3] = {0, 0, 0};
    // longrange
    double g = 1.0;
    int gmax[4] = {1000, 1000, 1000, 1000};   // gmax[0] = -1: math.huge
    int rings = 1000;                          // rings of 5 lattices of the math.huge sum
    double mag_prism[3] = {1, 1, 1};           // Magnetostatic: prism (cell) dimensions
    double mag_tol = 0.00001;                  // Magnetostatic: crossover tolerance
    double ABC[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    int open[3] = {0, 0, 1};
    std::vector<double> t6[6];
    bool t6_valid = false;
    bool t6_edited = false;
    std::vector<double> t9[9];
    bool plan_dirty = true;
    std::unique_ptr<ConvPlan> plan;
    // LongRange2D / Dipole2D: the arrays set for (dest i, src j), component
    // ab, at [((i nz + j) 9 + ab) nx ny + y nx + x] (allocated on first use);
    // per-layer source-moment and destination-field scales; the reference's
    // newDataRequired / compileRequired flags
    std::vector<double> t2;
    std::vector<double> lr2_src, lr2_dst;
    bool lr2_newdata = true, lr2_compile = true;
    // Dipole2D builder: unit cell A, B, C per layer, offset per layer,
    // truncation {radial, x, y, z}
    std::vector<double> d2_abc, d2_off, d2_grain;
    int d2_trunc[4] = {25, 25, 25, 25};
    std::unique_ptr<LR2DPlan> lr2;
};

struct mlb_llg {
    int kind;
    int tof = 1;
    int disable_renorm = 0;
    double precess = 1.0, damp = 1.0;
};

// A captured step: one graph per spin-buffer parity q and per carry c
// (index q + 2 c); c = 1 when the convolution's SPEC already holds the
// forward x transform of the current spins (left there by the previous
// step's fused x pass), so the step starts at the (y,z) pass.
// Carried steps captured in one graph by a plan (an even count: a graph
// starts and ends on the same spin buffer).
constexpr int kMultiSteps = 4;

struct mlb_plan {
    mlb_system* s = nullptr;
    std::vector<mlb_op*> ops;
    mlb_llg* l = nullptr;
    bool timing = false;            // event nodes around every kernel
    bool timeline = false;          // device timeline of the fused (y,z) and x passes
    DBuf<unsigned long long> tl;    // its four stamps (ConvK::tl)
    cudaGraphExec_t exec[4] = {nullptr, nullptr, nullptr, nullptr};
    // carried steady state: kMultiSteps consecutive steps in one graph per
    // starting parity (null: none; plans with event nodes or a device
    // timeline keep one step per graph)
    cudaGraphExec_t multi[2] = {nullptr, nullptr};
    std::vector<mlb::ProfCaptured> ev[4];
    mlb_op* carry_op = nullptr;   // the convolution whose SPEC a step leaves carried (null: none)
    std::vector<mlb::ProfCaptured>* last = nullptr;
    unsigned long long version = 0;
};

namespace {

void nm_guard(mlb_system* s, int q);

std::set<mlb_system*> g_systems;
unsigned long long g_ms_token = 0;
unsigned long long g_spec_token = 0;
// bumped by every parameter setter; a plan captured under an older value
// is captured again before its next launch
unsigned long long g_version = 1;
using mlb::ProfCaptured;

// ------------------------------------------------------------------ system helpers
int slot_find(const mlb_system* s, const char* name)
{
    for (size_t i = 0; i < s->slots.size(); i++)
        if (name_eq(s->slots[i].name, name)) return (int)i;
    return -1;
}

int slot_register(mlb_system* s, const char* name)
{
    int i = slot_find(s, name);
    if (i >= 0) return i;
    Slot sl;
    sl.name = name;
    s->slots.push_back(sl);
    return (int)s->slots.size() - 1;
}

void slot_alloc(mlb_system* s, Slot& sl)
{
    if (sl.h[0]) return;
    for (int c = 0; c < 3; c++) CK(cudaMalloc(&sl.h[c], (size_t)s->rb * std::max(1, s->n)));
}

// Byte offset of element i of a state array.
inline void* elem(void* p, size_t i, int rb) { return static_cast<char*>(p) + i * (size_t)rb; }

// Host values in FP64 -> n reals of width rb on the device (stream order).
void put_reals(mlb_system* s, void* dst, const double* src, size_t n)
{
    if (n == 0) return;
    if (s->rb == 8) {
        CK(cudaMemcpyAsync(dst, src, sizeof(double) * n, cudaMemcpyHostToDevice, s->st));
        return;
    }
    std::vector<float> f(n);
    for (size_t i = 0; i < n; i++) f[i] = (float)src[i];
    CK(cudaMemcpyAsync(dst, f.data(), sizeof(float) * n, cudaMemcpyHostToDevice, s->st));
}

// n reals of width rb on the device -> FP64 host values (synchronises).
void get_reals(mlb_system* s, double* dst, const void* src, size_t n)
{
    if (n == 0) return;
    if (s->rb == 8) {
        CK(cudaMemcpyAsync(dst, src, sizeof(double) * n, cudaMemcpyDeviceToHost, s->st));
        CK(cudaStreamSynchronize(s->st));
        return;
    }
    std::vector<float> f(n);
    CK(cudaMemcpyAsync(f.data(), src, sizeof(float) * n, cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    for (size_t i = 0; i < n; i++) dst[i] = f[i];
}

// Value as stored at width rb.
inline double round_to(double v, int rb) { return rb == 8 ? v : (double)(float)v; }

void refresh_ms(mlb_system* s)
{
    if (!s->ms_dirty) return;
    s->ms_uniform = true;
    s->ms_u = s->n ? s->ms_host[0] : 0.0;
    for (int i = 1; i < s->n; i++)
        if (s->ms_host[i] != s->ms_u) { s->ms_uniform = false; break; }
    s->ms_dirty = false;
}

SysK sysk(mlb_system* s, int buf)
{
    refresh_ms(s);
    SysK k;
    k.nx = s->nx; k.ny = s->ny; k.nz = s->nz; k.n = s->n;
    k.x = s->sp[buf][0]; k.y = s->sp[buf][1]; k.z = s->sp[buf][2];
    k.ms = s->ms; k.ms_u = s->ms_u; k.ms_uniform = s->ms_uniform ? 1 : 0;
    k.site_alpha = s->sa; k.site_gamma = s->sg;
    k.alpha = s->alpha; k.gamma = s->gamma;
    return k;
}

int buffer_for_gen(mlb_system* s, long long gen)
{
    if (gen == s->gen) return s->cur;
    if (gen == s->gen - 1) return 1 - s->cur;
    fail(MLB_ESTATE, "internal: lazy field refers to an overwritten spin generation");
}

// ------------------------------------------------------------------ operator compile
void check_site(const mlb_op* op, int idx)
{
    if (idx < 0 || idx >= op->nx * op->ny * op->nz)
        fail(MLB_ERANGE, "site index " + std::to_string(idx) + " outside the operator");
}

// Exchange pathways -> six-direction stencil when the pathway multiset is
// exactly a nearest-neighbour lattice with one J per direction, else CSR by
// target site keeping insertion order.
void compile_exchange(mlb_op* op)
{
    if (!op->ex_dirty) return;
    const int nx = op->nx, ny = op->ny, nz = op->nz, n = nx * ny * nz;
    const size_t np = op->ef.size();
    ExchangeK k{};
    k.normalize = op->normalize ? 1 : 0;
    bool stencil = np > 0;
    double Jd[6];
    bool seen[6] = {false, false, false, false, false, false};
    int pbc[3] = {0, 0, 0};
    const int dims[3] = {nx, ny, nz};
    for (size_t p = 0; p < np && stencil; p++) {
        const int f = op->ef[p], t = op->et[p];
        const int fc[3] = {f % nx, (f / nx) % ny, f / (nx * ny)};
        const int tc[3] = {t % nx, (t / nx) % ny, t / (nx * ny)};
        int dir = -1, wrap = 0;
        for (int a = 0; a < 3; a++) {
            const int d = fc[a] - tc[a];
            if (d == 0) continue;
            if (dir >= 0) { stencil = false; break; }
            if (d == 1) dir = 2 * a;
            else if (d == -1) dir = 2 * a + 1;
            else if (dims[a] > 2 && d == -(dims[a] - 1)) { dir = 2 * a; wrap = 1; }
            else if (dims[a] > 2 && d == dims[a] - 1) { dir = 2 * a + 1; wrap = 1; }
            else { stencil = false; break; }
            if (wrap) pbc[a] = 1;
        }
        if (!stencil) break;
        if (dir < 0) { stencil = false; break; }
        if (!seen[dir]) { seen[dir] = true; Jd[dir] = op->eJ[p]; }
        else if (Jd[dir] != op->eJ[p]) stencil = false;
    }
    if (stencil) {
        // The candidate must reproduce the pathway multiset exactly: every
        // (target, direction) at most once, and per direction as many paths
        // as targets that have that neighbour.
        std::vector<unsigned char> hit((size_t)n * 6, 0);
        long long cnt[6] = {0, 0, 0, 0, 0, 0};
        for (size_t p = 0; p < np && stencil; p++) {
            const int f = op->ef[p], t = op->et[p];
            const int fc[3] = {f % nx, (f / nx) % ny, f / (nx * ny)};
            const int tc[3] = {t % nx, (t / nx) % ny, t / (nx * ny)};
            int dir = -1;
            for (int a = 0; a < 3; a++) {
                const int d = fc[a] - tc[a];
                if (d == 0) continue;
                dir = (d == 1 || (dims[a] > 2 && d == -(dims[a] - 1))) ? 2 * a : 2 * a + 1;
            }
            unsigned char& h = hit[(size_t)t * 6 + dir];
            if (h) stencil = false;
            h = 1;
            cnt[dir]++;
        }
        for (int d = 0; d < 6 && stencil; d++) {
            if (!seen[d]) continue;
            const int a = d >> 1;
            const long long want = pbc[a] ? (long long)n : (long long)n - n / dims[a];
            if (cnt[d] != want) stencil = false;
        }
    }
    if (stencil) {
        k.mode = EX_STENCIL;
        for (int d = 0; d < 6; d++) k.J[d] = seen[d] ? Jd[d] : 0.0;
        for (int a = 0; a < 3; a++) k.pbc[a] = pbc[a];
        op->eptr.release(); op->ecol.release(); op->eval.release();
    } else if (np > 0) {
        k.mode = EX_CSR;
        std::vector<int> cnt(n + 1, 0);
        for (size_t p = 0; p < np; p++) cnt[op->et[p] + 1]++;
        for (int i = 0; i < n; i++) cnt[i + 1] += cnt[i];
        std::vector<int> col(np);
        std::vector<double> val(np);
        std::vector<int> pos(cnt.begin(), cnt.end() - 1);
        for (size_t p = 0; p < np; p++) {
            const int q = pos[op->et[p]]++;
            col[q] = op->ef[p];
            val[q] = op->eJ[p];
        }
        op->eptr.alloc(n + 1); op->ecol.alloc(np); op->eval.alloc(np);
        CK(cudaMemcpy(op->eptr.p, cnt.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(op->ecol.p, col.data(), sizeof(int) * np, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(op->eval.p, val.data(), sizeof(double) * np, cudaMemcpyHostToDevice));
        k.ptr = op->eptr.p; k.col = op->ecol.p; k.val = op->eval.p;
    } else {
        k.mode = EX_NONE;
    }
    op->exk = k;
    op->ex_dirty = false;
}

// Per-site operator lists (generic / uniaxial / cubic anisotropy) -> uniform
// constants when every site has exactly one op with identical parameters,
// else CSR by site (list order kept).  global_scale is folded into K.
void compile_aniso(mlb_op* op)
{
    if (!op->a_dirty && op->gs_compiled == op->gs) return;
    const int n = op->nx * op->ny * op->nz;
    const int npar = op->kind == MLB_OP_ANISOTROPY ? 4 : (op->kind == MLB_OP_UNIAXIAL ? 5 : 12);
    const int nax = op->kind == MLB_OP_CUBIC ? 9 : 3;
    const int nk = npar - nax;
    const size_t no = op->asite.size();
    bool uniform = (int)no == n && n > 0;
    if (uniform) {
        std::vector<char> hit(n, 0);
        for (size_t j = 0; j < no && uniform; j++) {
            if (hit[op->asite[j]]) uniform = false;
            hit[op->asite[j]] = 1;
            for (int q = 0; q < npar && uniform; q++)
                if (op->apar[j * npar + q] != op->apar[q]) uniform = false;
        }
    }
    const int mode = no == 0 ? ANI_NONE : (uniform ? ANI_UNIFORM : ANI_CSR);
    const double gs = op->gs;
    if (mode == ANI_CSR) {
        std::vector<int> cnt(n + 1, 0);
        for (size_t j = 0; j < no; j++) cnt[op->asite[j] + 1]++;
        for (int i = 0; i < n; i++) cnt[i + 1] += cnt[i];
        std::vector<double> ax(no * nax), kk(no * nk);
        std::vector<int> pos(cnt.begin(), cnt.end() - 1);
        for (size_t j = 0; j < no; j++) {
            const int q = pos[op->asite[j]]++;
            for (int a = 0; a < nax; a++) ax[q * nax + a] = op->apar[j * npar + a];
            for (int a = 0; a < nk; a++) kk[q * nk + a] = op->apar[j * npar + nax + a] * gs;
        }
        op->aptr.alloc(n + 1); op->aaxes.alloc(ax.size()); op->aK.alloc(kk.size());
        CK(cudaMemcpy(op->aptr.p, cnt.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(op->aaxes.p, ax.data(), sizeof(double) * ax.size(), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(op->aK.p, kk.data(), sizeof(double) * kk.size(), cudaMemcpyHostToDevice));
    }
    if (op->kind == MLB_OP_ANISOTROPY) {
        AniK k{};
        k.mode = mode;
        if (mode == ANI_UNIFORM) {
            for (int a = 0; a < 3; a++) k.axis[a] = op->apar[a];
            k.K = op->apar[3] * gs;
        } else if (mode == ANI_CSR) { k.ptr = op->aptr.p; k.axes = op->aaxes.p; k.Ks = op->aK.p; }
        op->anik = k;
    } else if (op->kind == MLB_OP_UNIAXIAL) {
        UniK k{};
        k.mode = mode;
        k.quirk = op->quirks ? 1 : 0;
        if (mode == ANI_UNIFORM) {
            for (int a = 0; a < 3; a++) k.axis[a] = op->apar[a];
            k.K1 = op->apar[3] * gs; k.K2 = op->apar[4] * gs;
        } else if (mode == ANI_CSR) { k.ptr = op->aptr.p; k.axes = op->aaxes.p; k.K12 = op->aK.p; }
        op->unik = k;
    } else {
        CubK k{};
        k.mode = mode;
        k.quirk = op->quirks ? 1 : 0;
        if (mode == ANI_UNIFORM) {
            for (int a = 0; a < 9; a++) k.axes[a] = op->apar[a];
            for (int a = 0; a < 3; a++) k.K[a] = op->apar[9 + a] * gs;
        } else if (mode == ANI_CSR) { k.ptr = op->aptr.p; k.axs = op->aaxes.p; k.Ks = op->aK.p; }
        op->cubk = k;
    }
    op->a_dirty = false;
    op->gs_compiled = gs;
}

void compile_thermal_scale(mlb_op* op)
{
    if (!op->tscale_dirty) return;
    const int n = op->nx * op->ny * op->nz;
    op->dscale.alloc(n);
    CK(cudaMemcpy(op->dscale.p, op->tscale.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    op->tscale_dirty = false;
}

// ------------------------------------------------------------------ convolution plans
bool is_conv(int kind)
{
    return kind == MLB_OP_DIPOLE || kind == MLB_OP_LONGRANGE || kind == MLB_OP_LONGRANGE3D ||
           kind == MLB_OP_MAGNETOSTATIC;
}

void plan_sizes(mlb_op* op, ConvPlan& P)
{
    ConvK& k = P.k;
    const size_t cb = (size_t)2 * P.rb;   // bytes per complex value
    k.nx = op->nx; k.ny = op->ny; k.nz = op->nz;
    if (op->kind == MLB_OP_LONGRANGE3D) {
        k.Px = op->nx; k.Py = op->ny; k.Pz = op->nz;
        k.general = 1;
    } else {
        // a user tensor need not be inversion symmetric, so its transform is
        // complex: multiply with the general 3x3 complex form
        k.general = (op->kind == MLB_OP_LONGRANGE || op->t6_edited) ? 1 : 0;
        const bool ox = op->kind == MLB_OP_DIPOLE && op->open[0];
        const bool oy = op->kind == MLB_OP_DIPOLE && op->open[1];
        k.Px = ox ? nice_len(2 * op->nx - 1) : op->nx;
        k.Py = oy ? nice_len(2 * op->ny - 1) : op->ny;
        k.Pz = op->nz == 1 ? 1 : nice_len(2 * op->nz - 1);
    }
    k.Kx = k.Px / 2 + 1;
    k.nrep = 1;
    k.run_if = nullptr;
    int ty = 16;
    while (ty > 1 && (size_t)2 * ty * k.Px * cb > 96 * 1024) ty /= 2;
    k.ty = ty;
    k.split = 0;
    k.spec2 = nullptr;
    // the power-of-two FP32 fast path has its own limits; the general
    // kernels hold a whole padded (y,z) plane of three components twice;
    // larger planes take the split (y,z) passes
    if (P.rb == 4 && mlb::conv_fast_ok(k)) return;
    if ((size_t)6 * k.Py * k.Pz * cb > 227 * 1024) {
        k.split = 1;
        if (mlb::split_smem(k, P.rb) > 227 * 1024)
            fail(MLB_EUNSUP, "padded lengths " + std::to_string(k.Py) + "x" + std::to_string(k.Pz) +
                                 " exceed the split passes of this build at " + std::to_string(8 * P.rb) +
                                 "-bit precision");
        if (P.rb == 4 && mlb::conv_fast_ok(k)) return;
    }
    if ((size_t)2 * k.Px * cb > 96 * 1024) fail(MLB_EUNSUP, "x length too large");
}

void ensure_t6_layout(mlb_op* op)
{
    const size_t ne = (size_t)op->nx * op->ny * (2 * op->nz - 1);
    for (int q = 0; q < 6; q++)
        if (op->t6[q].size() != ne) op->t6[q].assign(ne, 0.0);
}

// The FP32 split passes with power-of-two planes (the register z pass) can
// read a quarter tensor.
bool quarter_ok(const ConvK& k, int rb)
{
    auto p2 = [](int v) { return v >= 32 && v <= 512 && (v & (v - 1)) == 0; };
    return rb == 4 && k.split && !k.general && mlb::conv_fast_ok(k) && p2(k.Py) && p2(k.Pz);
}

// Whether the FP64 transformed tensor W holds the per-axis parities of a
// point-dipole tensor on an orthogonal lattice to 1e-10 of its largest
// element (rounding of the transform is ~1e-15 of it; a tensor without the
// parities misses by O(1)).
bool tensor_has_parities(const double2* W, const ConvK& k, cudaStream_t st)
{
    DBuf<unsigned long long> out;
    out.alloc(3);
    CK(cudaMemsetAsync(out.p, 0, sizeof(unsigned long long) * 3, st));
    CK(mlb::launch_tensor_symcheck(W, k.Px, k.Py, k.Pz, k.Kx, out.p, st));
    unsigned long long h[3];
    CK(cudaMemcpyAsync(h, out.p, sizeof(h), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    double d[3];
    memcpy(d, h, sizeof(d));
    return d[0] > 0 && d[1] <= 1e-10 * d[0] && d[2] <= 1e-10 * d[0];
}

// ------------------------------------------------------------------ Magnetostatic tensor
// The deprecated Magnetostatic operator (M/cpu/magnetostatics): LongRange
// with the volume-averaged interaction of rectangular prisms.  Element
// functions of M/cpu/magnetostatics/gamma_ab_v.cpp (after J. Geophys. Res.
// 98 B6 9551, 1993): the demagnetising tensor N_ab of a prism (dx, dy, dz)
// seen from another at offset (X, Y, Z), as second differences of f and g
// with the reference's guards (a zero denominator in invtan, phi = asinh with
// 1000 sign(n) for d = 0).  Host FP64, as the reference computes it.
namespace mg {
double invtan(double num, double den)
{
    if (den == 0) return num > 0 ? M_PI * 0.5 : -M_PI * 0.5;
    return std::atan(num / den);
}
double sgn(double x) { return x > 0 ? 1.0 : (x < 0 ? -1.0 : 0.0); }
double phi(double n, double d)
{
    if (n == 0) return 0;
    if (d == 0) return 1000 * sgn(n);
    const double p = n / d;
    return std::log(p + std::sqrt(1.0 + p * p));
}
double gfun(double x, double y, double z)
{
    const double xx = x * x, yy = y * y, zz = z * z;
    const double R = std::sqrt(xx + yy + zz);
    return (x * y * z) * phi(z, std::sqrt(xx + yy)) + (y / 6.0) * (3.0 * zz - yy) * phi(x, std::sqrt(yy + zz)) +
           (x / 6.0) * (3.0 * zz - xx) * phi(y, std::sqrt(xx + zz)) - (z * zz / 6.0) * invtan(x * y, (z * R)) -
           (z * yy / 2.0) * invtan(x * z, (y * R)) - (z * xx / 2.0) * invtan(y * z, (x * R)) - (x * y * R / 3.0);
}
double G2(double x, double y, double z) { return gfun(x, y, z) - gfun(x, y, 0); }
double G1(double X, double Y, double Z, double dx, double dz)
{
    return G2(X + dx, Y, Z + dz) - G2(X + dx, Y, Z) - G2(X, Y, Z + dz) + G2(X, Y, Z);
}
double G0(double X, double Y, double Z, double dx, double dy, double dz)
{
    return G1(X, Y, Z, dx, dz) - G1(X, Y - dy, Z, dx, dz) - G1(X, Y, Z - dz, dx, dz) + G1(X, Y - dy, Z - dz, dx, dz);
}
double ffun(double x, double y, double z)
{
    const double xx = x * x, yy = y * y, zz = z * z;
    const double R = std::sqrt(xx + yy + zz);
    return y * 0.5 * (zz - xx) * phi(y, std::sqrt(xx + zz)) + z * 0.5 * (yy - xx) * phi(z, std::sqrt(xx + yy)) -
           x * y * z * invtan(y * z, x * R) + (1.0 / 6.0) * (2.0 * xx - yy - zz) * R;
}
double F2(double X, double Y, double Z) { return ffun(X, Y, Z) - ffun(X, 0, Z) - ffun(X, Y, 0) + ffun(X, 0, 0); }
double F1(double X, double Y, double Z, double dy, double dz)
{
    return F2(X, Y, Z) - F2(X, Y - dy, Z) - F2(X, Y, Z - dz) + F2(X, Y - dy, Z - dz);
}
double F0(double X, double Y, double Z, double dy, double dz)
{
    return F1(X, Y + dy, Z + dz, dy, dz) - F1(X, Y, Z + dz, dy, dz) - F1(X, Y + dy, Z, dy, dz) + F1(X, Y, Z, dy, dz);
}
double Nxx(double X, double Y, double Z, double dx, double dy, double dz)
{
    const double tau = dx * dy * dz;
    return -1.0 * (1.0 / (4.0 * M_PI * tau)) * (2.0 * F0(X, Y, Z, dy, dz) - F0(X + dx, Y, Z, dy, dz) - F0(X - dx, Y, Z, dy, dz));
}
double Nxy(double X, double Y, double Z, double dx, double dy, double dz)
{
    const double tau = dx * dy * dz;
    return -1.0 * (1.0 / (4.0 * M_PI * tau)) *
           (G0(X, Y, Z, dx, dy, dz) - G0(X - dx, Y, Z, dx, dy, dz) - G0(X, Y + dy, Z, dx, dy, dz) +
            G0(X - dx, Y + dy, Z, dx, dy, dz));
}
// XX, XY, XZ, YY, YZ, ZZ (gamma_ab_v.cpp:135-188)
double gamma_v(int c, double x, double y, double z, const double* p)
{
    switch (c) {
    case 0: return Nxx(x, y, z, p[0], p[1], p[2]);
    case 1: return Nxy(x, y, z, p[0], p[1], p[2]);
    case 2: return Nxy(x, z, y, p[0], p[2], p[1]);
    case 3: return Nxx(y, x, z, p[1], p[0], p[2]);
    case 4: return Nxy(y, z, x, p[1], p[2], p[0]);
    default: return Nxx(z, y, x, p[2], p[1], p[0]);
    }
}
// the point-dipole elements (dipolesupport.cpp:32-70)
double gamma_dip(int c, double rx, double ry, double rz)
{
    const double r = std::sqrt(rx * rx + ry * ry + rz * rz);
    if (r < 1E-40) return 0;
    const double ir = 1.0 / r, ir3 = ir * ir * ir, ir5 = ir3 * ir * ir;
    switch (c) {
    case 0: return -1.0 * (ir3 - 3.0 * rx * rx * ir5);
    case 1: return -1.0 * (-3.0 * rx * ry * ir5);
    case 2: return -1.0 * (-3.0 * rx * rz * ir5);
    case 3: return -1.0 * (ir3 - 3.0 * ry * ry * ir5);
    case 4: return -1.0 * (-3.0 * ry * rz * ir5);
    default: return -1.0 * (ir3 - 3.0 * rz * rz * ir5);
    }
}
bool equal_tol(double a, double b, double tol)
{
    if (a == 0 && b == 0) return true;
    if (b == 0 || a == 0) return false;
    const double t1 = std::fabs((a - b) / a), t2 = std::fabs((a - b) / b);
    return t1 < tol && t2 < tol;
}
struct Pt {
    double x, y, z, r2;
};
} // namespace mg

// magnetostaticsLoad for a finite truncation (magnetostaticssupport.cpp:
// 799-866, getGAB with smin = 0 :191-318, getGAB_range :81-187): per element
// (k from -nz+1, then j, i) the images inside the truncation (the tests of
// the Dipole sum, truemax[4] taken large) in X-outer Y-inner order, sorted by
// r^2 with std::sort as the reference sorts them; per component, from the
// nearest out, the prism tensor until the first image where it and the point
// dipole (1/(4 pi) x prism volume x gamma_dip) agree within the crossover
// tolerance, the point dipole from there on; the crossover restarts at every
// element.  Elements are independent: host threads take them in chunks.
void build_magnetostatic_t6(mlb_op* op)
{
    if (op->gmax[0] < 0)
        fail(MLB_EUNSUP, "Magnetostatic truncation math.huge: the reference's ring sum (getGAB with smin > 0) "
                         "keeps only the last of each ring's eight ranges, so it is not a lattice sum");
    const int nx = op->nx, ny = op->ny, nz = op->nz;
    const size_t ne = (size_t)nx * ny * (2 * nz - 1);
    ensure_t6_layout(op);
    const int* gm = op->gmax;
    const double* A = op->ABC;
    const double* prism = op->mag_prism;
    const double tol = op->mag_tol;
    const double volume = prism[0] * prism[1] * prism[2];
    const int G = gm[0];
    std::atomic<size_t> next(0);
    const size_t chunk = 16;
    auto work = [&]() {
        std::vector<mg::Pt> pts;
        for (;;) {
            const size_t e0 = next.fetch_add(chunk);
            if (e0 >= ne) break;
            for (size_t e = e0; e < std::min(ne, e0 + chunk); e++) {
                const int i = (int)(e % nx), j = (int)((e / nx) % ny);
                const int k = (int)(e / ((size_t)nx * ny)) - (nz - 1);
                pts.clear();
                if (std::abs(k) <= gm[0]) {
                    for (int X = -(G - 1); X <= G - 1; X++) {
                        const int xx = X * nx + i;
                        if (!(std::abs(xx) <= gm[2] && std::abs(xx) <= gm[0])) continue;
                        for (int Y = -(G - 1); Y <= G - 1; Y++) {
                            const int yy = Y * ny + j;
                            if (!(std::abs(yy) <= gm[3] && std::abs(yy) <= gm[0])) continue;
                            if (((double)xx * xx + (double)yy * yy + (double)k * k) <= ((double)gm[0] * (double)gm[0])) {
                                mg::Pt q;
                                q.x = ((double)xx) * A[0] + ((double)yy) * A[3] + ((double)k) * A[6];
                                q.y = ((double)xx) * A[1] + ((double)yy) * A[4] + ((double)k) * A[7];
                                q.z = ((double)xx) * A[2] + ((double)yy) * A[5] + ((double)k) * A[8];
                                q.r2 = q.x * q.x + q.y * q.y + q.z * q.z;
                                pts.push_back(q);
                            }
                        }
                    }
                }
                std::sort(pts.begin(), pts.end(), [](const mg::Pt& a, const mg::Pt& b) { return a.r2 < b.r2; });
                for (int c = 0; c < 6; c++) {
                    double cross_r2 = 1e10, g = 0;
                    for (const mg::Pt& q : pts) {
                        double dip = 0, mag;
                        if (tol > 0) dip = (1.0 / (M_PI * 4.0)) * volume * mg::gamma_dip(c, q.x, q.y, q.z);
                        if (q.r2 >= cross_r2) {
                            mag = dip;
                        } else {
                            mag = mg::gamma_v(c, q.x, q.y, q.z, prism);
                            if (tol > 0 && mg::equal_tol(mag, dip, tol) && q.r2 > 0 && q.r2 < cross_r2) cross_r2 = q.r2;
                        }
                        g += mag;
                    }
                    op->t6[c][e] = g;
                }
            }
        }
    };
    const unsigned nt = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    std::vector<std::thread> th;
    for (unsigned t = 1; t < nt; t++) th.emplace_back(work);
    work();
    for (std::thread& t : th) t.join();
    op->t6_valid = true;
}

// Build or rebuild the tensor spectrum of op (FP64 on the GPU), stored at
// rb bytes per real for the systems it is applied to.
void build_plan(mlb_op* op, cudaStream_t st, int rb)
{
    if (!op->plan_dirty && op->plan && op->plan->rb == rb) return;
    std::unique_ptr<ConvPlan> P(new ConvPlan());
    P->rb = rb;
    CK(cudaGetDevice(&P->device));
    plan_sizes(op, *P);
    ConvK& k = P->k;
    const int Px = k.Px, Py = k.Py, Pz = k.Pz;
    // twiddle tables: float (per-step FFTs) and double (tensor FFT)
    std::vector<float2> twf;
    std::vector<double2> twd;
    const int lens[3] = {Px, Py, Pz};
    for (int a = 0; a < 3; a++) {
        P->L[a] = make_len(lens[a], (int)twf.size());
        append_twiddles(twf, lens[a]);
        append_twiddles(twd, lens[a]);
    }
    if (rb == 8) {
        P->tw.alloc(sizeof(double2) * twd.size());
        CK(cudaMemcpy(P->tw.p, twd.data(), sizeof(double2) * twd.size(), cudaMemcpyHostToDevice));
    } else {
        P->tw.alloc(sizeof(float2) * twf.size());
        CK(cudaMemcpy(P->tw.p, twf.data(), sizeof(float2) * twf.size(), cudaMemcpyHostToDevice));
    }
    DBuf<double2> twdd;
    twdd.alloc(twd.size());
    CK(cudaMemcpy(twdd.p, twd.data(), sizeof(double2) * twd.size(), cudaMemcpyHostToDevice));

    const int ncomp = k.general ? 9 : 6;
    const size_t plane = (size_t)Px * Py * Pz;
    DBuf<double2> W;
    W.alloc(plane * ncomp);
    CK(cudaMemsetAsync(W.p, 0, sizeof(double2) * plane * ncomp, st));
    const size_t ne = (size_t)op->nx * op->ny * (2 * op->nz - 1);
    if (op->kind == MLB_OP_MAGNETOSTATIC && !op->t6_valid) build_magnetostatic_t6(op);
    if (op->kind == MLB_OP_DIPOLE && !op->t6_valid) {
        if (op->open[0] || op->open[1]) {
            if (!(op->open[0] && op->open[1])) fail(MLB_EUNSUP, "mixed periodic/open in-plane Dipole");
            CK(mlb::launch_tensor_open(op->nx, op->ny, op->nz, op->ABC, Px, Py, Pz, W.p, st));
        } else {
            const int zsign = op->quirks ? -1 : 1;
            if (op->gmax[0] < 0)   // truncation math.huge: the reference's ring sum
                CK(mlb::launch_tensor_rings(op->nx, op->ny, op->nz, op->rings, 5, op->ABC, Px, Py, Pz, zsign, W.p, st));
            else
                CK(mlb::launch_tensor_lattice(op->nx, op->ny, op->nz, op->gmax, op->ABC, Px, Py, Pz, zsign, W.p,
                                              st));
            // keep the reference-layout tensor on the host (getMatrix / tensor arrays)
            DBuf<double> raw;
            raw.alloc(ne * 6);
            CK(mlb::launch_tensor_extract_ref(op->nx, op->ny, op->nz, Px, Py, Pz, zsign, W.p, raw.p, st));
            std::vector<double> h(ne * 6);
            CK(cudaMemcpyAsync(h.data(), raw.p, sizeof(double) * ne * 6, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            for (int q = 0; q < 6; q++) op->t6[q].assign(h.begin() + q * ne, h.begin() + (q + 1) * ne);
            op->t6_valid = true;
        }
    } else if (op->kind == MLB_OP_LONGRANGE3D) {
        std::vector<double2> h(plane * 9);
        for (int q = 0; q < 9; q++) {
            if (op->t9[q].size() != plane) continue;
            for (size_t i = 0; i < plane; i++) h[q * plane + i] = make_double2(op->t9[q][i], 0.0);
        }
        CK(cudaMemcpy(W.p, h.data(), sizeof(double2) * h.size(), cudaMemcpyHostToDevice));
    } else {
        // host tensor (user-set LongRange, or an edited Dipole tensor), z offset
        // k = source - target at padded index (zsign*k mod Pz)
        ensure_t6_layout(op);
        const int zsign = op->quirks ? -1 : 1;
        // six planes (symmetric real path) or nine (general path, XY=YX ...)
        static const int map9[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
        std::vector<double2> h(plane * ncomp, make_double2(0, 0));
        for (int q = 0; q < ncomp; q++)
            for (int kk = -(op->nz - 1); kk < op->nz; kk++) {
                int zi = (zsign * kk) % Pz;
                if (zi < 0) zi += Pz;
                for (int j = 0; j < op->ny; j++)
                    for (int i = 0; i < op->nx; i++) {
                        const size_t src = (size_t)i + op->nx * ((size_t)j + op->ny * (size_t)(kk + op->nz - 1));
                        const int qq = ncomp == 9 ? map9[q] : q;
                        h[q * plane + ((size_t)zi * Py + j) * Px + i] = make_double2(op->t6[qq][src], 0.0);
                    }
            }
        CK(cudaMemcpy(W.p, h.data(), sizeof(double2) * h.size(), cudaMemcpyHostToDevice));
    }
    CK(mlb::launch_fft3d_d(W.p, ncomp, Px, Py, Pz, P->L, twdd.p, -1, st));
    if (k.general) {
        P->ten9.alloc((size_t)k.Kx * Py * Pz * 9 * 2 * rb);
        CK(mlb::launch_tensor_pack9(W.p, Px, Py, Pz, k.Kx, P->ten9.p, rb, k.split, st));
    } else if ((quarter_ok(k, rb) || (rb == 4 && mlb::yz_col3_ok(k))) && tensor_has_parities(W.p, k, st)) {
        // the split FP32 passes and the single-CTA-plane (y,z) kernel read a
        // quarter of the tensor (ky <= Py/2, kz <= Pz/2)
        k.quarter = 1;
        const size_t q6 = (size_t)(Py / 2 + 1) * (Pz / 2 + 1) * 6;
        const size_t per_kx = k.split ? q6 : ((q6 + 3) & ~(size_t)3);
        P->ten6.alloc((size_t)k.Kx * per_kx * rb);
        CK(cudaMemsetAsync(P->ten6.p, 0, (size_t)k.Kx * per_kx * rb, st));
        CK(mlb::launch_tensor_pack6q(W.p, Px, Py, Pz, k.Kx, reinterpret_cast<float*>(P->ten6.p), k.split ? 0 : 1, st));
    } else {
        P->ten6.alloc((size_t)k.Kx * Py * Pz * 6 * rb);
        DBuf<double> mi;
        mi.alloc(1);
        CK(cudaMemsetAsync(mi.p, 0, sizeof(double), st));
        CK(mlb::launch_tensor_pack6(W.p, Px, Py, Pz, k.Kx, P->ten6.p, mi.p, rb, k.split, st));
        CK(cudaMemcpyAsync(&P->max_imag, mi.p, sizeof(double), cudaMemcpyDeviceToHost, st));
    }
    P->spec.alloc((size_t)k.Kx * 3 * op->nz * op->ny * 2 * rb);
    if (k.split) {
        P->spec2.alloc((size_t)k.Kx * Py * 3 * op->nz * 2 * rb);
        k.spec2 = P->spec2.p;
    }
    CK(cudaStreamSynchronize(st));
    op->plan = std::move(P);
    op->plan_dirty = false;
}

// ------------------------------------------------------------------ LongRange2D / Dipole2D
bool is_lr2d(int kind)
{
    return kind == MLB_OP_LONGRANGE2D || kind == MLB_OP_DIPOLE2D || kind == MLB_OP_MAGNETOSTATICS2D;
}

void ensure_t2(mlb_op* op)
{
    const size_t n = (size_t)op->nz * op->nz * 9 * op->nx * op->ny;
    if (op->t2.size() != n) op->t2.assign(n, 0.0);
}

// Point-dipole tensor elements of the Dipole2D builder (demag.cpp:3-56):
// d2_xx(X, Y, Z) = -(1/r^3 - 3 X X / r^5), d2_xy(X, Y, Z) = 3 X Y / r^5 with
// r = |(X, Y, Z)| summed in argument order, zero at r < 1e-80; the other
// seven elements are these two with permuted arguments.
double d2_xx(double X, double Y, double Z)
{
    const double r = std::sqrt(X * X + Y * Y + Z * Z);
    if (r < 1e-80) return 0.0;
    const double ir = 1.0 / r;
    const double ir3 = ir * ir * ir;
    const double ir5 = ir3 * ir * ir;
    return -1.0 * (ir3 - 3.0 * X * X * ir5);
}
double d2_xy(double X, double Y, double Z)
{
    const double r = std::sqrt(X * X + Y * Y + Z * Z);
    if (r < 1e-80) return 0.0;
    const double ir = 1.0 / r;
    const double ir3 = ir * ir * ir;
    const double ir5 = ir3 * ir * ir;
    return -1.0 * (-3.0 * X * Y * ir5);
}

// Dipole2D makeData (dip2d_luafuncs.lua:540-660): zero every array, then for
// each (dest, src) with |src - dest| <= truncation z and each (X, Y) in the x
// and y truncation ranges add the nine elements of r = p_src - p_dest at
// (X mod nx, Y mod ny), positions from idx2pos (:516-538).  Both positions
// are taken at the same (X, Y), so r is the offset between the layers alone,
// and idx2pos takes the x part of the B step from B's y component; both as
// in the reference.
void dipole2d_make(mlb_op* op)
{
    const int nx = op->nx, ny = op->ny, nz = op->nz;
    ensure_t2(op);
    std::fill(op->t2.begin(), op->t2.end(), 0.0);
    const size_t plane = (size_t)nx * ny;
    auto pos = [&](int i, int j, int layer, double out[3]) {
        double dz[3] = {0, 0, 0};
        for (int Z = 0; Z < layer; Z++)
            for (int c = 0; c < 3; c++) dz[c] = dz[c] + op->d2_abc[Z * 9 + 6 + c];
        const double* A = &op->d2_abc[0];
        const double* B = &op->d2_abc[3];
        const double di[3] = {i * A[0], i * A[1], i * A[2]};
        const double dj[3] = {j * B[1], j * B[1], j * B[2]};
        const double* off = &op->d2_off[layer * 3];
        for (int c = 0; c < 3; c++) out[c] = di[c] + dj[c] + dz[c] + off[c];
    };
    const int tX = op->d2_trunc[1], tY = op->d2_trunc[2], tZ = op->d2_trunc[3];
    for (int d = 0; d < nz; d++)
        for (int sidx = 0; sidx < nz; sidx++) {
            if (std::abs(sidx - d) > tZ) continue;
            double* T = &op->t2[((size_t)d * nz + sidx) * 9 * plane];
            for (int X = -tX; X <= tX; X++)
                for (int Y = -tY; Y <= tY; Y++) {
                    double pd[3], ps[3];
                    pos(X, Y, d, pd);
                    pos(X, Y, sidx, ps);
                    const double rx = ps[0] - pd[0], ry = ps[1] - pd[1], rz = ps[2] - pd[2];
                    int x = X, y = Y;
                    if (x < 0) x += 100000 * nx;
                    if (y < 0) y += 100000 * ny;
                    x %= nx;
                    y %= ny;
                    // NXX NXY NXZ / NYX NYY NYZ / NZX NZY NZZ
                    const double v[9] = {d2_xx(rx, ry, rz), d2_xy(rx, ry, rz), d2_xy(rx, rz, ry),
                                         d2_xy(ry, rx, rz), d2_xx(ry, rx, rz), d2_xy(ry, rz, rx),
                                         d2_xy(rz, rx, ry), d2_xy(rz, ry, rx), d2_xx(rz, rx, ry)};
                    const size_t at = (size_t)y * nx + x;
                    for (int ab = 0; ab < 9; ab++) T[ab * plane + at] += v[ab];
                }
        }
    op->lr2_newdata = false;
    op->lr2_compile = true;
}

// Magnetostatics2D element functions: Newell's f and g (Newell, Williams
// and Dunlop, J. Geophys. Res. 98, 9551 (1993)) written with logarithms,
// log(num/den) and atan2 taken as 0 where the reference's helpers do
// (demag.cpp:190-210), and the 64-term combination for a source prism d1 and
// a destination prism d2 at offset (X, Y, Z) divided by 4 pi |d2|
// (demag.cpp:256-280, after Donahue).
double ms_log(double num, double den) { return (num == 0 || den == 0) ? 0.0 : std::log(num / den); }
double ms_atan(double num, double den) { return (num == 0 && den == 0) ? 0.0 : std::atan2(num, den); }

double ms_f(double X, double Y, double Z)
{
    const double x = std::fabs(X), y = std::fabs(Y), z = std::fabs(Z);
    const double xx = x * x, yy = y * y, zz = z * z;
    const double R = std::sqrt(xx + yy + zz);
    return (2 * xx - yy - zz) * R / 6 - x * y * z * ms_atan(y * z, x * R) +
           (y / 4) * (zz - xx) * ms_log((y + R) * (y + R), xx + zz) +
           (z / 4) * (yy - xx) * ms_log((z + R) * (z + R), xx + yy);
}

double ms_g(double X, double Y, double Z)
{
    const double x = std::fabs(X), y = std::fabs(Y), z = std::fabs(Z);
    const double xx = x * x, yy = y * y, zz = z * z;
    const double R = std::sqrt(xx + yy + zz);
    const double sg = (X < 0 ? -1.0 : 1.0) * (Y < 0 ? -1.0 : 1.0);
    return sg * (-x * y * R / 3 -
                 (z / 2) * (xx * ms_atan(y * z, x * R) + yy * ms_atan(x * z, y * R) + (zz / 3) * ms_atan(x * y, z * R)) +
                 (x * y * z / 2) * ms_log((z + R) * (z + R), xx + yy) +
                 (y / 12) * (3 * zz - yy) * ms_log((x + R) * (x + R), yy + zz) +
                 (x / 12) * (3 * zz - xx) * ms_log((y + R) * (y + R), xx + zz));
}

template <double (*F)(double, double, double)>
double ms_pair(double X, double Y, double Z, const double d1[3], const double d2[3])
{
    const double sg[4] = {1.0, -1.0, 1.0, -1.0};
    const double ox[4] = {0, d2[0], d2[0] - d1[0], -d1[0]};
    const double oy[4] = {0, d2[1], d2[1] - d1[1], -d1[1]};
    const double oz[4] = {0, d2[2], d2[2] - d1[2], -d1[2]};
    double sum = 0;
    for (int a = 0; a < 4; a++)
        for (int b = 0; b < 4; b++)
            for (int c = 0; c < 4; c++) sum = sum + sg[a] * sg[b] * sg[c] * F(X + ox[a], Y + oy[b], Z + oz[c]);
    return sum / (4.0 * M_PI * d2[0] * d2[1] * d2[2]);
}

// The nine elements XX..ZZ at r for source prism d1, destination prism d2
// (demag.cpp:283-350: YY, ZZ, XZ, YZ by permuting axes; YX = XY, ZX = XZ,
// ZY = YZ).
void ms_elements(double rx, double ry, double rz, const double d1[3], const double d2[3], double v[9])
{
    auto P = [](const double* d, int i, int j, int k, double* o) { o[0] = d[i]; o[1] = d[j]; o[2] = d[k]; };
    double a1[3], a2[3];
    const double xx = ms_pair<ms_f>(rx, ry, rz, d1, d2);
    const double xy = ms_pair<ms_g>(rx, ry, rz, d1, d2);
    P(d1, 0, 2, 1, a1); P(d2, 0, 2, 1, a2);
    const double xz = ms_pair<ms_g>(rx, rz, ry, a1, a2);
    P(d1, 1, 0, 2, a1); P(d2, 1, 0, 2, a2);
    const double yy = ms_pair<ms_f>(ry, rx, rz, a1, a2);
    P(d1, 1, 2, 0, a1); P(d2, 1, 2, 0, a2);
    const double yz = ms_pair<ms_g>(ry, rz, rx, a1, a2);
    P(d1, 2, 1, 0, a1); P(d2, 2, 1, 0, a2);
    const double zz = ms_pair<ms_f>(rz, ry, rx, a1, a2);
    v[0] = xx; v[1] = xy; v[2] = xz;
    v[3] = xy; v[4] = yy; v[5] = yz;
    v[6] = xz; v[7] = yz; v[8] = zz;
}

// Magnetostatics2D makeData (mag2d_luafuncs.lua:598-744): zero every array;
// for source layer z1 and destination layer z2 within truncation z, and
// each X, Y in [-truncation, truncation] within the x and y truncations,
// r = X A + Y B + (C_0 + .. + C_{z2-1}) - (C_0 + .. + C_{z1-1}) (A, B of the
// first layer), add -N(r; grain z1, grain z2) at (X mod nx, Y mod ny) of the
// arrays [z1][z2].  The layer pairs run on host threads, each pair's
// accumulation in the reference's order.
void magnetostatics2d_make(mlb_op* op)
{
    const int nx = op->nx, ny = op->ny, nz = op->nz;
    ensure_t2(op);
    std::fill(op->t2.begin(), op->t2.end(), 0.0);
    const size_t plane = (size_t)nx * ny;
    const double* A = &op->d2_abc[0];
    const double* B = &op->d2_abc[3];
    const int mx = op->d2_trunc[0], tX = op->d2_trunc[1], tY = op->d2_trunc[2], tZ = op->d2_trunc[3];
    auto cum = [&](int layer, double c[3]) {
        c[0] = c[1] = c[2] = 0;
        for (int j = 0; j < layer; j++)
            for (int q = 0; q < 3; q++) c[q] = c[q] + op->d2_abc[j * 9 + 6 + q];
    };
    auto pair = [&](int z1, int z2) {
        if (std::abs(z1 - z2) > tZ) return;
        double c1[3], c2[3];
        cum(z1, c1);
        cum(z2, c2);
        const double cx = c2[0] - c1[0], cy = c2[1] - c1[1], cz = c2[2] - c1[2];
        const double* g1 = &op->d2_grain[z1 * 3];
        const double* g2 = &op->d2_grain[z2 * 3];
        double* T = &op->t2[((size_t)z1 * nz + z2) * 9 * plane];
        for (int X = -mx; X <= mx; X++) {
            if (std::abs(X) > tX) continue;
            for (int Y = -mx; Y <= mx; Y++) {
                if (std::abs(Y) > tY) continue;
                const double rx = A[0] * X + B[0] * Y + cx;
                const double ry = A[1] * X + B[1] * Y + cy;
                const double rz = A[2] * X + B[2] * Y + cz;
                int x = X, y = Y;
                while (x < 0) x += 1000 * nx;
                while (y < 0) y += 1000 * ny;
                x %= nx;
                y %= ny;
                double v[9];
                ms_elements(rx, ry, rz, g1, g2, v);
                const size_t at = (size_t)y * nx + x;
                for (int ab = 0; ab < 9; ab++) T[ab * plane + at] += -v[ab];
            }
        }
    };
    const int npair = nz * nz;
    const int nth = std::max(1, std::min<int>(npair, (int)std::thread::hardware_concurrency()));
    std::atomic<int> next(0);
    std::vector<std::thread> pool;
    for (int t = 0; t < nth; t++)
        pool.emplace_back([&] {
            for (int p = next++; p < npair; p = next++) pair(p / nz, p % nz);
        });
    for (auto& th : pool) th.join();
    op->lr2_newdata = false;
    op->lr2_compile = true;
}

// compile (spinoperationlongrange2d.cpp:387-430): 2D transforms of every
// array in FP64 on the GPU, divided by nx ny, stored in the state precision
// rb.  The layer pairs go through a bounded FP64 work buffer in batches.
void build_lr2d(mlb_op* op, cudaStream_t st, int rb)
{
    if (!op->lr2_compile && op->lr2 && op->lr2->rb == rb) return;
    const int nx = op->nx, ny = op->ny, nz = op->nz;
    if (nz > MLB_LR2D_MAXZ) fail(MLB_EUNSUP, "LongRange2D supports at most 64 layers");
    std::unique_ptr<LR2DPlan> P(new LR2DPlan());
    P->rb = rb;
    ConvK& k = P->k;
    memset(&k, 0, sizeof(k));
    k.nx = nx; k.ny = ny; k.nz = nz;
    k.Px = nx; k.Py = ny; k.Pz = 1;
    k.Kx = nx / 2 + 1;
    k.general = 1;
    k.nrep = 1;
    const size_t cb = (size_t)2 * rb;
    int ty = 16;
    while (ty > 1 && (size_t)2 * ty * k.Px * cb > 96 * 1024) ty /= 2;
    k.ty = ty;
    if ((size_t)2 * k.Px * cb > 96 * 1024) fail(MLB_EUNSUP, "x length too large");
    if (mlb::lr2d_smem(k, rb) > 227 * 1024)
        fail(MLB_EUNSUP, "LongRange2D: 3 nz ny spectrum values per kx exceed shared memory at " +
                             std::to_string(8 * rb) + "-bit precision");
    std::vector<float2> twf;
    std::vector<double2> twd;
    const int lens[3] = {nx, ny, 1};
    for (int a = 0; a < 3; a++) {
        P->L[a] = make_len(lens[a], (int)twf.size());
        append_twiddles(twf, lens[a]);
        append_twiddles(twd, lens[a]);
    }
    if (rb == 8) {
        P->tw.alloc(sizeof(double2) * twd.size());
        CK(cudaMemcpy(P->tw.p, twd.data(), sizeof(double2) * twd.size(), cudaMemcpyHostToDevice));
    } else {
        P->tw.alloc(sizeof(float2) * twf.size());
        CK(cudaMemcpy(P->tw.p, twf.data(), sizeof(float2) * twf.size(), cudaMemcpyHostToDevice));
    }
    DBuf<double2> twdd;
    twdd.alloc(twd.size());
    CK(cudaMemcpy(twdd.p, twd.data(), sizeof(double2) * twd.size(), cudaMemcpyHostToDevice));
    ensure_t2(op);
    const size_t plane = (size_t)nx * ny;
    const int npair = nz * nz;
    P->Q.alloc((size_t)k.Kx * ny * npair * 9 * cb);
    // batch of layer pairs whose FP64 transforms fit 256 MB
    int bp = (int)std::max<size_t>(1, ((size_t)256 << 20) / (plane * 9 * sizeof(double2)));
    bp = std::min(bp, npair);
    DBuf<double2> W;
    W.alloc(plane * 9 * bp);
    std::vector<double2> h(plane * 9 * bp);
    for (int p0 = 0; p0 < npair; p0 += bp) {
        const int np = std::min(bp, npair - p0);
        for (size_t i = 0; i < plane * 9 * np; i++) h[i] = make_double2(op->t2[(size_t)p0 * 9 * plane + i], 0.0);
        CK(cudaMemcpyAsync(W.p, h.data(), sizeof(double2) * plane * 9 * np, cudaMemcpyHostToDevice, st));
        CK(mlb::launch_fft3d_d(W.p, 9 * np, nx, ny, 1, P->L, twdd.p, -1, st));
        CK(mlb::launch_lr2d_pack(W.p, nx, ny, nz, p0, np, P->Q.p, rb, st));
        CK(cudaStreamSynchronize(st));
    }
    P->spec.alloc((size_t)k.Kx * 3 * nz * ny * cb);
    if (rb == 4 && mlb::x_fast_ok(k) && mlb::split_y_fast_ok(k)) {
        // FP32 power-of-two planes: y transforms through a second spectrum
        P->spec2.alloc((size_t)k.Kx * ny * 3 * nz * cb);
        P->k.spec2 = P->spec2.p;
    }
    op->lr2 = std::move(P);
    op->lr2_compile = false;
}

// ------------------------------------------------------------------ lazy evaluation
struct TermsBuild {
    TermsK T;
    bool ok = true;
    double dt_sys;
    std::vector<int> conflict_slots;
};

void terms_init(TermsK& T)
{
    memset(&T, 0, sizeof(T));
    T.ex_gs = 1.0;
}

// Add one recorded term to T; false when T already holds a different op
// of the same kind (the fused kernel evaluates one of each).
bool terms_add(TermsK& T, const Term& t, bool th_sub, mlb_system* s, bool capture)
{
    mlb_op* op = t.op;
    switch (op->kind) {
    case MLB_OP_EXCHANGE:
        if (T.ex.mode != EX_NONE) return false;
        T.ex = op->exk;
        T.ex_gs = op->gs * t.weight;
        return true;
    case MLB_OP_ANISOTROPY:
        if (T.ani.mode != ANI_NONE) return false;
        T.ani = op->anik;
        return true;
    case MLB_OP_UNIAXIAL:
        if (T.uni.mode != ANI_NONE) return false;
        T.uni = op->unik;
        return true;
    case MLB_OP_CUBIC:
        if (T.cub.mode != ANI_NONE) return false;
        T.cub = op->cubk;
        return true;
    case MLB_OP_THERMAL:
        if (T.th.mode != TH_NONE || !th_sub) return false;
        T.th.mode = TH_PHILOX;
        T.th.T = t.T * t.gs;
        T.th.scale = op->tscale.empty() ? nullptr : op->dscale.p;
        T.th.seed = op->seed;
        // captured steps read the counter from the device step block
        T.th.counter = capture ? 0 : t.counter;
        T.th.dctr = capture ? &s->dstep[s->cur].th_counter : nullptr;
        return true;
    case MLB_OP_APPLIEDFIELD:
        if (T.zee.on) return false;
        T.zee.on = 1;
        for (int a = 0; a < 3; a++) T.zee.B[a] = t.B[a];
        T.zee.Bdev = capture ? s->dstep[s->cur].B : nullptr;
        return true;
    }
    return false;
}

bool add_addend(TermsK& T, void* const h[3], double w, bool thermal)
{
    if (T.nadd >= MLB_MAX_ADDENDS) return false;
    for (int c = 0; c < 3; c++) T.add[T.nadd][c] = h[c];
    T.addw[T.nadd] = w;
    T.add_is_thermal[T.nadd] = thermal ? 1 : 0;
    T.nadd++;
    return true;
}

void materialize(mlb_system* s, int si);

// Materialise every SUM slot that lists si (before si changes).
void before_mutate(mlb_system* s, int si)
{
    for (size_t j = 0; j < s->slots.size(); j++) {
        Slot& x = s->slots[j];
        if ((int)j != si && x.state == ST_SUM &&
            std::find(x.sum_list.begin(), x.sum_list.end(), si) != x.sum_list.end())
            materialize(s, (int)j);
    }
}

void eval_into(mlb_system* s, int buf, const TermsK& T, double dt_sys, Slot& out, int acc)
{
    slot_alloc(s, out);
    CK(mlb::launch_eval(sysk(s, buf), T, dt_sys, out.h, acc, s->rb, s->st));
}

// Evaluate a LAZY slot into its arrays (state becomes DATA).
void materialize_lazy(mlb_system* s, int si)
{
    Slot& sl = s->slots[si];
    const int buf = buffer_for_gen(s, sl.gen);
    const bool th_sub = name_eq(sl.name, "Thermal");
    // terms one kind at a time so any combination is handled
    slot_alloc(s, sl);
    if (!sl.base_data) {
        for (int c = 0; c < 3; c++) CK(cudaMemsetAsync(sl.h[c], 0, (size_t)s->rb * s->n, s->st));
    }
    for (const Term& t : sl.terms) {
        TermsK T;
        terms_init(T);
        if (!terms_add(T, t, true, s, false)) fail(MLB_ESTATE, "internal: term not representable");
        (void)th_sub;
        eval_into(s, buf, T, t.dt_sys, sl, 1);
    }
    sl.terms.clear();
    sl.state = ST_DATA;
    sl.base_data = false;
}

// Build the terms of a SUM definition over slots in list (weights 1).
// Slots that cannot join (different generation, conflicting kinds, too many
// addends) are materialised first; each retry turns one more slot into DATA.
void build_sum_terms(mlb_system* s, const std::vector<int>& list, TermsK& T, long long& gen, double& dt_sys,
                     bool capture, int thermal_slot)
{
    for (int iter = 0; iter <= (int)s->slots.size() + 1; iter++) {
        terms_init(T);
        gen = s->gen;
        dt_sys = s->dt;
        for (int j : list)
            if (s->slots[j].state == ST_LAZY) { gen = s->slots[j].gen; break; }
        bool restart = false;
        for (int j : list) {
            Slot& x = s->slots[j];
            const bool is_th = j == thermal_slot;
            if (x.state == ST_SUM) {
                if (capture) fail(MLB_ESTATE, "step is not fusable");
                materialize(s, j);
            }
            if (x.state == ST_LAZY) {
                bool ok = x.gen == gen;
                TermsK T2 = T;
                double dts = dt_sys;
                if (ok && x.base_data) ok = add_addend(T2, x.h, 1.0, is_th);
                for (const Term& t : x.terms) {
                    if (!ok) break;
                    const bool th_here = t.op->kind == MLB_OP_THERMAL;
                    if (th_here != is_th) { ok = false; break; }
                    ok = terms_add(T2, t, is_th, s, capture);
                    if (ok && th_here) dts = t.dt_sys;
                }
                if (!ok) {
                    if (capture) fail(MLB_ESTATE, "step is not fusable");
                    materialize(s, j);
                    restart = true;
                    break;
                }
                T = T2;
                dt_sys = dts;
            } else if (x.state == ST_DATA) {
                if (!add_addend(T, x.h, 1.0, is_th)) fail(MLB_EUNSUP, "too many materialised field slots in one sum");
            }
        }
        if (!restart) return;
    }
    fail(MLB_ESTATE, "internal: field sum did not settle");
}

void materialize(mlb_system* s, int si)
{
    Slot& sl = s->slots[si];
    switch (sl.state) {
    case ST_DATA:
        return;
    case ST_ZERO:
        slot_alloc(s, sl);
        for (int c = 0; c < 3; c++) CK(cudaMemsetAsync(sl.h[c], 0, (size_t)s->rb * s->n, s->st));
        sl.state = ST_DATA;
        return;
    case ST_LAZY:
        materialize_lazy(s, si);
        return;
    case ST_SUM: {
        std::vector<int> list = sl.sum_list;
        TermsK T;
        long long gen;
        double dt_sys;
        build_sum_terms(s, list, T, gen, dt_sys, false, slot_find(s, "Thermal"));
        Slot& out = s->slots[si];
        eval_into(s, buffer_for_gen(s, gen), T, dt_sys, out, 0);
        out.state = ST_DATA;
        out.sum_list.clear();
        return;
    }
    }
}

void materialize_all(mlb_system* s)
{
    for (size_t j = 0; j < s->slots.size(); j++)
        if (s->slots[j].state == ST_SUM) materialize(s, (int)j);
    for (size_t j = 0; j < s->slots.size(); j++)
        if (s->slots[j].state == ST_LAZY) materialize(s, (int)j);
}

// Materialise lazy records that depend on generation gen (before its buffer
// is overwritten).
void materialize_gen(mlb_system* s, long long gen)
{
    for (size_t j = 0; j < s->slots.size(); j++) {
        Slot& x = s->slots[j];
        if (x.state == ST_SUM) {
            bool dep = false;
            for (int k : x.sum_list)
                if (s->slots[k].state == ST_LAZY && s->slots[k].gen == gen) dep = true;
            if (dep) materialize(s, (int)j);
        }
    }
    for (size_t j = 0; j < s->slots.size(); j++)
        if (s->slots[j].state == ST_LAZY && s->slots[j].gen == gen) materialize(s, (int)j);
}

// Every lazy record of every system that references op (before op changes).
void materialize_users(mlb_op* op)
{
    for (mlb_system* s : g_systems) {
        bool any = false;
        for (Slot& x : s->slots)
            for (Term& t : x.terms)
                if (t.op == op) any = true;
        if (any) materialize_all(s);
    }
}

// ------------------------------------------------------------------ apply
void check_dims(const mlb_op* op, const mlb_system* s)
{
    if (op->nx != s->nx || op->ny != s->ny || op->nz != s->nz)
        fail(MLB_EINVAL, "operator and SpinSystem sizes differ");
}

// Learned-surrogate hooks (defined with mlb_surrogate below): the operator's
// field for this step from the surrogate or, when the device schedule asks
// for it, the exact convolution; and the end-of-step schedule update.
bool sur_hook(mlb_op* op, mlb_system* s, Slot& sl);
void sur_advance(mlb_system* s);

// Run a deferred inverse x pass on its own (the step took another path).
void flush_pending(mlb_system* s)
{
    if (!s->pend_op) return;
    mlb_op* op = s->pend_op;
    Slot& sl = s->slots[s->pend_si];
    s->pend_op = nullptr;
    s->pend_si = -1;
    ConvPlan& P = *op->plan;
    float* h[3] = {static_cast<float*>(sl.h[0]), static_cast<float*>(sl.h[1]), static_cast<float*>(sl.h[2])};
    CK(mlb::launch_conv_fast_ix(P.k, P.L, reinterpret_cast<const float2*>(P.tw.p), reinterpret_cast<float2*>(P.spec.p),
                                h, s->st));
}

void op_apply(mlb_op* op, mlb_system* s)
{
    check_dims(op, s);
    const int si = slot_register(s, op->slot.c_str());
    if (s->pend_op && (is_conv(op->kind) || is_lr2d(op->kind) || si == s->pend_si)) flush_pending(s);
    before_mutate(s, si);
    Slot& sl = s->slots[si];
    Term t{};
    t.op = op;
    t.weight = 1;
    t.gs = op->gs;
    t.dt_sys = s->dt;
    switch (op->kind) {
    case MLB_OP_EXCHANGE: {
        compile_exchange(op);
        sl.used = true;
        if (op->exk.mode == EX_NONE) {
            if (sl.state == ST_ZERO) { sl.state = ST_ZERO; }
            return;
        }
        if (sl.state == ST_LAZY && sl.gen != s->gen) materialize(s, si);
        if (sl.state == ST_SUM) materialize(s, si);
        if (sl.state == ST_ZERO) {
            sl.state = ST_LAZY; sl.base_data = false; sl.terms.assign(1, t); sl.gen = s->gen;
        } else if (sl.state == ST_DATA) {
            sl.state = ST_LAZY; sl.base_data = true; sl.terms.assign(1, t); sl.gen = s->gen;
        } else {
            bool merged = false;
            for (Term& x : sl.terms)
                if (x.op == op && x.gs == t.gs) { x.weight++; merged = true; }
            if (!merged) sl.terms.push_back(t);
        }
        return;
    }
    case MLB_OP_ANISOTROPY:
    case MLB_OP_UNIAXIAL:
    case MLB_OP_CUBIC:
        compile_aniso(op);
        sl.used = true;
        sl.state = ST_LAZY; sl.base_data = false; sl.terms.assign(1, t); sl.gen = s->gen;
        if (op->asite.empty()) { sl.state = ST_ZERO; sl.terms.clear(); }
        return;
    case MLB_OP_THERMAL: {
        compile_thermal_scale(op);
        sl.used = true;
        t.T = op->T;
        if (op->inject_pending) {
            // injected normals: evaluate now (parity mode)
            TermsK T;
            terms_init(T);
            T.th.mode = TH_INJECT;
            T.th.T = op->T * op->gs;
            T.th.scale = op->tscale.empty() ? nullptr : op->dscale.p;
            T.th.nx = op->inj[0].p; T.th.ny = op->inj[1].p; T.th.nz = op->inj[2].p;
            sl.terms.clear();
            sl.base_data = false;
            eval_into(s, s->cur, T, s->dt, sl, 0);
            sl.state = ST_DATA;
            op->inject_pending = false;
            return;
        }
        t.counter = op->counter++;
        sl.state = ST_LAZY; sl.base_data = false; sl.terms.assign(1, t); sl.gen = s->gen;
        return;
    }
    case MLB_OP_APPLIEDFIELD:
        sl.used = true;
        for (int a = 0; a < 3; a++) t.B[a] = op->B[a] * op->gs;
        sl.state = ST_LAZY; sl.base_data = false; sl.terms.assign(1, t); sl.gen = s->gen;
        return;
    case MLB_OP_LONGRANGE2D:
    case MLB_OP_DIPOLE2D:
    case MLB_OP_MAGNETOSTATICS2D: {
        // apply (spinoperationlongrange2d.cpp:430-530): makeNewData when new
        // data is required, compile when required, then the convolution
        if (op->lr2_newdata) {
            if (s->capturing) fail(MLB_ESTATE, "tensor changed during capture");
            if (op->kind == MLB_OP_DIPOLE2D) dipole2d_make(op);
            else if (op->kind == MLB_OP_MAGNETOSTATICS2D) magnetostatics2d_make(op);
            else fail(MLB_ESTATE, "make data function not set");
        }
        if (s->capturing && (op->lr2_compile || !op->lr2 || op->lr2->rb != s->rb))
            fail(MLB_ESTATE, "tensor changed during capture");
        build_lr2d(op, s->st, s->rb);
        sl.used = true;
        sl.terms.clear();
        sl.base_data = false;
        slot_alloc(s, sl);
        sl.state = ST_DATA;
        if (s->dry) return;
        LR2DPlan& P = *op->lr2;
        LR2DScale sc;
        memset(&sc, 0, sizeof(sc));
        for (int z = 0; z < op->nz; z++) {
            sc.src[z] = op->lr2_src[z];
            sc.dst[z] = op->lr2_dst[z] * op->gs;
        }
        const void* sp[3] = {s->sp[s->cur][0], s->sp[s->cur][1], s->sp[s->cur][2]};
        CK(mlb::launch_lr2d(P.k, P.L, P.tw.p, sp, P.spec.p, P.Q.p, sc, sl.h, s->rb, s->st));
        return;
    }
    case MLB_OP_DIPOLE:
    case MLB_OP_LONGRANGE:
    case MLB_OP_LONGRANGE3D:
    case MLB_OP_MAGNETOSTATIC: {
        if (s->capturing && (op->plan_dirty || !op->plan || op->plan->rb != s->rb))
            fail(MLB_ESTATE, "tensor changed during capture");
        build_plan(op, s->st, s->rb);
        sl.used = true;
        sl.terms.clear();
        sl.base_data = false;
        slot_alloc(s, sl);
        ConvPlan& P = *op->plan;
        P.k.g = op->g * op->gs / ((double)P.k.Px * P.k.Py * P.k.Pz);
        sl.state = ST_DATA;
        if (s->dry) return;
        if (s->sur && sur_hook(op, s, sl)) return;
        if (s->rb == 4 && mlb::conv_fast_ok(P.k)) {
            const float* sp[3] = {static_cast<const float*>(s->sp[s->cur][0]), static_cast<const float*>(s->sp[s->cur][1]),
                                  static_cast<const float*>(s->sp[s->cur][2])};
            float* h[3] = {static_cast<float*>(sl.h[0]), static_cast<float*>(sl.h[1]), static_cast<float*>(sl.h[2])};
            if (s->defer_x && P.k.nrep == 1 && !P.k.general) {
                // forward x pass only when SPEC does not already hold it
                const bool carry = s->capturing ? s->cap_carry
                                                : (s->spec_token != 0 && s->spec_token == P.spec_token);
                ConvK kk = P.k;
                kk.tl = s->capturing ? s->cap_tl : nullptr;
                CK(mlb::launch_conv_fast_fyz(kk, P.L, reinterpret_cast<const float2*>(P.tw.p), sp,
                                             reinterpret_cast<float2*>(P.spec.p),
                                             reinterpret_cast<const float*>(P.ten6.p), !carry, s->st));
                if (!s->capturing) P.spec_token = 0;
                s->pend_op = op;
                s->pend_si = si;
                return;
            }
            if (!s->capturing) P.spec_token = 0;
            CK(mlb::launch_conv_fast(P.k, P.L, reinterpret_cast<const float2*>(P.tw.p), sp,
                                     reinterpret_cast<float2*>(P.spec.p), reinterpret_cast<const float*>(P.ten6.p), h,
                                     s->st));
        } else {
            if (!s->capturing) P.spec_token = 0;
            const void* sp[3] = {s->sp[s->cur][0], s->sp[s->cur][1], s->sp[s->cur][2]};
            CK(mlb::launch_conv(P.k, P.L[0], P.L[1], P.L[2], P.tw.p, sp, P.spec.p, P.ten6.p, P.ten9.p, sl.h, s->rb,
                                s->st));
        }
        sl.state = ST_DATA;
        return;
    }
    }
    fail(MLB_EINVAL, "unknown operator kind");
}

// ------------------------------------------------------------------ llg
LlgK llgk(const mlb_llg* l, double dt, unsigned* status)
{
    LlgK k;
    k.status = status;
    k.type = l->kind == MLB_LLG_QUATERNION ? LLG_QUAT : LLG_CART;
    k.thermal_only_first_term = l->tof;
    k.renorm = l->disable_renorm ? 0 : 1;
    k.precess = l->precess;
    k.damp = l->damp;
    k.dt = dt;
    k.dt_zero = dt == 0.0 ? 1 : 0;
    return k;
}

// Constants of k_fused_fast when every parameter is uniform across sites;
// false sends the step to the general fused kernel.
template <typename R>
bool fast_fused_t(mlb_system* s, const TermsK& T, const mlb_llg* l, double dt, double dt_sys, FastKT<R>& F)
{
    refresh_ms(s);
    if (s->rb != (int)sizeof(R) || !s->ms_uniform || !(s->ms_u > 0.0) || s->sa || s->sg) return false;
    if (T.ex.mode == EX_CSR || T.ani.mode == ANI_CSR || T.uni.mode != ANI_NONE) return false;
    // one uniform cubic axis set alone (no simple anisotropy beside it)
    if (T.cub.mode == ANI_CSR || (T.cub.mode == ANI_UNIFORM && T.ani.mode != ANI_NONE)) return false;
    if (T.th.mode == TH_INJECT || (T.th.mode == TH_PHILOX && T.th.scale)) return false;
    if (T.nadd > 1 || (T.nadd == 1 && T.add_is_thermal[0])) return false;
    const double ms = s->ms_u, a = s->alpha, g = s->gamma;
    memset(&F, 0, sizeof(F));
    F.status = s->status;
    F.nx = s->nx; F.ny = s->ny; F.nz = s->nz;
    F.ex = T.ex.mode == EX_STENCIL;
    if (F.ex) {
        const double den = T.ex.normalize ? ms * ms : ms;
        for (int d = 0; d < 6; d++) F.J[d] = (R)((double)T.ex.J[d] * T.ex_gs / den);
        for (int c = 0; c < 3; c++) F.pbc[c] = T.ex.pbc[c];
    }
    F.ani = T.ani.mode == ANI_UNIFORM ? 1 : 0;
    if (F.ani) {
        for (int c = 0; c < 3; c++) F.axis[c] = (R)T.ani.axis[c];
        F.ani_c = (R)(2.0 * (double)T.ani.K / (ms * ms));
    }
    if (T.cub.mode == ANI_UNIFORM) {
        F.ani = 2;
        for (int q = 0; q < 9; q++) F.cub_n[q] = (R)T.cub.axes[q];
        for (int q = 0; q < 3; q++) F.cub_K[q] = (R)T.cub.K[q];
        F.cub_quirk = T.cub.quirk;
        F.cub_ims = (R)(1.0 / ms);
    }
    F.th = T.th.mode == TH_PHILOX && T.th.T != 0.0 && g > 0;
    if (F.th) {
        F.sigma = (R)std::sqrt((2.0 * a * (double)T.th.T) / (ms * dt_sys * g));
        F.seed = T.th.seed; F.counter = T.th.counter; F.dctr = T.th.dctr;
    }
    if (T.zee.on) {
        for (int c = 0; c < 3; c++) F.B[c] = (R)T.zee.B[c];
        F.Bdev = T.zee.Bdev;
    }
    F.addw = T.nadd == 1 ? (R)T.addw[0] : 0.f;
    F.llg_type = l->kind == MLB_LLG_QUATERNION ? LLG_QUAT : LLG_CART;
    F.tof = l->tof;
    F.renorm = l->disable_renorm ? 0 : 1;
    F.dt_zero = dt == 0.0;
    F.dt = (R)dt;
    F.precess = (R)l->precess;
    F.ms = (R)ms;
    const double gaa = g / (1.0 + a * a);
    if (F.llg_type == LLG_CART) {
        F.c_prec = (R)(l->tof ? l->precess * -gaa : -gaa);
        F.c_damp = (R)(l->tof ? l->damp * (a / ms) * gaa : (a / ms) * gaa);
    } else {
        F.c_damp = (R)(l->tof ? l->damp * a / ms : a / ms);
        F.c_rot = (R)(0.5 * g * dt / (1.0 + a * a));
    }
    return true;
}

bool fast_fused(mlb_system* s, const TermsK& T, const mlb_llg* l, double dt, double dt_sys, FastK& F)
{
    return fast_fused_t<float>(s, T, l, dt, dt_sys, F);
}

// Fused in-place step when Total is lazily defined; returns false when the
// caller must take the general path.
bool llg_fused(mlb_llg* l, mlb_system* s, double dt)
{
    Slot& tot = s->slots[0];
    const int th = slot_find(s, "Thermal");
    std::vector<int> list;
    if (tot.state == ST_SUM) list = tot.sum_list;
    else if (tot.state == ST_DATA) list.push_back(0);
    else if (tot.state == ST_LAZY) return false;
    // records of the previous generation are about to be overwritten
    materialize_gen(s, s->gen - 1);
    TermsK T;
    long long gen;
    double dt_sys;
    // Thermal slot: its field must be subtracted even when not summed
    bool th_in = th >= 0 && std::find(list.begin(), list.end(), th) != list.end();
    if (th >= 0 && !th_in && s->slots[th].state != ST_ZERO) {
        materialize(s, th);
    }
    build_sum_terms(s, list, T, gen, dt_sys, s->capturing, th);
    if (gen != s->gen) {
        if (s->capturing) fail(MLB_ESTATE, "step is not fusable");
        flush_pending(s);
        return false;
    }
    if (th >= 0 && !th_in && s->slots[th].state == ST_DATA) {
        if (!add_addend(T, s->slots[th].h, 0.0, true)) {
            flush_pending(s);
            return false;
        }
    }
    const int nb = 1 - s->cur;
    if (!s->dry) nm_guard(s, nb);
    FastK F;
    FastKT<double> Fd;
    bool carried = false;   // SPEC ends holding the new spins' x transform
    bool advanced = false;  // a kernel of the step wrote the next step's block
    if (s->dry) {
        // bookkeeping only: the kernels of this step ran in a captured graph
    } else if (fast_fused(s, T, l, dt, dt_sys, F)) {
        const float* sp[3];
        const float* ad[3] = {nullptr, nullptr, nullptr};
        float* out[3];
        for (int c = 0; c < 3; c++) {
            sp[c] = static_cast<const float*>(s->sp[s->cur][c]);
            out[c] = static_cast<float*>(s->sp[nb][c]);
            if (T.nadd == 1) ad[c] = static_cast<const float*>(T.add[0][c]);
        }
        ConvPlan* CP = s->pend_op ? s->pend_op->plan.get() : nullptr;
        mlb_op* pend_op_was = s->pend_op;
        if (CP && T.nadd == 1 && T.add[0][0] == s->slots[s->pend_si].h[0] && mlb::xstep_ok(CP->k, F)) {
            float* h[3] = {static_cast<float*>(s->slots[s->pend_si].h[0]),
                           static_cast<float*>(s->slots[s->pend_si].h[1]),
                           static_cast<float*>(s->slots[s->pend_si].h[2])};
            s->pend_op = nullptr;
            s->pend_si = -1;
            ConvK kx = CP->k;
            kx.tl = s->capturing ? s->cap_tl : nullptr;
            if (s->capturing) {
                F.adv_cur = s->dstep + s->cur;
                F.adv_next = s->dstep + (1 - s->cur);
                advanced = true;
            }
            CK(mlb::launch_xstep(kx, CP->L, reinterpret_cast<const float2*>(CP->tw.p),
                                 reinterpret_cast<float2*>(CP->spec.p), F, true, sp, h, out, s->st));
            carried = true;
            if (s->capturing) {
                s->cap_xstep = pend_op_was;
            } else {
                CP->spec_token = ++g_spec_token;
                s->spec_token = CP->spec_token;
            }
        } else {
            flush_pending(s);
            CK(mlb::launch_fused_fast(F, sp, ad, out, s->st));
        }
    } else if (s->rb == 8 && fast_fused_t<double>(s, T, l, dt, dt_sys, Fd)) {
        // FP64 state with uniform parameters: the fast kernel in double
        flush_pending(s);
        const double* sp[3];
        const double* ad[3] = {nullptr, nullptr, nullptr};
        double* out[3];
        for (int c = 0; c < 3; c++) {
            sp[c] = static_cast<const double*>(s->sp[s->cur][c]);
            out[c] = static_cast<double*>(s->sp[nb][c]);
            if (T.nadd == 1) ad[c] = static_cast<const double*>(T.add[0][c]);
        }
        CK(mlb::launch_fused_fast_f64(Fd, sp, ad, out, s->st));
    } else {
        flush_pending(s);
        FusedK P;
        P.sys = sysk(s, s->cur);
        P.terms = T;
        P.llg = llgk(l, dt, s->status);
        P.ox = s->sp[nb][0]; P.oy = s->sp[nb][1]; P.oz = s->sp[nb][2];
        CK(mlb::launch_fused(P, dt_sys, s->rb, s->st));
    }
    if (s->capturing && !advanced) CK(mlb::launch_advance_step(s->dstep + s->cur, s->dstep + (1 - s->cur), s->st));
    if (!carried && !s->capturing && !s->dry) s->spec_token = 0;
    s->cur = nb;
    s->gen++;
    return true;
}

void llg_apply(mlb_llg* l, mlb_system* from, double scale, mlb_system* dmdt, mlb_system* to, int advance)
{
    if (from->nx != dmdt->nx || from->nx != to->nx || from->ny != dmdt->ny || from->ny != to->ny ||
        from->nz != dmdt->nz || from->nz != to->nz)
        fail(MLB_EINVAL, "SpinSystems of different sizes");
    if (from->rb != dmdt->rb || from->rb != to->rb) fail(MLB_EINVAL, "SpinSystems of different precisions");
    const double dt = scale * dmdt->dt;
    const bool cart = l->kind != MLB_LLG_QUATERNION;
    bool done = false;
    if (from == dmdt && dmdt == to) done = llg_fused(l, from, dt);
    from->last_fused = done;
    if (!done) {
        flush_pending(from);
        if (dmdt != from) flush_pending(dmdt);
        if (to != from && to != dmdt) flush_pending(to);
        if (from->capturing) fail(MLB_ESTATE, "step is not fusable");
        to->spec_token = 0;
        materialize(dmdt, 0);
        const int th = slot_find(dmdt, "Thermal");
        if (th >= 0) materialize(dmdt, th);
        // the destination's spins change in place: settle its lazy fields
        // (an internal system's old fields are never read: drop them)
        if (to->internal) {
            for (Slot& x : to->slots)
                if (x.state == ST_LAZY || x.state == ST_SUM) {
                    x.state = ST_ZERO;
                    x.terms.clear();
                    x.sum_list.clear();
                }
        } else {
            materialize_all(to);
        }
        if (to != dmdt) { materialize(dmdt, 0); if (th >= 0) materialize(dmdt, th); }
        if (from != to && !(cart && dt == 0.0) && to->ms_token != from->ms_token) {
            // the new spins carry the source's magnitudes (skipped when the
            // destination already holds them, e.g. the copies of RK stages)
            CK(cudaMemcpyAsync(to->ms, from->ms, (size_t)from->rb * from->n, cudaMemcpyDeviceToDevice, to->st));
            to->ms_host = from->ms_host;
            to->ms_dirty = true;
            to->ms_token = from->ms_token;
        }
        if (from->st != to->st || dmdt->st != to->st) {
            CK(cudaStreamSynchronize(from->st));
            CK(cudaStreamSynchronize(dmdt->st));
        }
        const void* m[3] = {dmdt->sp[dmdt->cur][0], dmdt->sp[dmdt->cur][1], dmdt->sp[dmdt->cur][2]};
        const void* H[3] = {dmdt->slots[0].h[0], dmdt->slots[0].h[1], dmdt->slots[0].h[2]};
        const void* Ht[3] = {nullptr, nullptr, nullptr};
        if (th >= 0) for (int c = 0; c < 3; c++) Ht[c] = dmdt->slots[th].h[c];
        void* out[3] = {to->sp[to->cur][0], to->sp[to->cur][1], to->sp[to->cur][2]};
        nm_guard(to, to->cur);
        CK(mlb::launch_llg(sysk(from, from->cur), m, H, Ht, dmdt->sa, dmdt->sg, dmdt->alpha, dmdt->gamma,
                           llgk(l, dt, to->status), out, to->rb, to->st));
    }
    if (cart) {
        if (dt != 0.0 && advance) to->time = from->time + dt;
    } else if (advance) {
        to->time = from->time + dt;
    }
    // an attached surrogate's device schedule advances with every step of
    // its system, whether issued by do_step or as individual calls
    if (to->sur && !to->dry) sur_advance(to);
}

void sum_fields(mlb_system* s)
{
    Slot& tot = s->slots[0];
    std::vector<int> list;
    for (size_t j = 1; j < s->slots.size(); j++)
        if (s->slots[j].used) list.push_back((int)j);
    tot.terms.clear();
    tot.base_data = false;
    tot.sum_list = list;
    tot.state = list.empty() ? ST_ZERO : ST_SUM;
}

void reset_fields(mlb_system* s)
{
    for (Slot& x : s->slots) {
        x.used = false;
        x.state = ST_ZERO;
        x.terms.clear();
        x.sum_list.clear();
        x.base_data = false;
    }
}

// Before the system's stream writes spin buffer q (q < 0: either buffer):
// the stream waits for the side-stream netMoment reads of that buffer.
void nm_guard(mlb_system* s, int q)
{
    if (s->capturing) return;   // a captured step is guarded where its graph is launched
    for (int k = 0; k < 4; k++)
        if (s->nm_reading[k] && (q < 0 || s->nm_buf[k] == q)) {
            CK(cudaStreamWaitEvent(s->st, s->nm_ev[k], 0));
            s->nm_reading[k] = false;
        }
}

void spins_changing(mlb_system* s)
{
    // lazy records read the current buffer, which is about to change
    nm_guard(s, -1);
    flush_pending(s);
    materialize_all(s);
    s->spec_token = 0;
}

// A write of the current spin buffer alone (moment magnitudes and site
// arrays kept): only the records that read that buffer (the current
// generation) are settled; those of the previous generation read the other
// buffer, which the write leaves as it is.
void current_spins_changing(mlb_system* s)
{
    nm_guard(s, s->cur);
    flush_pending(s);
    auto reads_current = [&](const Slot& x) { return x.state == ST_LAZY && x.gen == s->gen; };
    for (size_t j = 0; j < s->slots.size(); j++) {
        if (s->slots[j].state != ST_SUM) continue;
        bool cur = false;
        for (int m : s->slots[j].sum_list)
            if (reads_current(s->slots[m])) cur = true;
        if (cur) materialize(s, (int)j);
    }
    for (size_t j = 0; j < s->slots.size(); j++)
        if (reads_current(s->slots[j])) materialize(s, (int)j);
    s->spec_token = 0;
}

mlb_system* make_system(int nx, int ny, int nz, int rb)
{
    if (rb != 4 && rb != 8) fail(MLB_EINVAL, "bytes per real must be 4 or 8");
    if (nx < 1 || ny < 1 || nz < 1) fail(MLB_EINVAL, "dimensions must be positive");
    const long long n = (long long)nx * ny * nz;
    if (n > (1LL << 31) - 1) fail(MLB_EUNSUP, "more than 2^31-1 sites");
    std::unique_ptr<mlb_system> s(new mlb_system());
    s->nx = nx; s->ny = ny; s->nz = nz; s->n = (int)n;
    s->rb = rb;
    CK(cudaStreamCreateWithFlags(&s->own, cudaStreamNonBlocking));
    s->st = s->own;
    for (int b = 0; b < 2; b++)
        for (int c = 0; c < 3; c++) {
            CK(cudaMalloc(&s->sp[b][c], (size_t)rb * n));
            CK(cudaMemset(s->sp[b][c], 0, (size_t)rb * n));
        }
    CK(cudaMalloc(&s->ms, (size_t)rb * n));
    CK(cudaMemset(s->ms, 0, (size_t)rb * n));
    s->ms_host.assign(n, 0.0);
    s->ms_dirty = true;
    s->ms_token = ++g_ms_token;
    CK(cudaMalloc(&s->dstep, 2 * sizeof(DevStep)));
    CK(cudaMemset(s->dstep, 0, 2 * sizeof(DevStep)));
    CK(cudaMalloc(&s->status, sizeof(unsigned)));
    CK(cudaMemset(s->status, 0, sizeof(unsigned)));
    CK(cudaMallocHost(&s->nm_host, sizeof(double) * 30));
    // pinned memory is mapped for the device under unified addressing; the
    // call fails (host side) where it is not
    CK(cudaHostGetDevicePointer((void**)&s->nm_host_dev, s->nm_host, 0));
    CK(cudaMalloc(&s->nm_counter, sizeof(unsigned)));
    CK(cudaMemset(s->nm_counter, 0, sizeof(unsigned)));
    s->red_nb = (int)std::min<long long>(1024, std::max<long long>(1, (n + 255) / 256));
    CK(cudaMalloc(&s->red, sizeof(double) * 6 * s->red_nb));
    CK(cudaMalloc(&s->redout, sizeof(double) * 8));
    CK(cudaMalloc(&s->red_a, sizeof(double) * 6 * s->red_nb));
    CK(cudaMalloc(&s->redout_a, sizeof(double) * 8));
    CK(cudaMalloc(&s->nm_counter_a, sizeof(unsigned)));
    CK(cudaMemset(s->nm_counter_a, 0, sizeof(unsigned)));
    slot_register(s.get(), "Total");
    mlb_system* r = s.release();
    g_systems.insert(r);
    return r;
}

void free_system(mlb_system* s)
{
    if (!s) return;
    g_systems.erase(s);
    cudaStreamSynchronize(s->st);
    for (int b = 0; b < 2; b++)
        for (int c = 0; c < 3; c++) cudaFree(s->sp[b][c]);
    cudaFree(s->ms);
    cudaFree(s->sa);
    cudaFree(s->sg);
    cudaFree(s->dstep);
    cudaFree(s->status);
    for (int q = 0; q < 2; q++)
        for (int d = 0; d < 5; d++)
            if (s->nm_exec[q][d]) cudaGraphExecDestroy(s->nm_exec[q][d]);
    if (s->nm_st) cudaStreamSynchronize(s->nm_st);
    for (int k = 0; k < 4; k++) {
        if (s->nm_ev[k]) cudaEventDestroy(s->nm_ev[k]);
        if (s->nm_go[k]) cudaEventDestroy(s->nm_go[k]);
    }
    if (s->nm_st) cudaStreamDestroy(s->nm_st);
    cudaFreeHost(s->nm_host);
    cudaFree(s->nm_counter);
    cudaFree(s->red);
    cudaFree(s->redout);
    cudaFree(s->nm_counter_a);
    cudaFree(s->red_a);
    cudaFree(s->redout_a);
    for (Slot& x : s->slots)
        for (int c = 0; c < 3; c++) cudaFree(x.h[c]);
    if (s->own) cudaStreamDestroy(s->own);
    delete s;
}

void upload_site_array(mlb_system* s, void** dst, const double* a)
{
    spins_changing(s);
    if (!a) {
        if (*dst) { CK(cudaStreamSynchronize(s->st)); cudaFree(*dst); }
        *dst = nullptr;
        return;
    }
    if (!*dst) CK(cudaMalloc(dst, (size_t)s->rb * s->n));
    put_reals(s, *dst, a, s->n);
    CK(cudaStreamSynchronize(s->st));
}

// The canonical script step.  Nothing outside runs between its calls, so the
// inverse x pass of a fast-path convolution may wait for the LLG update
// (defer_x) and run fused with it.
// copySpinsFrom (spinsystem.cpp:393-409): spins and moment magnitudes.
void copy_spins(mlb_system* dst, mlb_system* src)
{
    if (dst == src) return;
    const size_t bytes = (size_t)src->rb * src->n;
    spins_changing(dst);
    if (src->st != dst->st) CK(cudaStreamSynchronize(src->st));
    for (int c = 0; c < 3; c++)
        CK(cudaMemcpyAsync(dst->sp[dst->cur][c], src->sp[src->cur][c], bytes, cudaMemcpyDeviceToDevice, dst->st));
    if (dst->ms_token != src->ms_token) {
        CK(cudaMemcpyAsync(dst->ms, src->ms, bytes, cudaMemcpyDeviceToDevice, dst->st));
        dst->ms_host = src->ms_host;
        dst->ms_dirty = true;
        dst->ms_token = src->ms_token;
    }
}

// SpinSystem::diff (spinsystem.cpp:301-307): sum_i |a_i - b_i| per component
// and the length of that vector, FP64 on the device.
void system_diff(mlb_system* a, mlb_system* b, double out4[4])
{
    if (a->nx != b->nx || a->ny != b->ny || a->nz != b->nz) fail(MLB_EINVAL, "size mismatch");
    if (a->rb != b->rb) fail(MLB_EINVAL, "precision mismatch");
    if (a->st != b->st) CK(cudaStreamSynchronize(b->st));
    const void* pa[3] = {a->sp[a->cur][0], a->sp[a->cur][1], a->sp[a->cur][2]};
    const void* pb[3] = {b->sp[b->cur][0], b->sp[b->cur][1], b->sp[b->cur][2]};
    CK(mlb::launch_diff(pa, pb, a->n, a->red, a->red_nb, a->redout, a->rb, a->st));
    double r[3];
    CK(cudaMemcpyAsync(r, a->redout, sizeof(r), cudaMemcpyDeviceToHost, a->st));
    CK(cudaStreamSynchronize(a->st));
    out4[0] = r[0]; out4[1] = r[1]; out4[2] = r[2];
    out4[3] = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
}

void do_step(mlb_system* s, mlb_op* const* ops, int nops, mlb_llg* l)
{
    reset_fields(s);
    s->defer_x = true;
    try {
        for (int i = 0; i < nops; i++) op_apply(ops[i], s);
        sum_fields(s);
        llg_apply(l, s, 1.0, s, s, 1);
    } catch (...) {
        s->defer_x = false;
        try {
            flush_pending(s);
        } catch (...) {
            s->pend_op = nullptr;
            s->pend_si = -1;
        }
        throw;
    }
    s->defer_x = false;
    flush_pending(s);
}

void advance_sweep(mlb_op* const* ops, int nops)
{
    for (int i = 0; i < nops; i++)
        if (ops[i]->kind == MLB_OP_APPLIEDFIELD)
            for (int a = 0; a < 3; a++) ops[i]->B[a] += ops[i]->dB[a];
}

struct HostState {
    int cur;
    long long gen;
    double time;
    std::vector<Slot> slots;
    std::vector<uint64_t> ctr;
    std::vector<std::array<double, 3>> B;
    bool last_fused;
};

HostState save_state(mlb_system* s, const std::vector<mlb_op*>& ops)
{
    HostState h;
    h.cur = s->cur; h.gen = s->gen; h.time = s->time; h.slots = s->slots; h.last_fused = s->last_fused;
    for (mlb_op* o : ops) {
        h.ctr.push_back(o->counter);
        h.B.push_back({o->B[0], o->B[1], o->B[2]});
    }
    return h;
}

// Restore the bookkeeping saved by save_state.  Slot registrations and
// their device arrays made in between are kept (new slots return to ZERO).
void load_state(mlb_system* s, const std::vector<mlb_op*>& ops, const HostState& h)
{
    s->cur = h.cur; s->gen = h.gen; s->time = h.time; s->last_fused = h.last_fused;
    for (size_t i = 0; i < s->slots.size(); i++) {
        Slot& x = s->slots[i];
        void* keep[3] = {x.h[0], x.h[1], x.h[2]};
        if (i < h.slots.size()) {
            const bool had = h.slots[i].h[0] != nullptr;
            x = h.slots[i];
            // an array allocated since then stays; a DATA state needs the
            // array it had
            if (!had) for (int c = 0; c < 3; c++) x.h[c] = keep[c];
        } else {
            x.used = false; x.state = ST_ZERO; x.terms.clear(); x.sum_list.clear(); x.base_data = false;
        }
    }
    for (size_t i = 0; i < ops.size(); i++) {
        ops[i]->counter = h.ctr[i];
        for (int a = 0; a < 3; a++) ops[i]->B[a] = h.B[i][a];
    }
}

// the device timeline's stamps back to (earliest = all ones, latest = 0)
void plan_timeline_reset(mlb_plan* p)
{
    const unsigned long long init[4] = {~0ull, 0ull, ~0ull, 0ull};
    CK(cudaMemcpy(p->tl.p, init, sizeof(init), cudaMemcpyHostToDevice));
}

void plan_release(mlb_plan* p)
{
    for (int q = 0; q < 2; q++) {
        if (p->multi[q]) cudaGraphExecDestroy(p->multi[q]);
        p->multi[q] = nullptr;
    }
    for (int q = 0; q < 4; q++) {
        if (p->exec[q]) cudaGraphExecDestroy(p->exec[q]);
        p->exec[q] = nullptr;
        for (ProfCaptured& r : p->ev[q]) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
        p->ev[q].clear();
    }
    p->last = nullptr;
}

// Capture one step for each spin-buffer parity.  A dry pass first runs the
// host logic (compiling operators, building tensor spectra, allocating
// slots) so that the captured pass only enqueues kernels.
void plan_capture(mlb_plan* p)
{
    mlb_system* s = p->s;
    const int nops = (int)p->ops.size();
    for (mlb_op* o : p->ops) {
        check_dims(o, s);
        if (o->kind == MLB_OP_THERMAL && o->inject_pending) fail(MLB_ESTATE, "injected noise cannot be replayed");
    }
    int nth = 0, nz = 0;
    for (mlb_op* o : p->ops) { nth += o->kind == MLB_OP_THERMAL; nz += o->kind == MLB_OP_APPLIEDFIELD; }
    if (nth > 1 || nz > 1) fail(MLB_ESTATE, "a captured step holds at most one Thermal and one AppliedField");
    plan_release(p);
    nm_guard(s, -1);
    const HostState h0 = save_state(s, p->ops);
    try {
        s->dry = true;
        do_step(s, p->ops.data(), nops, p->l);
        s->dry = false;
        if (!s->last_fused) fail(MLB_ESTATE, "step is not fusable");
        load_state(s, p->ops, h0);
        CK(cudaStreamSynchronize(s->st));
        p->carry_op = nullptr;
        for (int q = 0; q < 4; q++) {
            if (q >= 2 && !p->carry_op) break;   // no fused x pass: no carried variant
            s->cur = q & 1;
            s->cap_carry = q >= 2;
            cudaGraph_t graph = nullptr;
            CK(cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal));
            s->capturing = true;
            s->cap_xstep = nullptr;
            s->cap_tl = p->timeline ? p->tl.p : nullptr;
            if (p->timing) mlb::prof_set_capture_sink(&p->ev[q]);
            bool ok = true;
            std::string why;
            try {
                do_step(s, p->ops.data(), nops, p->l);
            } catch (Err& e) {
                ok = false;
                why = e.msg;
            }
            mlb::prof_set_capture_sink(nullptr);
            s->capturing = false;
            s->cap_carry = false;
            s->cap_tl = nullptr;
            if (q < 2) {
                // the carried variants exist only when both parities end in the fused x pass
                if (q == 0) p->carry_op = s->cap_xstep;
                else if (p->carry_op != s->cap_xstep) p->carry_op = nullptr;
            }
            cudaError_t e = cudaStreamEndCapture(s->st, &graph);
            if (!ok || e != cudaSuccess) {
                if (graph) cudaGraphDestroy(graph);
                cudaGetLastError();
                fail(MLB_ESTATE, "step capture failed: " + (ok ? std::string(cudaGetErrorString(e)) : why));
            }
            e = cudaGraphInstantiate(&p->exec[q], graph, 0);
            cudaGraphDestroy(graph);
            if (e != cudaSuccess) fail(MLB_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
            load_state(s, p->ops, h0);
        }
        // kMultiSteps carried steps in one graph: the host logic of the steps
        // runs one after the other while the stream is captured, so the
        // graph holds the single-step graphs' kernels in sequence with the
        // dependent-launch edges kept across the step boundaries (the next
        // step's first pass is scheduled while the last one drains).  A step
        // that does not end in the fused x pass leaves the plan without it.
        if (p->carry_op && !p->timing && !p->timeline) {
            for (int q = 0; q < 2; q++) {
                s->cur = q;
                cudaGraph_t graph = nullptr;
                CK(cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal));
                s->capturing = true;
                bool ok = true;
                try {
                    for (int j = 0; j < kMultiSteps && ok; j++) {
                        s->cap_carry = true;
                        s->cap_xstep = nullptr;
                        do_step(s, p->ops.data(), nops, p->l);
                        ok = s->cap_xstep == p->carry_op;
                        advance_sweep(p->ops.data(), nops);
                    }
                } catch (Err&) {
                    ok = false;
                }
                s->capturing = false;
                s->cap_carry = false;
                cudaError_t e = cudaStreamEndCapture(s->st, &graph);
                if (ok && e == cudaSuccess) e = cudaGraphInstantiate(&p->multi[q], graph, 0);
                if (graph) cudaGraphDestroy(graph);
                if (!ok || e != cudaSuccess) {
                    cudaGetLastError();
                    p->multi[q] = nullptr;
                }
                load_state(s, p->ops, h0);
            }
            if (!p->multi[0] || !p->multi[1]) {
                for (int q = 0; q < 2; q++) {
                    if (p->multi[q]) cudaGraphExecDestroy(p->multi[q]);
                    p->multi[q] = nullptr;
                }
            }
        }
    } catch (...) {
        s->dry = false;
        s->capturing = false;
        s->cap_carry = false;
        s->cap_tl = nullptr;
        mlb::prof_set_capture_sink(nullptr);
        load_state(s, p->ops, h0);
        throw;
    }
    p->version = g_version;
}

void advance_host(mlb_plan* p)
{
    mlb_system* s = p->s;
    const double dt = s->dt;
    for (mlb_op* o : p->ops)
        if (o->kind == MLB_OP_THERMAL) o->counter++;
    s->cur = 1 - s->cur;
    s->gen++;
    const bool cart = p->l->kind != MLB_LLG_QUATERNION;
    if (!cart || dt != 0.0) s->time = s->time + dt;
}

// nsteps captured steps; the host state and lazy field records end as after
// nsteps canonical script steps.
void plan_launch(mlb_plan* p, int nsteps)
{
    if (nsteps <= 0) return;
    mlb_system* s = p->s;
    if (p->version != g_version) plan_capture(p);
    DevStep h;
    memset(&h, 0, sizeof(h));
    for (mlb_op* o : p->ops) {
        if (o->kind == MLB_OP_THERMAL) h.th_counter = o->counter;
        if (o->kind == MLB_OP_APPLIEDFIELD)
            for (int a = 0; a < 3; a++) { h.B[a] = o->B[a] * o->gs; h.dB[a] = o->dB[a] * o->gs; }
    }
    // upload only what the device block does not already hold (consecutive
    // launches: the steps advanced it exactly as the host mirror below)
    if (!s->dstep_known || s->dstep_cur != s->cur || memcmp(&h, &s->dstep_mirror, sizeof(h)) != 0) {
        // (a pageable source is staged before cudaMemcpyAsync returns)
        CK(cudaMemcpyAsync(s->dstep + s->cur, &h, sizeof(h), cudaMemcpyHostToDevice, s->st));
        s->dstep_mirror = h;
    }
    // each step writes the next step's block (the fused x pass, or
    // k_advance_step)
    for (int k = 0; k < nsteps; k++) {
        s->dstep_mirror.th_counter += 1ull;
        for (int a = 0; a < 3; a++) s->dstep_mirror.B[a] += s->dstep_mirror.dB[a];
    }
    s->dstep_known = true;
    ConvPlan* CP = p->carry_op ? p->carry_op->plan.get() : nullptr;
    for (int k = 0; k < nsteps; k++) {
        const bool carry = CP && s->spec_token != 0 && s->spec_token == CP->spec_token;
        if (carry && p->multi[s->cur] && nsteps - k >= kMultiSteps) {
            // kMultiSteps carried steps in one launch; they write both spin
            // buffers
            nm_guard(s, -1);
            CK(cudaGraphLaunch(p->multi[s->cur], s->st));
            p->last = nullptr;
            for (int j = 0; j < kMultiSteps; j++, k++) {
                CP->spec_token = ++g_spec_token;
                s->spec_token = CP->spec_token;
                if (k < nsteps - 1) {
                    advance_host(p);
                    advance_sweep(p->ops.data(), (int)p->ops.size());
                }
            }
            k--;   // the loop's increment
            continue;
        }
        const int gi = s->cur + (carry ? 2 : 0);
        nm_guard(s, 1 - s->cur);   // the step writes the other spin buffer
        CK(cudaGraphLaunch(p->exec[gi], s->st));
        p->last = &p->ev[gi];
        if (CP) {
            // the step's fused x pass left SPEC holding the new spins' transform
            CP->spec_token = ++g_spec_token;
            s->spec_token = CP->spec_token;
        }
        if (k < nsteps - 1) {
            advance_host(p);
            advance_sweep(p->ops.data(), (int)p->ops.size());
        }
    }
    // the last step once more without launching: lazy field records
    s->dry = true;
    try {
        do_step(s, p->ops.data(), (int)p->ops.size(), p->l);
    } catch (...) {
        s->dry = false;
        throw;
    }
    s->dry = false;
    advance_sweep(p->ops.data(), (int)p->ops.size());
    s->dstep_cur = s->cur;   // the block the next step reads
}

// ------------------------------------------------------------------ packed ensembles
struct EnsClass {
    int nx, ny, nz, nrep;
    long long base;             // first packed site of the class
    mlb_op* dip = nullptr;      // tensor spectrum holder for this size
    bool fast = true;           // power-of-two fast passes (else the generic ones, replica by replica)
    int yz_variant = 0;         // tuned (y,z) pass of the fast path (ConvK::yz_variant)
    cudaStream_t st = nullptr;  // branch of the captured step
    cudaEvent_t done = nullptr;
};

void ens_free_graphs(mlb_ensemble* e);

} // namespace

struct mlb_ensemble {
    int nrep = 0;
    long long ntot = 0;
    std::vector<int> pos;            // user replica -> packed replica index
    std::vector<int4> rinfo_h;       // packed order: {nx, ny, nz, first site}
    std::vector<EnsClass> cls;
    float* sp[2][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};
    int cur = 0;
    float* H[3] = {nullptr, nullptr, nullptr};
    float ms = 0.f;
    bool have_ms = false;
    mlb_ensemble_cfg cfg;
    bool configured = false;
    DevStep* dstep = nullptr;
    cudaStream_t st = nullptr, own = nullptr;
    cudaEvent_t fork = nullptr;
    int4* rinfo = nullptr;
    int* brep = nullptr;
    int* bstart = nullptr;
    int nblk = 0;
    int bs = 0;                       // fused-kernel tile size (autotuned)
    int grid = 0;                     // fused-kernel CTAs (autotuned; < nblk: persistent)
    bool tuned = false;
    std::string tune_log;
    cudaGraphExec_t exec[2] = {nullptr, nullptr};
    double time = 0.0;
    uint64_t counter = 0;
    // per packed replica: temperature, applied field at the next step and
    // its per-step sweep (host values); device: field ping-pong by spin
    // buffer, sweep, thermal deviation
    std::vector<double> rT, rB, rdB;
    double* d_rB[2] = {nullptr, nullptr};
    double* d_rdB = nullptr;
    float* d_rsig = nullptr;
    bool rpar_dirty = true;
    double* mom = nullptr;
    unsigned* status = nullptr;       // device status word (bit 0: a non-finite spin)
};

namespace {

struct EnsTune {
    int bs = 256, grid = 0;
    std::vector<int> yz;   // per class
};
std::map<std::string, EnsTune> g_ens_tuned;   // tuning key -> choices (this process)
std::mutex g_ens_tune_mu;

void ens_free_graphs(mlb_ensemble* e)
{
    for (int q = 0; q < 2; q++) {
        if (e->exec[q]) cudaGraphExecDestroy(e->exec[q]);
        e->exec[q] = nullptr;
    }
}

void ens_block_table(mlb_ensemble* e, int bs)
{
    std::vector<int> br, bstv;
    for (int r = 0; r < e->nrep; r++) {
        const int4 ri = e->rinfo_h[r];
        const int n = ri.x * ri.y * ri.z;
        for (int s0 = 0; s0 < n; s0 += bs) { br.push_back(r); bstv.push_back(s0); }
    }
    cudaFree(e->brep);
    cudaFree(e->bstart);
    e->brep = nullptr; e->bstart = nullptr;
    CK(cudaMalloc(&e->brep, sizeof(int) * br.size()));
    CK(cudaMalloc(&e->bstart, sizeof(int) * br.size()));
    CK(cudaMemcpy(e->brep, br.data(), sizeof(int) * br.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(e->bstart, bstv.data(), sizeof(int) * bstv.size(), cudaMemcpyHostToDevice));
    e->nblk = (int)br.size();
    e->bs = bs;
}

bool ens_thermal(const mlb_ensemble* e)
{
    if (!(e->cfg.gamma > 0)) return false;
    for (double T : e->rT)
        if (T != 0.0) return true;
    return false;
}

// Device copies of the per-replica parameters (the field goes to the buffer
// the next step reads: the one of the current spin buffer).
void ens_upload_params(mlb_ensemble* e)
{
    if (!e->rpar_dirty) return;
    const int n = e->nrep;
    const mlb_ensemble_cfg& c = e->cfg;
    std::vector<float> sig(n, 0.f);
    for (int r = 0; r < n; r++)
        if (e->rT[r] != 0.0 && c.gamma > 0)
            sig[r] = (float)std::sqrt((2.0 * c.alpha * e->rT[r]) / (e->ms * c.dt * c.gamma));
    CK(cudaStreamSynchronize(e->st));
    CK(cudaMemcpy(e->d_rB[e->cur], e->rB.data(), sizeof(double) * 3 * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(e->d_rdB, e->rdB.data(), sizeof(double) * 3 * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(e->d_rsig, sig.data(), sizeof(float) * n, cudaMemcpyHostToDevice));
    e->rpar_dirty = false;
}

// The host's view of the per-replica fields after the steps run so far.
void ens_download_fields(mlb_ensemble* e)
{
    if (e->rpar_dirty) return;
    CK(cudaStreamSynchronize(e->st));
    CK(cudaMemcpy(e->rB.data(), e->d_rB[e->cur], sizeof(double) * 3 * e->nrep, cudaMemcpyDeviceToHost));
}

FastK ens_fastk(mlb_ensemble* e)
{
    const mlb_ensemble_cfg& c = e->cfg;
    const double ms = e->ms, a = c.alpha, g = c.gamma, dt = c.dt;
    FastK F;
    memset(&F, 0, sizeof(F));
    F.ex = c.J != 0.0;
    for (int d = 0; d < 6; d++) F.J[d] = (float)(c.J / (ms * ms));
    for (int q = 0; q < 3; q++) F.pbc[q] = c.pbc[q] ? 1 : 0;
    const double al = std::sqrt(c.axis[0] * c.axis[0] + c.axis[1] * c.axis[1] + c.axis[2] * c.axis[2]);
    F.ani = c.K != 0.0 && al > 0;
    if (F.ani) {
        for (int q = 0; q < 3; q++) F.axis[q] = (float)(c.axis[q] / al);
        F.ani_c = (float)(2.0 * c.K / (ms * ms));
    }
    F.th = ens_thermal(e);
    if (F.th) {
        F.seed = c.seed;
        F.counter = 0;
        F.dctr = &e->dstep->th_counter;
    }
    F.Bdev = nullptr;   // per replica (EnsLaunch::rB)
    F.status = e->status;
    F.addw = 1.f;
    F.llg_type = c.llg == MLB_LLG_QUATERNION ? LLG_QUAT : LLG_CART;
    F.tof = 1;
    F.renorm = 1;
    F.dt_zero = dt == 0.0;
    F.dt = (float)dt;
    F.precess = 1.f;
    F.ms = (float)ms;
    const double gaa = g / (1.0 + a * a);
    if (F.llg_type == LLG_CART) {
        F.c_prec = (float)-gaa;
        F.c_damp = (float)((a / ms) * gaa);
    } else {
        F.c_damp = (float)(a / ms);
        F.c_rot = (float)(0.5 * g * dt / (1.0 + a * a));
    }
    return F;
}

// The dipole field of every replica of class c from the spins s into H, on
// stream st: the fast passes over all the class's replicas at once, or the
// generic passes replica by replica (sizes outside the fast kernels).
void ens_class_conv(mlb_ensemble* e, EnsClass& c, const float* const s[3], cudaStream_t st)
{
    ConvPlan& P = *c.dip->plan;
    const long long n = (long long)c.nx * c.ny * c.nz;
    if (c.fast) {
        ConvK k = P.k;
        k.yz_variant = c.yz_variant;
        const float* cs[3] = {s[0] + c.base, s[1] + c.base, s[2] + c.base};
        float* ch[3] = {e->H[0] + c.base, e->H[1] + c.base, e->H[2] + c.base};
        CK(mlb::launch_conv_fast(k, P.L, reinterpret_cast<const float2*>(P.tw.p), cs,
                                 reinterpret_cast<float2*>(P.spec.p), reinterpret_cast<const float*>(P.ten6.p), ch,
                                 st));
        return;
    }
    ConvK k = P.k;
    k.nrep = 1;
    for (int r = 0; r < c.nrep; r++) {
        const long long o = c.base + r * n;
        const void* cs[3] = {s[0] + o, s[1] + o, s[2] + o};
        void* ch[3] = {e->H[0] + o, e->H[1] + o, e->H[2] + o};
        CK(mlb::launch_conv(k, P.L[0], P.L[1], P.L[2], P.tw.p, cs, P.spec.p, P.ten6.p, P.ten9.p, ch, 4, st));
    }
}

EnsLaunch ens_launch(mlb_ensemble* e, int q)
{
    EnsLaunch E{};
    E.nblk = e->nblk; E.bs = e->bs; E.brep = e->brep; E.bstart = e->bstart; E.rinfo = e->rinfo;
    E.grid = e->grid;
    E.rB = e->d_rB[q]; E.rBn = e->d_rB[1 - q]; E.rdB = e->d_rdB; E.rsig = e->d_rsig;
    return E;
}

// One step on spin buffer q: every class's dipole passes on a branch of its
// own (the branches run concurrently in the captured graph), joined before
// the fused step kernel over all replicas.
void ens_enqueue_step(mlb_ensemble* e, int q)
{
    const float* s[3] = {e->sp[q][0], e->sp[q][1], e->sp[q][2]};
    float* o[3] = {e->sp[1 - q][0], e->sp[1 - q][1], e->sp[1 - q][2]};
    const float* add[3] = {nullptr, nullptr, nullptr};
    if (e->cfg.g != 0.0) {
        const bool branch = e->cls.size() > 1;
        if (branch) CK(cudaEventRecord(e->fork, e->st));
        for (EnsClass& c : e->cls) {
            if (branch) {
                CK(cudaStreamWaitEvent(c.st, e->fork, 0));
                ens_class_conv(e, c, s, c.st);
                CK(cudaEventRecord(c.done, c.st));
            } else {
                ens_class_conv(e, c, s, e->st);
            }
        }
        if (branch)
            for (EnsClass& c : e->cls) CK(cudaStreamWaitEvent(e->st, c.done, 0));
        for (int q3 = 0; q3 < 3; q3++) add[q3] = e->H[q3];
    }
    CK(mlb::launch_fused_ens(ens_fastk(e), ens_launch(e, q), s, add, o, e->st));
    CK(mlb::launch_advance_step(e->dstep, e->dstep, e->st));
}

// ---------------------------------------------------------------- ensemble tuner
// Choices per ensemble: the (y,z) pass variant of every fast class (the
// register kernel where it applies, or the shared-memory Stockham kernel)
// and the fused kernel's tile size and grid (one CTA per tile, or
// persistent CTAs walking the tile table).  Each candidate is timed with
// CUDA events on the ensemble's stream over repeated launches on the
// current state (the passes write only H and the other spin buffer).  The
// choices are kept per process and in a cache file keyed by the device and
// the classes: MLB_TUNE_CACHE names the file ("off": none), else
// $XDG_CACHE_HOME/maglua_b200/tune.txt or ~/.cache/maglua_b200/tune.txt.
std::string tune_cache_path()
{
    const char* p = std::getenv("MLB_TUNE_CACHE");
    if (p) return strcasecmp(p, "off") == 0 ? std::string() : std::string(p);
    const char* x = std::getenv("XDG_CACHE_HOME");
    if (x && *x) return std::string(x) + "/maglua_b200/tune.txt";
    const char* h = std::getenv("HOME");
    if (h && *h) return std::string(h) + "/.cache/maglua_b200/tune.txt";
    return std::string();
}

std::string ens_tune_key(mlb_ensemble* e)
{
    int dev = 0;
    cudaDeviceProp pr;
    CK(cudaGetDevice(&dev));
    CK(cudaGetDeviceProperties(&pr, dev));
    std::string k = std::string(pr.name) + "/" + std::to_string(pr.multiProcessorCount) + "/" +
                    (e->cfg.llg == MLB_LLG_QUATERNION ? "Q" : "C") + (e->cfg.g != 0.0 ? "D" : "-") +
                    (ens_thermal(e) ? "T" : "-") + "/";
    for (char& ch : k)
        if (ch == ' ') ch = '_';
    for (EnsClass& c : e->cls)
        k += std::to_string(c.nx) + "x" + std::to_string(c.ny) + "x" + std::to_string(c.nz) + "*" +
             std::to_string(c.nrep) + ";";
    return k;
}

bool tune_file_lookup(const std::string& key, EnsTune& t, size_t ncls)
{
    const std::string path = tune_cache_path();
    if (path.empty()) return false;
    FILE* f = std::fopen(path.c_str(), "r");
    if (!f) return false;
    char line[4096];
    bool found = false;
    while (std::fgets(line, sizeof(line), f)) {
        std::string l(line);
        const size_t sp = l.find(' ');
        if (sp == std::string::npos || l.substr(0, sp) != key) continue;
        EnsTune u;
        int pos = 0;
        const char* v = l.c_str() + sp + 1;
        if (std::sscanf(v, "%d %d%n", &u.bs, &u.grid, &pos) != 2) continue;
        v += pos;
        for (size_t i = 0; i < ncls; i++) {
            int y = 0, m = 0;
            if (std::sscanf(v, "%d%n", &y, &m) != 1) break;
            u.yz.push_back(y);
            v += m;
        }
        if (u.yz.size() == ncls && (u.bs == 128 || u.bs == 256 || u.bs == 512)) { t = u; found = true; }
    }
    std::fclose(f);
    return found;
}

void tune_file_store(const std::string& key, const EnsTune& t)
{
    const std::string path = tune_cache_path();
    if (path.empty()) return;
    const size_t sl = path.rfind('/');
    if (sl != std::string::npos) {
        // create the cache directory (and its parent) when missing
        const std::string dir = path.substr(0, sl);
        const size_t sl2 = dir.rfind('/');
        if (sl2 != std::string::npos && sl2 > 0) mkdir(dir.substr(0, sl2).c_str(), 0755);
        mkdir(dir.c_str(), 0755);
    }
    FILE* f = std::fopen(path.c_str(), "a");
    if (!f) return;
    std::fprintf(f, "%s %d %d", key.c_str(), t.bs, t.grid);
    for (int y : t.yz) std::fprintf(f, " %d", y);
    std::fprintf(f, "\n");
    std::fclose(f);
}

template <class Fn>
float ens_time(mlb_ensemble* e, Fn&& fn, int reps)
{
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    fn();
    CK(cudaEventRecord(a, e->st));
    for (int k = 0; k < reps; k++) fn();
    CK(cudaEventRecord(b, e->st));
    CK(cudaEventSynchronize(b));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return ms / reps;
}

void ens_autotune(mlb_ensemble* e)
{
    const std::string key = ens_tune_key(e);
    EnsTune t;
    bool have = false;
    {
        std::lock_guard<std::mutex> lk(g_ens_tune_mu);
        auto it = g_ens_tuned.find(key);
        if (it != g_ens_tuned.end()) { t = it->second; have = true; }
    }
    if (!have && tune_file_lookup(key, t, e->cls.size())) {
        have = true;
        e->tune_log = "tuner: cached choices for " + key + "\n";
    }
    const float* s[3] = {e->sp[e->cur][0], e->sp[e->cur][1], e->sp[e->cur][2]};
    if (!have) {
        char buf[256];
        std::string log = "tuner: " + key + "\n";
        // (y,z) pass variant per fast class
        for (EnsClass& c : e->cls) {
            int best_v = 0;
            if (e->cfg.g != 0.0 && c.fast) {
                float best = 1e30f;
                // 2 (the 384-thread register kernel) differs from 0 only for 256-wide planes
                const int nv = c.dip->plan->k.Py == 256 ? 3 : 2;
                for (int v = 0; v < nv; v++) {
                    c.yz_variant = v;
                    const float ms = ens_time(e, [&] { ens_class_conv(e, c, s, e->st); }, 10);
                    std::snprintf(buf, sizeof(buf), "  class %dx%dx%d (%d replicas): (y,z) %s %.1f us per evaluation\n",
                                  c.nx, c.ny, c.nz, c.nrep,
                                  v == 0 ? "automatic" : (v == 1 ? "Stockham" : "register, one thread per column"),
                                  1e3 * ms);
                    log += buf;
                    if (ms < best) { best = ms; best_v = v; }
                }
            }
            c.yz_variant = best_v;
            t.yz.push_back(best_v);
        }
        // fused step: tile size x grid
        const float* add[3] = {nullptr, nullptr, nullptr};
        if (e->cfg.g != 0.0) for (int q = 0; q < 3; q++) add[q] = e->H[q];
        float* o[3] = {e->sp[1 - e->cur][0], e->sp[1 - e->cur][1], e->sp[1 - e->cur][2]};
        int dev = 0, nsm = 148;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        float best = 1e30f;
        // the tuner's launches write the field of the step after next into
        // a scratch copy of the field buffer, not into the live one
        double* scratchB = nullptr;
        CK(cudaMalloc(&scratchB, sizeof(double) * 3 * e->nrep));
        for (int bs : {128, 256, 512}) {
            ens_block_table(e, bs);
            for (int per_sm : {0, 2, 4, 8}) {
                e->grid = per_sm ? per_sm * nsm : 0;
                if (e->grid >= e->nblk) continue;
                EnsLaunch E = ens_launch(e, e->cur);
                E.rBn = scratchB;
                const FastK F = ens_fastk(e);
                const float ms = ens_time(e, [&] { CK(mlb::launch_fused_ens(F, E, s, add, o, e->st)); }, 10);
                std::snprintf(buf, sizeof(buf), "  fused step: tile %d sites, %s: %.1f us\n", bs,
                              per_sm ? (std::to_string(e->grid) + " persistent CTAs").c_str()
                                     : (std::to_string(e->nblk) + " CTAs (one per tile)").c_str(),
                              1e3 * ms);
                log += buf;
                if (ms < best) { best = ms; t.bs = bs; t.grid = e->grid; }
            }
        }
        cudaFree(scratchB);
        std::snprintf(buf, sizeof(buf), "  chosen: tile %d, grid %d (0 = one CTA per tile)\n", t.bs, t.grid);
        log += buf;
        e->tune_log = log;
        tune_file_store(key, t);
    }
    {
        std::lock_guard<std::mutex> lk(g_ens_tune_mu);
        g_ens_tuned[key] = t;
    }
    for (size_t i = 0; i < e->cls.size(); i++) e->cls[i].yz_variant = i < t.yz.size() ? t.yz[i] : 0;
    ens_block_table(e, t.bs);
    e->grid = t.grid;
    e->tuned = true;
}

void ens_prepare(mlb_ensemble* e)
{
    if (!e->configured) fail(MLB_ESTATE, "ensemble not configured");
    if (!e->have_ms) fail(MLB_ESTATE, "ensemble spins not set");
    ens_upload_params(e);
    if (e->exec[0]) return;
    const mlb_ensemble_cfg& c = e->cfg;
    if (c.g != 0.0) {
        for (EnsClass& k : e->cls) {
            if (!k.dip) {
                k.dip = new mlb_op();
                k.dip->kind = MLB_OP_DIPOLE;
                k.dip->nx = k.nx; k.dip->ny = k.ny; k.dip->nz = k.nz;
                k.dip->slot = "Dipole";
            }
            k.dip->open[0] = c.open_xy ? 1 : 0;
            k.dip->open[1] = c.open_xy ? 1 : 0;
            k.dip->open[2] = 1;
            k.dip->t6_valid = false;
            k.dip->plan_dirty = true;
            build_plan(k.dip, e->st, 4);
            ConvPlan& P = *k.dip->plan;
            k.fast = mlb::conv_fast_ok(P.k) && !P.k.split;
            P.k.g = c.g / ((double)P.k.Px * P.k.Py * P.k.Pz);
            P.k.nrep = k.fast ? k.nrep : 1;
            P.spec.alloc((size_t)P.k.Kx * 3 * k.nz * k.ny * P.k.nrep * sizeof(float2));
        }
    }
    if (!e->tuned) ens_autotune(e);
    CK(cudaStreamSynchronize(e->st));
    for (int q = 0; q < 2; q++) {
        cudaGraph_t graph = nullptr;
        CK(cudaStreamBeginCapture(e->st, cudaStreamCaptureModeThreadLocal));
        bool ok = true;
        std::string why;
        try {
            ens_enqueue_step(e, q);
        } catch (Err& er) {
            ok = false;
            why = er.msg;
        }
        cudaError_t ce = cudaStreamEndCapture(e->st, &graph);
        if (!ok || ce != cudaSuccess) {
            if (graph) cudaGraphDestroy(graph);
            ens_free_graphs(e);
            fail(MLB_ESTATE, "ensemble capture failed: " + (ok ? std::string(cudaGetErrorString(ce)) : why));
        }
        ce = cudaGraphInstantiate(&e->exec[q], graph, 0);
        cudaGraphDestroy(graph);
        if (ce != cudaSuccess) { ens_free_graphs(e); fail(MLB_ECUDA, cudaGetErrorString(ce)); }
    }
}

} // namespace

// ====================================================================== C ABI
extern "C" {

const char* mlb_last_error(void) { return g_err.c_str(); }

int mlb_profile_begin(void)
{
    return guard([&] { mlb::prof_begin(); });
}

int mlb_profile_end(int cap, char* names, double* ms, int* launches, int* count)
{
    return guard([&] { *count = mlb::prof_end(cap, names, ms, launches); });
}

int mlb_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    const Philox4 r = philox4x32_10(ctr[0], ctr[1], ctr[2], ctr[3], key[0], key[1]);
    for (int i = 0; i < 4; i++) out[i] = r.v[i];
    return MLB_OK;
}
int mlb_version(void) { return 1; }

int mlb_init(int device)
{
    return guard([&] {
        CK(cudaSetDevice(device));
        CK(cudaFree(0));
        CK(mlb::conv_configure());
        CK(mlb::fftreg_init());
        CK(mlb::conv_fast_configure());
        CK(mlb::sur_configure());
    });
}

int mlb_system_create(int nx, int ny, int nz, mlb_system** out)
{
    return guard([&] {
        if (!out) fail(MLB_EINVAL, "null output");
        *out = make_system(nx, ny, nz, 4);
    });
}

int mlb_system_create_ex(int nx, int ny, int nz, int real_bytes, mlb_system** out)
{
    return guard([&] {
        if (!out) fail(MLB_EINVAL, "null output");
        *out = make_system(nx, ny, nz, real_bytes);
    });
}

int mlb_system_real_bytes(const mlb_system* s, int* out)
{
    return guard([&] { *out = s->rb; });
}

int mlb_system_destroy(mlb_system* s)
{
    return guard([&] {
        g_version++; free_system(s); });
}

int mlb_system_dims(const mlb_system* s, int out[3])
{
    return guard([&] {
        out[0] = s->nx; out[1] = s->ny; out[2] = s->nz;
    });
}

int mlb_system_status(mlb_system* s, int clear, unsigned* flags)
{
    return guard([&] {
        if (!s || !flags) fail(MLB_EINVAL, "null argument");
        CK(cudaStreamSynchronize(s->st));
        CK(cudaMemcpy(flags, s->status, sizeof(unsigned), cudaMemcpyDeviceToHost));
        if (clear) CK(cudaMemset(s->status, 0, sizeof(unsigned)));
    });
}

int mlb_system_set_stream(mlb_system* s, void* stream)
{
    return guard([&] {
        g_version++;
        CK(cudaStreamSynchronize(s->st));
        s->st = stream ? (cudaStream_t)stream : s->own;
    });
}

int mlb_system_get_stream(const mlb_system* s, void** stream)
{
    return guard([&] { *stream = (void*)s->st; });
}

int mlb_system_synchronize(mlb_system* s)
{
    return guard([&] { CK(cudaStreamSynchronize(s->st)); });
}

int mlb_system_set_spin(mlb_system* s, int idx, double sx, double sy, double sz)
{
    return guard([&] {
        g_version++;
        if (idx < 0 || idx >= s->n) fail(MLB_ERANGE, "site outside the SpinSystem");
        spins_changing(s);
        const double v[3] = {sx, sy, sz};
        for (int c = 0; c < 3; c++) put_reals(s, elem(s->sp[s->cur][c], idx, s->rb), &v[c], 1);
        const double m = std::sqrt(sx * sx + sy * sy + sz * sz);
        put_reals(s, elem(s->ms, idx, s->rb), &m, 1);
        s->ms_host[idx] = round_to(m, s->rb);
        s->ms_dirty = true;
        s->ms_token = ++g_ms_token;
        CK(cudaStreamSynchronize(s->st));
    });
}

int mlb_system_get_spin(mlb_system* s, int idx, double out4[4])
{
    return guard([&] {
        if (idx < 0 || idx >= s->n) fail(MLB_ERANGE, "site outside the SpinSystem");
        for (int c = 0; c < 3; c++) get_reals(s, &out4[c], elem(s->sp[s->cur][c], idx, s->rb), 1);
        out4[3] = s->ms_host[idx];
    });
}

int mlb_system_set_spins(mlb_system* s, const double* x, const double* y, const double* z, const double* ms)
{
    return guard([&] {
        g_version++;
        if (!x || !y || !z) fail(MLB_EINVAL, "null spin array");
        spins_changing(s);
        const double* src[3] = {x, y, z};
        for (int c = 0; c < 3; c++) put_reals(s, s->sp[s->cur][c], src[c], s->n);
        for (int i = 0; i < s->n; i++)
            s->ms_host[i] = ms ? ms[i] : std::sqrt(x[i] * x[i] + y[i] * y[i] + z[i] * z[i]);
        put_reals(s, s->ms, s->ms_host.data(), s->n);
        for (int i = 0; i < s->n; i++) s->ms_host[i] = round_to(s->ms_host[i], s->rb);
        s->ms_dirty = true;
        s->ms_token = ++g_ms_token;
        CK(cudaStreamSynchronize(s->st));
    });
}

int mlb_system_get_spins(mlb_system* s, double* x, double* y, double* z, double* ms)
{
    return guard([&] {
        double* dst[3] = {x, y, z};
        for (int c = 0; c < 3; c++)
            if (dst[c]) get_reals(s, dst[c], s->sp[s->cur][c], s->n);
        if (ms)
            for (int i = 0; i < s->n; i++) ms[i] = s->ms_host[i];
    });
}

int mlb_system_upload_f32(mlb_system* s, const float* x, const float* y, const float* z, const float* ms)
{
    return guard([&] {
        // captured steps hold device pointers and the moment magnitudes'
        // constants, not spin values: a write of the spins alone keeps them
        // (the carried spectrum and lazy records are settled below)
        if (ms) {
            g_version++;
            spins_changing(s);
        } else {
            current_spins_changing(s);
        }
        const float* src[3] = {x, y, z};
        if (s->rb == 4) {
            for (int c = 0; c < 3; c++)
                CK(cudaMemcpyAsync(s->sp[s->cur][c], src[c], sizeof(float) * s->n, cudaMemcpyHostToDevice, s->st));
            if (ms) CK(cudaMemcpyAsync(s->ms, ms, sizeof(float) * s->n, cudaMemcpyHostToDevice, s->st));
        } else {
            std::vector<double> d(s->n);
            for (int c = 0; c < 3; c++) {
                for (int i = 0; i < s->n; i++) d[i] = src[c][i];
                put_reals(s, s->sp[s->cur][c], d.data(), s->n);
            }
            if (ms) {
                for (int i = 0; i < s->n; i++) d[i] = ms[i];
                put_reals(s, s->ms, d.data(), s->n);
            }
        }
        if (ms) {
            bool changed = false;
            for (int i = 0; i < s->n; i++)
                if (s->ms_host[i] != (double)ms[i]) { s->ms_host[i] = ms[i]; changed = true; }
            if (changed) { s->ms_dirty = true; s->ms_token = ++g_ms_token; }
        }
    });
}

int mlb_system_download_f32(mlb_system* s, float* x, float* y, float* z)
{
    return guard([&] {
        float* dst[3] = {x, y, z};
        if (s->rb == 4) {
            for (int c = 0; c < 3; c++)
                if (dst[c])
                    CK(cudaMemcpyAsync(dst[c], s->sp[s->cur][c], sizeof(float) * s->n, cudaMemcpyDeviceToHost, s->st));
        } else {
            std::vector<double> d(s->n);
            for (int c = 0; c < 3; c++) {
                if (!dst[c]) continue;
                get_reals(s, d.data(), s->sp[s->cur][c], s->n);
                for (int i = 0; i < s->n; i++) dst[c][i] = (float)d[i];
            }
        }
    });
}

int mlb_system_set_param(mlb_system* s, int which, double v)
{
    return guard([&] {
        g_version++;
        switch (which) {
        case MLB_ALPHA:
            // setAlpha drops per-site values (SpinSystem::setAlpha :1003-1008)
            if (s->sa) { spins_changing(s); CK(cudaStreamSynchronize(s->st)); cudaFree(s->sa); s->sa = nullptr; }
            s->alpha = v;
            break;
        case MLB_GAMMA:
            if (s->sg) { spins_changing(s); CK(cudaStreamSynchronize(s->st)); cudaFree(s->sg); s->sg = nullptr; }
            s->gamma = v;
            break;
        case MLB_DT: s->dt = v; break;
        case MLB_TIME: s->time = v; break;
        default: fail(MLB_EINVAL, "unknown parameter");
        }
    });
}

int mlb_system_get_param(const mlb_system* s, int which, double* v)
{
    return guard([&] {
        switch (which) {
        case MLB_ALPHA: *v = s->alpha; break;
        case MLB_GAMMA: *v = s->gamma; break;
        case MLB_DT: *v = s->dt; break;
        case MLB_TIME: *v = s->time; break;
        default: fail(MLB_EINVAL, "unknown parameter");
        }
    });
}

int mlb_system_set_site_alpha(mlb_system* s, const double* a)
{
    return guard([&] {
        g_version++; upload_site_array(s, &s->sa, a); });
}

int mlb_system_set_site_gamma(mlb_system* s, const double* g)
{
    return guard([&] {
        g_version++; upload_site_array(s, &s->sg, g); });
}

int mlb_system_reset_fields(mlb_system* s)
{
    return guard([&] { reset_fields(s); });
}

int mlb_system_sum_fields(mlb_system* s)
{
    return guard([&] {
        before_mutate(s, 0);
        sum_fields(s);
    });
}

int mlb_system_sum_fields_custom(mlb_system* s, const char* dest, int n, const char* const* src, const double* w)
{
    return guard([&] {
        const int d = slot_register(s, dest);
        before_mutate(s, d);
        // materialise the sources and the destination, then a weighted sum
        std::vector<int> idx;
        std::vector<double> ww;
        for (int k = 0; k < n; k++) {
            const int j = slot_find(s, src[k]);
            if (j < 0 || !s->slots[j].used) continue;
            materialize(s, j);
            idx.push_back(j);
            ww.push_back(w ? w[k] : 1.0);
        }
        Slot& out = s->slots[d];
        out.terms.clear();
        out.sum_list.clear();
        slot_alloc(s, out);
        // accumulate in batches of addends
        int acc = 0;
        size_t k = 0;
        do {
            TermsK T;
            terms_init(T);
            for (; k < idx.size() && T.nadd < MLB_MAX_ADDENDS; k++) {
                const int j = idx[k];
                if (j == d) {
                    // the destination is also a source: copy it aside first
                    fail(MLB_EUNSUP, "destination listed among the sources");
                }
                add_addend(T, s->slots[j].h, ww[k], false);
            }
            eval_into(s, s->cur, T, s->dt, out, acc);
            acc = 1;
        } while (k < idx.size());
        out.state = ST_DATA;
    });
}

int mlb_system_get_field(mlb_system* s, const char* slot, double* hx, double* hy, double* hz)
{
    return guard([&] {
        const int j = slot_find(s, slot);
        if (j < 0) fail(MLB_ENOTFOUND, std::string("Unknown field type `") + slot + "'");
        materialize(s, j);
        double* dst[3] = {hx, hy, hz};
        for (int c = 0; c < 3; c++)
            if (dst[c]) get_reals(s, dst[c], s->slots[j].h[c], s->n);
    });
}

int mlb_system_set_field(mlb_system* s, const char* slot, const double* hx, const double* hy, const double* hz)
{
    return guard([&] {
        g_version++;
        const int j = slot_register(s, slot);
        before_mutate(s, j);
        materialize(s, j);
        const double* src[3] = {hx, hy, hz};
        for (int c = 0; c < 3; c++)
            if (src[c]) put_reals(s, s->slots[j].h[c], src[c], s->n);
        CK(cudaStreamSynchronize(s->st));
    });
}

int mlb_system_slot_used(mlb_system* s, const char* slot, int* used)
{
    return guard([&] {
        const int j = slot_find(s, slot);
        if (j < 0) fail(MLB_ENOTFOUND, std::string("Unknown field type `") + slot + "'");
        *used = s->slots[j].used ? 1 : 0;
    });
}

int mlb_system_set_slot_used(mlb_system* s, const char* slot, int used)
{
    return guard([&] {
        const int j = slot_find(s, slot);
        if (j < 0) fail(MLB_ENOTFOUND, std::string("Unknown field type`") + slot + "'");
        s->slots[j].used = used != 0;
    });
}

int mlb_system_ensure_slot(mlb_system* s, const char* slot)
{
    return guard([&] { slot_register(s, slot); });
}

// The netMoment reduction of the current spins with its copy to pinned
// destination d (6 doubles at nm_host + 6 d), enqueued on the system's stream
// as one captured graph per spin buffer and destination.
static void netmoment_enqueue(mlb_system* s, double m, int d, cudaStream_t st)
{
    const int q = s->cur;
    // the synchronous read (d = 0) and the slots (on their own stream) use
    // separate partial sums and counters
    double* red = d ? s->red_a : s->red;
    double* redout = d ? s->redout_a : s->redout;
    unsigned* counter = d ? s->nm_counter_a : s->nm_counter;
    if (!s->nm_exec[q][d] || s->nm_m[q][d] != m) {
        if (s->nm_exec[q][d]) { cudaGraphExecDestroy(s->nm_exec[q][d]); s->nm_exec[q][d] = nullptr; }
        CK(cudaStreamSynchronize(s->st));
        if (s->nm_st) CK(cudaStreamSynchronize(s->nm_st));
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal));
        // one kernel: the last block writes the sums into the pinned slot
        // the slots' reads (d > 0) run on a few SMs next to the following steps
        const int nb = std::min(s->red_nb, mlb::netmoment_blocks(s->n, d > 0));
        cudaError_t e = mlb::launch_netmoment_one(s->sp[q][0], s->sp[q][1], s->sp[q][2], s->n, m, red, nb, counter,
                                                  s->nm_host_dev + 6 * d, redout, s->rb, s->st);
        cudaError_t e2 = cudaStreamEndCapture(s->st, &g);
        if (e == cudaSuccess) e = e2;
        if (e == cudaSuccess) e = cudaGraphInstantiate(&s->nm_exec[q][d], g, 0);
        if (g) cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            cudaGetLastError();
            fail(MLB_ECUDA, std::string("netMoment graph: ") + cudaGetErrorString(e));
        }
        s->nm_m[q][d] = m;
    }
    CK(cudaGraphLaunch(s->nm_exec[q][d], st));
}

static void netmoment_out(const double* r, double out8[8])
{
    out8[0] = r[0]; out8[1] = r[1]; out8[2] = r[2];
    out8[3] = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    out8[4] = r[3]; out8[5] = r[4]; out8[6] = r[5];
    out8[7] = std::sqrt(r[3] * r[3] + r[4] * r[4] + r[5] * r[5]);
}

int mlb_system_netmoment(mlb_system* s, double m, double out8[8])
{
    return guard([&] {
        netmoment_enqueue(s, m, 0, s->st);
        CK(cudaStreamSynchronize(s->st));
        double r[6];
        for (int k = 0; k < 6; k++) r[k] = s->nm_host[k];
        netmoment_out(r, out8);
    });
}

int mlb_system_netmoment_async(mlb_system* s, double m, int slot)
{
    return guard([&] {
        if (slot < 0 || slot > 3) fail(MLB_EINVAL, "netMoment slot must be 0..3");
        if (!s->nm_st) CK(cudaStreamCreateWithFlags(&s->nm_st, cudaStreamNonBlocking));
        if (!s->nm_ev[slot]) CK(cudaEventCreateWithFlags(&s->nm_ev[slot], cudaEventDisableTiming));
        if (!s->nm_go[slot]) CK(cudaEventCreateWithFlags(&s->nm_go[slot], cudaEventDisableTiming));
        // a slot still reading a buffer: the system's stream waits for it
        // before anything later, as before this call reused it
        if (s->nm_reading[slot]) {
            CK(cudaStreamWaitEvent(s->st, s->nm_ev[slot], 0));
            s->nm_reading[slot] = false;
        }
        // the reduction of the current spins runs on the side stream once
        // the system's stream has produced them, next to the following steps
        CK(cudaEventRecord(s->nm_go[slot], s->st));
        CK(cudaStreamWaitEvent(s->nm_st, s->nm_go[slot], 0));
        netmoment_enqueue(s, m, 1 + slot, s->nm_st);
        CK(cudaEventRecord(s->nm_ev[slot], s->nm_st));
        s->nm_buf[slot] = s->cur;
        s->nm_reading[slot] = true;
        s->nm_pending[slot] = true;
    });
}

int mlb_system_netmoment_wait(mlb_system* s, int slot, double out8[8])
{
    return guard([&] {
        if (slot < 0 || slot > 3) fail(MLB_EINVAL, "netMoment slot must be 0..3");
        if (!s->nm_pending[slot]) fail(MLB_ESTATE, "no netMoment enqueued in this slot");
        CK(cudaEventSynchronize(s->nm_ev[slot]));
        s->nm_pending[slot] = false;
        netmoment_out(s->nm_host + 6 * (1 + slot), out8);
    });
}

int mlb_system_field_dot(mlb_system* s, const char* slot, double* out)
{
    return guard([&] {
        const int j = slot_find(s, slot);
        if (j < 0) fail(MLB_ENOTFOUND, std::string("Unknown field type `") + slot + "'");
        materialize(s, j);
        const void* sp[3] = {s->sp[s->cur][0], s->sp[s->cur][1], s->sp[s->cur][2]};
        const void* h[3] = {s->slots[j].h[0], s->slots[j].h[1], s->slots[j].h[2]};
        CK(mlb::launch_dot(sp, h, s->n, s->red, s->red_nb, s->redout, s->rb, s->st));
        CK(cudaMemcpyAsync(out, s->redout, sizeof(double), cudaMemcpyDeviceToHost, s->st));
        CK(cudaStreamSynchronize(s->st));
    });
}

int mlb_system_diff(mlb_system* a, mlb_system* b, double out4[4])
{
    return guard([&] { system_diff(a, b, out4); });
}

// ---------------------------------------------------------------- encode / decode
// The LuaBaseObject byte stream of a SpinSystem as the reference's CPU build
// writes it (SpinSystem::encode / decode, spinsystem.cpp:669-851; the
// primitives, luabaseobject.cpp:142-205 and 250-360; an object exported as a
// Lua value, luamigrate.cpp:75-76 and 265-275): native-endian int32, double
// and char, no padding.  An object is LUA_TUSERDATA (7), its type id, char
// 111 and its index in the stream's object list (or char 222 and the index
// of an object written before), then its fields.
namespace {

const int kLuaNil = 0;
const int kLuaUserdata = 7;
const signed char kEncNew = 111;
const signed char kEncOld = (signed char)222;

// hash32 (factory.cpp:123-131): MurmurHash3 x86_32 (Austin Appleby's
// published algorithm) of the type name with seed 1000, in the reference's
// form: its tail block rotates by 16 bits where the published one rotates by
// 15 (MurmurHash3.cpp:137-143).  Kept so that type ids match its streams.
int32_t type_id(const char* name)
{
    const uint32_t c1 = 0xcc9e2d51u, c2 = 0x1b873593u;
    auto rotl = [](uint32_t x, int r) { return (x << r) | (x >> (32 - r)); };
    const size_t len = std::strlen(name);
    const unsigned char* d = reinterpret_cast<const unsigned char*>(name);
    uint32_t h = 1000;
    const size_t nb = len / 4;
    for (size_t i = 0; i < nb; i++) {
        uint32_t k = (uint32_t)d[4 * i] | ((uint32_t)d[4 * i + 1] << 8) | ((uint32_t)d[4 * i + 2] << 16) |
                     ((uint32_t)d[4 * i + 3] << 24);
        k = rotl(k * c1, 15) * c2;
        h = rotl(h ^ k, 13) * 5 + 0xe6546b64u;
    }
    const unsigned char* t = d + 4 * nb;
    uint32_t k = 0;
    switch (len & 3) {
    case 3: k ^= (uint32_t)t[2] << 16; [[fallthrough]];
    case 2: k ^= (uint32_t)t[1] << 8; [[fallthrough]];
    case 1:
        k ^= t[0];
        k = rotl(k * c1, 16) * c2;
        h ^= k;
    }
    h ^= (uint32_t)len;
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return (int32_t)h;
}

struct StreamOut {
    std::vector<char> b;
    void put(const void* p, size_t n) { b.insert(b.end(), (const char*)p, (const char*)p + n); }
    void i32(int32_t v) { put(&v, 4); }
    void f64(double v) { put(&v, 8); }
    void ch(signed char v) { put(&v, 1); }
    void header(const char* type, int idx) { i32(kLuaUserdata); i32(type_id(type)); ch(kEncNew); i32(idx); }
    // Array<double>::encode (M/cpu/array/array_core_cpu.h:200-225): version
    // 0, the size, then flag 1 and one value when every value compares
    // equal, else flag 0 and all of them.
    void darray(int idx, const mlb_system* s, const std::vector<double>& a)
    {
        header("Array.Double", idx);
        ch(0);
        i32(s->nx); i32(s->ny); i32(s->nz);
        bool same = true;
        for (int i = 1; i < s->n && same; i++) same = (a[i] == a[0]);
        if (same) { i32(1); f64(a[0]); }
        else { i32(0); put(a.data(), sizeof(double) * a.size()); }
    }
};

struct StreamIn {
    const char* p;
    size_t len, pos = 0;
    void take(void* d, size_t n)
    {
        if (n > len - pos) fail(MLB_EINVAL, "malformed stream: ends early");
        std::memcpy(d, p + pos, n);
        pos += n;
    }
    int32_t i32() { int32_t v; take(&v, 4); return v; }
    double f64() { double v; take(&v, 8); return v; }
    signed char ch() { signed char v; take(&v, 1); return v; }
};

// decodeLuaBaseObject (luabaseobject.cpp:307-360) of an Array.Double of the
// system's size; an old-object entry refers to one decoded before.
std::vector<double> read_darray(StreamIn& in, int nx, int ny, int nz, std::map<int, std::vector<double>>& seen)
{
    if (in.i32() != kLuaUserdata) fail(MLB_EINVAL, "malformed stream: expected an object");
    if (in.i32() != type_id("Array.Double")) fail(MLB_EUNSUP, "array type other than Array.Double");
    const signed char magic = in.ch();
    const int idx = in.i32();
    if (magic == kEncOld) {
        auto it = seen.find(idx);
        if (it == seen.end()) fail(MLB_EINVAL, "malformed stream: unknown object index");
        return it->second;
    }
    if (magic != kEncNew) fail(MLB_EINVAL, "malformed stream: bad object flag");
    if (in.ch() != 0) fail(MLB_EUNSUP, "unknown Array version");
    const int x = in.i32(), y = in.i32(), z = in.i32();
    if (x != nx || y != ny || z != nz) fail(MLB_EINVAL, "array size differs from the system's");
    const size_t n = (size_t)nx * ny * nz;
    std::vector<double> a(n);
    const int flag = in.i32();
    if (flag == 1) {
        const double v = in.f64();
        std::fill(a.begin(), a.end(), v);
    } else if (flag == 0) {
        in.take(a.data(), sizeof(double) * n);
    } else {
        fail(MLB_EINVAL, "malformed stream: bad array flag");
    }
    seen[idx] = a;
    return a;
}

}  // namespace

int mlb_system_encode(mlb_system* s, int first_index, void* buf, size_t cap, size_t* len, int* objects)
{
    return guard([&] {
        if (!s || !len) fail(MLB_EINVAL, "null argument");
        if (first_index < 0) fail(MLB_EINVAL, "negative object index");
        if (s->capturing) fail(MLB_ESTATE, "encode during capture");
        std::vector<double> a[4];
        for (int c = 0; c < 3; c++) {
            a[c].resize(s->n);
            get_reals(s, a[c].data(), s->sp[s->cur][c], s->n);
        }
        a[3] = s->ms_host;
        StreamOut o;
        o.header("SpinSystem", first_index);
        o.ch(0);
        o.i32(s->nx); o.i32(s->ny); o.i32(s->nz);
        o.f64(s->alpha); o.f64(s->dt); o.f64(s->gamma); o.f64(s->time);
        int idx = first_index + 1;
        for (int c = 0; c < 4; c++) o.darray(idx++, s, a[c]);
        for (void* site : {s->sa, s->sg}) {
            o.i32(site ? 1 : 0);
            if (!site) continue;
            std::vector<double> v(s->n);
            get_reals(s, v.data(), site, s->n);
            o.darray(idx++, s, v);
        }
        o.i32(0);   // no site carries extra data
        *len = o.b.size();
        if (objects) *objects = idx - first_index;
        if (!buf) return;
        if (cap < o.b.size()) fail(MLB_EINVAL, "buffer smaller than the stream");
        std::memcpy(buf, o.b.data(), o.b.size());
    });
}

int mlb_system_decode(const void* buf, size_t len, int real_bytes, mlb_system** out, size_t* used, int* objects)
{
    return guard([&] {
        if (!buf || !out) fail(MLB_EINVAL, "null argument");
        *out = nullptr;
        StreamIn in{static_cast<const char*>(buf), len};
        if (in.i32() != kLuaUserdata) fail(MLB_EINVAL, "malformed stream: expected an object");
        if (in.i32() != type_id("SpinSystem")) fail(MLB_EINVAL, "stream does not hold a SpinSystem");
        if (in.ch() != kEncNew) fail(MLB_EINVAL, "malformed stream: bad object flag");
        in.i32();
        if (in.ch() != 0) fail(MLB_EUNSUP, "unknown SpinSystem version");
        const int nx = in.i32(), ny = in.i32(), nz = in.i32();
        if (nx <= 0 || ny <= 0 || nz <= 0) fail(MLB_EINVAL, "malformed stream: bad system size");
        if ((long long)nx * ny * nz > (1LL << 31) - 1) fail(MLB_EUNSUP, "more than 2^31-1 sites");
        const double alpha = in.f64(), dt = in.f64(), gamma = in.f64(), time = in.f64();
        std::map<int, std::vector<double>> seen;
        std::vector<double> a[4];
        for (int c = 0; c < 4; c++) a[c] = read_darray(in, nx, ny, nz, seen);
        std::vector<double> site[2];
        bool has[2] = {false, false};
        for (int k = 0; k < 2; k++) {
            has[k] = in.i32() != 0;
            if (has[k]) site[k] = read_darray(in, nx, ny, nz, seen);
        }
        // sites' extra data: Lua values, which this library does not hold;
        // a stream whose every site has nil is accepted
        const int nextra = in.i32();
        if (nextra > 0) fail(MLB_EUNSUP, "sites carry extra data (Lua values)");
        if (nextra < 0)
            for (long long i = 0; i < (long long)nx * ny * nz; i++)
                if (in.i32() != kLuaNil) fail(MLB_EUNSUP, "sites carry extra data (Lua values)");
        if (!used && in.pos != in.len) fail(MLB_EINVAL, "malformed stream: trailing bytes");
        mlb_system* s = make_system(nx, ny, nz, real_bytes);
        try {
            s->alpha = alpha; s->dt = dt; s->gamma = gamma; s->time = time;
            const double* src[3] = {a[0].data(), a[1].data(), a[2].data()};
            for (int c = 0; c < 3; c++) put_reals(s, s->sp[s->cur][c], src[c], s->n);
            for (int i = 0; i < s->n; i++) s->ms_host[i] = a[3][i];
            put_reals(s, s->ms, s->ms_host.data(), s->n);
            for (int i = 0; i < s->n; i++) s->ms_host[i] = round_to(s->ms_host[i], s->rb);
            s->ms_dirty = true;
            s->ms_token = ++g_ms_token;
            if (has[0]) upload_site_array(s, &s->sa, site[0].data());
            if (has[1]) upload_site_array(s, &s->sg, site[1].data());
            CK(cudaStreamSynchronize(s->st));
        } catch (...) {
            mlb_system_destroy(s);
            throw;
        }
        *out = s;
        if (used) *used = in.pos;
        if (objects) *objects = 1 + (int)seen.size();   // the system and the arrays new in the stream
    });
}

// ---------------------------------------------------------------- operator and LLG streams
// The bytes the reference's CPU build writes for its operators and
// integrators inside a checkpoint, as an exported Lua value: LUA_TUSERDATA,
// the type id, char 111 and the object's index, then the class's encode
// (M/ = src/modules/):
//   SpinOperation base  char 0, nx, ny, nz, global scale (M/cpu/core/spinoperation.cpp:67-75)
//   Exchange            base, char 1, normalizeMoments, pbc[3], count, (from, to, J) per pathway
//                       (M/cpu/exchange/spinoperationexchange.cpp:52-73)
//   Anisotropy          base, char 0, count, (site, axis[3], K) (spinoperationanisotropy.cpp:191-207)
//   Anisotropy.Uniaxial base, char 0, count, (site, axis[3], K1, K2) (..._uniaxial.cpp:181-199)
//   Anisotropy.Cubic    base, char 0, count, (site, axis1[3], axis2[3], K[3]) (..._cubic.cpp:239-258)
//   Thermal             base, char 0, temperature, the scale array by its own encode: char 111,
//                       its index, char 0, nx, ny, nz, flag, one value or all
//                       (M/cpu/thermal/spinoperationthermal.cpp:51-61, array_core_cpu.h:200-225)
//   AppliedField        base, char 0, B[3] (spinoperationappliedfield.cpp:33-42)
//   Dipole              LongRange's encode (base, char 0, gmax[4], g, ABC[9],
//                       spinoperationlongrange.cpp:55-68), char 0 (spinoperationdipole.cpp:35-41)
//   LLG.Cartesian / LLG.Quaternion  char 1, thermalOnlyFirstTerm, disableRenormalization,
//                       precession and damping scales (M/cpu/llg/llg.cpp:50-60)
// Pathway sites are 0-based, as stored.  A plain LongRange is not written:
// LongRange::encode begins with no object header, so no reader (the
// reference's decodeLuaBaseObject included) can take its stream back.
// Reading: the reference's Thermal::decode hands the stream to
// Array::decode, which does not read the array's header (char 111 and
// index) that the array's encode wrote; this reader takes the header.
namespace {

const char* op_type_name(int kind)
{
    switch (kind) {
    case MLB_OP_EXCHANGE: return "Exchange";
    case MLB_OP_ANISOTROPY: return "Anisotropy";
    case MLB_OP_UNIAXIAL: return "Anisotropy.Uniaxial";
    case MLB_OP_CUBIC: return "Anisotropy.Cubic";
    case MLB_OP_THERMAL: return "Thermal";
    case MLB_OP_APPLIEDFIELD: return "AppliedField";
    case MLB_OP_DIPOLE: return "Dipole";
    }
    return nullptr;
}

void put_stream(const StreamOut& o, void* buf, size_t cap, size_t* len)
{
    *len = o.b.size();
    if (buf && cap >= o.b.size()) std::memcpy(buf, o.b.data(), o.b.size());
    else if (buf) fail(MLB_ERANGE, "buffer smaller than the stream (" + std::to_string(o.b.size()) + " bytes)");
}

void ck_rc(int rc)
{
    if (rc != MLB_OK) fail(rc, g_err);
}

} // namespace

int mlb_op_encode(mlb_op* op, int first_index, void* buf, size_t cap, size_t* len, int* objects)
{
    return guard([&] {
        if (!op || !len) fail(MLB_EINVAL, "null argument");
        if (first_index < 0) fail(MLB_EINVAL, "negative object index");
        const char* name = op_type_name(op->kind);
        if (!name)
            fail(MLB_EUNSUP, op->kind == MLB_OP_LONGRANGE
                                 ? "LongRange::encode writes no object header: its stream cannot be read back"
                                 : "this operator has no encoded form in the reference");
        StreamOut o;
        o.header(name, first_index);
        int nobj = 1;
        o.ch(0);                       // SpinOperation::encode
        o.i32(op->nx); o.i32(op->ny); o.i32(op->nz);
        o.f64(op->gs);
        switch (op->kind) {
        case MLB_OP_EXCHANGE:
            o.ch(1);
            o.i32(op->normalize ? 1 : 0);
            for (int a = 0; a < 3; a++) o.i32(op->ex_pbc[a]);
            o.i32((int)op->ef.size());
            for (size_t p = 0; p < op->ef.size(); p++) { o.i32(op->ef[p]); o.i32(op->et[p]); o.f64(op->eJ[p]); }
            break;
        case MLB_OP_ANISOTROPY:
        case MLB_OP_UNIAXIAL:
        case MLB_OP_CUBIC: {
            o.ch(0);
            o.i32((int)op->asite.size());
            const int per = op->kind == MLB_OP_ANISOTROPY ? 4 : (op->kind == MLB_OP_UNIAXIAL ? 5 : 12);
            for (size_t j = 0; j < op->asite.size(); j++) {
                const double* v = &op->apar[j * per];
                o.i32(op->asite[j]);
                if (op->kind == MLB_OP_CUBIC) {
                    for (int a = 0; a < 6; a++) o.f64(v[a]);     // two axes; the third is computed
                    for (int a = 0; a < 3; a++) o.f64(v[9 + a]);
                } else {
                    for (int a = 0; a < per; a++) o.f64(v[a]);
                }
            }
            break;
        }
        case MLB_OP_THERMAL: {
            o.ch(0);
            o.f64(op->T);
            // the scale array, written by its own encode (object header without type)
            o.ch(kEncNew);
            o.i32(first_index + 1);
            o.ch(0);
            o.i32(op->nx); o.i32(op->ny); o.i32(op->nz);
            const size_t n = (size_t)op->nx * op->ny * op->nz;
            bool same = true;
            for (size_t i = 1; i < op->tscale.size() && same; i++) same = op->tscale[i] == op->tscale[0];
            if (op->tscale.empty() || same) {
                o.i32(1);
                o.f64(op->tscale.empty() ? 1.0 : op->tscale[0]);
            } else {
                o.i32(0);
                o.put(op->tscale.data(), sizeof(double) * n);
            }
            nobj = 2;
            break;
        }
        case MLB_OP_APPLIEDFIELD:
            o.ch(0);
            for (int a = 0; a < 3; a++) o.f64(op->B[a]);
            break;
        case MLB_OP_DIPOLE:
            o.ch(0);
            for (int a = 0; a < 4; a++) o.i32(op->gmax[a]);
            o.f64(op->g);
            for (int a = 0; a < 9; a++) o.f64(op->ABC[a]);
            o.ch(0);
            break;
        }
        put_stream(o, buf, cap, len);
        if (objects) *objects = nobj;
    });
}

int mlb_op_decode(const void* buf, size_t len, mlb_op** out, size_t* used, int* objects)
{
    return guard([&] {
        if (!buf || !out) fail(MLB_EINVAL, "null argument");
        *out = nullptr;
        StreamIn in{static_cast<const char*>(buf), len};
        if (in.i32() != kLuaUserdata) fail(MLB_EINVAL, "malformed stream: expected an object");
        const int32_t tid = in.i32();
        int kind = 0;
        for (int k : {MLB_OP_EXCHANGE, MLB_OP_ANISOTROPY, MLB_OP_UNIAXIAL, MLB_OP_CUBIC, MLB_OP_THERMAL,
                      MLB_OP_APPLIEDFIELD, MLB_OP_DIPOLE})
            if (tid == type_id(op_type_name(k))) kind = k;
        if (!kind) fail(MLB_EUNSUP, "stream does not hold an operator this library reads");
        if (in.ch() != kEncNew) fail(MLB_EINVAL, "malformed stream: bad object flag");
        const int idx = in.i32();
        if (in.ch() != 0) fail(MLB_EUNSUP, "unknown SpinOperation version");
        const int nx = in.i32(), ny = in.i32(), nz = in.i32();
        if (nx <= 0 || ny <= 0 || nz <= 0) fail(MLB_EINVAL, "malformed stream: bad operator size");
        if ((long long)nx * ny * nz > (1LL << 31) - 1) fail(MLB_EUNSUP, "more than 2^31-1 sites");
        const double gs = in.f64();
        mlb_op* op = nullptr;
        ck_rc(mlb_op_create(kind, nx, ny, nz, &op));
        std::unique_ptr<mlb_op> hold(op);
        op->gs = gs;
        int nobj = 1;
        switch (kind) {
        case MLB_OP_EXCHANGE: {
            const int v = in.ch();
            if (v < 0 || v > 1) fail(MLB_EUNSUP, "unknown Exchange version");
            op->normalize = v >= 1 ? in.i32() != 0 : false;   // version 0: old-style, not normalised
            for (int a = 0; a < 3; a++) op->ex_pbc[a] = in.i32();
            const int np = in.i32();
            if (np < 0) fail(MLB_EINVAL, "malformed stream: negative pathway count");
            std::vector<int> f(np), t(np);
            std::vector<double> J(np);
            for (int p = 0; p < np; p++) { f[p] = in.i32(); t[p] = in.i32(); J[p] = in.f64(); }
            ck_rc(mlb_exchange_add_paths(op, f.data(), t.data(), J.data(), np));
            break;
        }
        case MLB_OP_ANISOTROPY:
        case MLB_OP_UNIAXIAL:
        case MLB_OP_CUBIC: {
            if (in.ch() != 0) fail(MLB_EUNSUP, "unknown Anisotropy version");
            const int nops = in.i32();
            if (nops < 0) fail(MLB_EINVAL, "malformed stream: negative count");
            for (int j = 0; j < nops; j++) {
                const int site = in.i32();
                if (kind == MLB_OP_ANISOTROPY) {
                    // Anisotropy::decode stores the axis as written
                    // (addAnisotropy, spinoperationanisotropy.cpp:172-187);
                    // only the Lua add normalises it
                    if (site < 0 || site >= nx * ny * nz) fail(MLB_EINVAL, "malformed stream: site outside");
                    op->asite.push_back(site);
                    for (int a = 0; a < 4; a++) op->apar.push_back(in.f64());
                    op->a_dirty = true;
                } else if (kind == MLB_OP_UNIAXIAL) {
                    // through addAnisotropy, as Uniaxial's decode (it scales by 1/dot(a, a))
                    double ax[3];
                    for (double& v : ax) v = in.f64();
                    const double k1 = in.f64(), k2 = in.f64();
                    ck_rc(mlb_uniaxial_add(op, site, ax, k1, k2));
                } else {
                    double a1[3], a2[3], K[3];
                    for (double& v : a1) v = in.f64();
                    for (double& v : a2) v = in.f64();
                    for (double& v : K) v = in.f64();
                    ck_rc(mlb_cubic_add(op, site, a1, a2, K));
                }
            }
            break;
        }
        case MLB_OP_THERMAL: {
            if (in.ch() != 0) fail(MLB_EUNSUP, "unknown Thermal version");
            op->T = in.f64();
            if (in.ch() != kEncNew) fail(MLB_EUNSUP, "Thermal scale array: expected a new object");
            in.i32();
            if (in.ch() != 0) fail(MLB_EUNSUP, "unknown Array version");
            if (in.i32() != nx || in.i32() != ny || in.i32() != nz) fail(MLB_EINVAL, "scale array size differs");
            const size_t n = (size_t)nx * ny * nz;
            const int flag = in.i32();
            if (flag == 1) {
                const double v = in.f64();
                if (v != 1.0) op->tscale.assign(n, v);
            } else if (flag == 0) {
                op->tscale.resize(n);
                in.take(op->tscale.data(), sizeof(double) * n);
            } else {
                fail(MLB_EINVAL, "malformed stream: bad array flag");
            }
            op->tscale_dirty = !op->tscale.empty();
            nobj = 2;
            break;
        }
        case MLB_OP_APPLIEDFIELD:
            if (in.ch() != 0) fail(MLB_EUNSUP, "unknown AppliedField version");
            for (int a = 0; a < 3; a++) op->B[a] = in.f64();
            break;
        case MLB_OP_DIPOLE: {
            if (in.ch() != 0) fail(MLB_EUNSUP, "unknown LongRange version");
            int gm[4];
            for (int& v : gm) v = in.i32();
            const double g = in.f64();
            double abc[9];
            for (double& v : abc) v = in.f64();
            if (in.ch() != 0) fail(MLB_EUNSUP, "unknown Dipole version");
            for (int a = 0; a < 4; a++) op->gmax[a] = gm[a];
            op->g = g;
            std::memcpy(op->ABC, abc, sizeof(abc));
            break;
        }
        }
        (void)idx;
        if (used) *used = in.pos;
        else if (in.pos != len) fail(MLB_EINVAL, "stream continues after the operator");
        if (objects) *objects = nobj;
        *out = hold.release();
    });
}

int mlb_llg_encode(mlb_llg* l, int first_index, void* buf, size_t cap, size_t* len, int* objects)
{
    return guard([&] {
        if (!l || !len) fail(MLB_EINVAL, "null argument");
        if (first_index < 0) fail(MLB_EINVAL, "negative object index");
        StreamOut o;
        o.header(l->kind == MLB_LLG_QUATERNION ? "LLG.Quaternion" : "LLG.Cartesian", first_index);
        o.ch(1);
        o.i32(l->tof);
        o.i32(l->disable_renorm);
        o.f64(l->precess);
        o.f64(l->damp);
        put_stream(o, buf, cap, len);
        if (objects) *objects = 1;
    });
}

int mlb_llg_decode(const void* buf, size_t len, mlb_llg** out, size_t* used, int* objects)
{
    return guard([&] {
        if (!buf || !out) fail(MLB_EINVAL, "null argument");
        *out = nullptr;
        StreamIn in{static_cast<const char*>(buf), len};
        if (in.i32() != kLuaUserdata) fail(MLB_EINVAL, "malformed stream: expected an object");
        const int32_t tid = in.i32();
        int kind = -1;
        if (tid == type_id("LLG.Cartesian")) kind = MLB_LLG_CARTESIAN;
        if (tid == type_id("LLG.Quaternion")) kind = MLB_LLG_QUATERNION;
        if (kind < 0) fail(MLB_EUNSUP, "stream does not hold an LLG.Cartesian or LLG.Quaternion");
        if (in.ch() != kEncNew) fail(MLB_EINVAL, "malformed stream: bad object flag");
        in.i32();
        // LLG::decode (llg.cpp:62-88): versions 0 and 1, scales from version 1
        const int v = in.ch();
        if (v < 0 || v > 1) fail(MLB_EUNSUP, "unknown LLG version");
        std::unique_ptr<mlb_llg> l(new mlb_llg());
        l->kind = kind;
        l->tof = in.i32();
        l->disable_renorm = in.i32();
        if (v == 1) { l->precess = in.f64(); l->damp = in.f64(); }
        if (used) *used = in.pos;
        else if (in.pos != len) fail(MLB_EINVAL, "stream continues after the LLG object");
        if (objects) *objects = 1;
        *out = l.release();
    });
}

int mlb_llg_kind(const mlb_llg* l, int* kind)
{
    return guard([&] {
        if (!l || !kind) fail(MLB_EINVAL, "null argument");
        *kind = l->kind;
    });
}

int mlb_exchange_set_pbc(mlb_op* op, int px, int py, int pz)
{
    return guard([&] {
        if (!op || op->kind != MLB_OP_EXCHANGE) fail(MLB_EINVAL, "not an Exchange operator");
        op->ex_pbc[0] = px ? 1 : 0; op->ex_pbc[1] = py ? 1 : 0; op->ex_pbc[2] = pz ? 1 : 0;
    });
}

int mlb_exchange_get_pbc(const mlb_op* op, int pbc[3])
{
    return guard([&] {
        if (!op || op->kind != MLB_OP_EXCHANGE) fail(MLB_EINVAL, "not an Exchange operator");
        for (int a = 0; a < 3; a++) pbc[a] = op->ex_pbc[a];
    });
}

int mlb_system_copy(mlb_system* dst, mlb_system* src, int with_fields)
{
    return guard([&] {
        g_version++;
        if (dst->nx != src->nx || dst->ny != src->ny || dst->nz != src->nz) fail(MLB_EINVAL, "size mismatch");
        if (dst->rb != src->rb) fail(MLB_EINVAL, "precision mismatch");
        if (dst == src) return;
        copy_spins(dst, src);
        if (!with_fields) return;   // copySpinsTo: spins and magnitudes only
        const size_t bytes = (size_t)src->rb * src->n;
        dst->alpha = src->alpha; dst->gamma = src->gamma; dst->dt = src->dt; dst->time = src->time;
        CK(cudaStreamSynchronize(dst->st));
        upload_site_array(dst, &dst->sa, nullptr);
        upload_site_array(dst, &dst->sg, nullptr);
        if (src->sa) {
            CK(cudaMalloc(&dst->sa, bytes));
            CK(cudaMemcpy(dst->sa, src->sa, bytes, cudaMemcpyDeviceToDevice));
        }
        if (src->sg) {
            CK(cudaMalloc(&dst->sg, bytes));
            CK(cudaMemcpy(dst->sg, src->sg, bytes, cudaMemcpyDeviceToDevice));
        }
        if (with_fields) {
            materialize_all(src);
            reset_fields(dst);
            for (Slot& x : src->slots) {
                const int j = slot_register(dst, x.name.c_str());
                Slot& y = dst->slots[j];
                y.used = x.used;
                if (x.state == ST_DATA) {
                    slot_alloc(dst, y);
                    for (int c = 0; c < 3; c++)
                        CK(cudaMemcpy(y.h[c], x.h[c], bytes, cudaMemcpyDeviceToDevice));
                    y.state = ST_DATA;
                }
            }
        }
        CK(cudaDeviceSynchronize());
    });
}

// ---------------------------------------------------------------- operators
int mlb_op_create(int kind, int nx, int ny, int nz, mlb_op** out)
{
    return guard([&] {
        if (nx < 1 || ny < 1 || nz < 1) fail(MLB_EINVAL, "dimensions must be positive");
        std::unique_ptr<mlb_op> op(new mlb_op());
        op->kind = kind;
        op->nx = nx; op->ny = ny; op->nz = nz;
        switch (kind) {
        case MLB_OP_EXCHANGE: op->slot = "Exchange"; break;
        case MLB_OP_ANISOTROPY: op->slot = "Anisotropy"; break;
        case MLB_OP_UNIAXIAL: op->slot = "UniaxialAnisotropy"; break;
        case MLB_OP_CUBIC: op->slot = "CubicAnisotropy"; break;
        case MLB_OP_THERMAL: op->slot = "Thermal"; break;
        case MLB_OP_APPLIEDFIELD: op->slot = "Zeeman"; break;
        case MLB_OP_DIPOLE: op->slot = "Dipole"; break;
        case MLB_OP_LONGRANGE: op->slot = "LongRange"; break;
        case MLB_OP_MAGNETOSTATIC: op->slot = "Magnetostatic"; break;
        case MLB_OP_LONGRANGE3D: op->slot = "LongRange3D"; break;
        case MLB_OP_LONGRANGE2D: op->slot = "LongRange2D"; break;
        case MLB_OP_DIPOLE2D: op->slot = "Dipole2D"; break;
        case MLB_OP_MAGNETOSTATICS2D: op->slot = "Magnetostatics2D"; break;
        default: fail(MLB_EINVAL, "unknown operator kind");
        }
        if (is_lr2d(kind)) {
            op->lr2_src.assign(nz, 1.0);
            op->lr2_dst.assign(nz, 1.0);
            op->d2_abc.assign((size_t)nz * 9, 0.0);
            for (int z = 0; z < nz; z++) op->d2_abc[z * 9] = op->d2_abc[z * 9 + 4] = op->d2_abc[z * 9 + 8] = 1.0;
            op->d2_off.assign((size_t)nz * 3, 0.0);
            op->d2_grain.assign((size_t)nz * 3, 1.0);
        }
        *out = op.release();
    });
}

int mlb_op_destroy(mlb_op* op)
{
    return guard([&] {
        g_version++;
        if (!op) return;
        materialize_users(op);
        cudaDeviceSynchronize();
        delete op;
    });
}

int mlb_op_kind(const mlb_op* op, int* kind) { return guard([&] { *kind = op->kind; }); }

int mlb_op_set_scale(mlb_op* op, double gs)
{
    return guard([&] {
        g_version++;
        materialize_users(op);
        op->gs = gs;
    });
}

int mlb_op_get_scale(const mlb_op* op, double* gs) { return guard([&] { *gs = op->gs; }); }

int mlb_op_set_slot_name(mlb_op* op, const char* name)
{
    return guard([&] {
        g_version++;
        if (!name || !*name) fail(MLB_EINVAL, "empty slot name");
        op->slot = name;
    });
}

int mlb_op_get_slot_name(const mlb_op* op, char* buf, size_t len)
{
    return guard([&] {
        if (!buf || len == 0) fail(MLB_EINVAL, "null buffer");
        snprintf(buf, len, "%s", op->slot.c_str());
    });
}

int mlb_op_set_quirks(mlb_op* op, int on)
{
    return guard([&] {
        g_version++;
        materialize_users(op);
        op->quirks = on != 0;
        op->a_dirty = true;
        op->plan_dirty = true;
    });
}

int mlb_op_apply(mlb_op* op, mlb_system* s)
{
    return guard([&] { op_apply(op, s); });
}

int mlb_op_apply_many(mlb_op* op, mlb_system* const* s, int n)
{
    return guard([&] {
        for (int i = 0; i < n; i++) op_apply(op, s[i]);
    });
}

int mlb_exchange_add_path(mlb_op* op, int from, int to, double J)
{
    return guard([&] {
        g_version++;
        if (op->kind != MLB_OP_EXCHANGE) fail(MLB_EINVAL, "not an Exchange operator");
        check_site(op, from);
        check_site(op, to);
        if (J == 0) return; // addPath ignores zero strengths (:330)
        materialize_users(op);
        op->ef.push_back(from); op->et.push_back(to); op->eJ.push_back(J);
        op->ex_dirty = true;
    });
}

int mlb_exchange_add_paths(mlb_op* op, const int* from, const int* to, const double* J, int n)
{
    return guard([&] {
        g_version++;
        if (op->kind != MLB_OP_EXCHANGE) fail(MLB_EINVAL, "not an Exchange operator");
        for (int p = 0; p < n; p++) { check_site(op, from[p]); check_site(op, to[p]); }
        materialize_users(op);
        for (int p = 0; p < n; p++) {
            if (J[p] == 0) continue;
            op->ef.push_back(from[p]); op->et.push_back(to[p]); op->eJ.push_back(J[p]);
        }
        op->ex_dirty = true;
    });
}

int mlb_exchange_set_normalize(mlb_op* op, int on)
{
    return guard([&] {
        g_version++;
        materialize_users(op);
        op->normalize = on != 0;
        op->ex_dirty = true;
    });
}

int mlb_exchange_num_paths(const mlb_op* op, int* n) { return guard([&] { *n = (int)op->ef.size(); }); }

int mlb_anisotropy_add(mlb_op* op, int site, const double axis[3], double K)
{
    return guard([&] {
        g_version++;
        if (op->kind != MLB_OP_ANISOTROPY) fail(MLB_EINVAL, "not an Anisotropy operator");
        check_site(op, site);
        const double len = std::sqrt(axis[0] * axis[0] + axis[1] * axis[1] + axis[2] * axis[2]);
        if (!(len > 0)) return; // l_add: zero axis is not added
        materialize_users(op);
        op->asite.push_back(site);
        for (int a = 0; a < 3; a++) op->apar.push_back(axis[a] / len);
        op->apar.push_back(K);
        op->a_dirty = true;
    });
}

int mlb_uniaxial_add(mlb_op* op, int site, const double axis[3], double K1, double K2)
{
    return guard([&] {
        g_version++;
        if (op->kind != MLB_OP_UNIAXIAL) fail(MLB_EINVAL, "not an Anisotropy.Uniaxial operator");
        check_site(op, site);
        materialize_users(op);
        // addAnisotropy scales by 1/dot(a,a) (..._uniaxial.cpp:172-174)
        const double len = axis[0] * axis[0] + axis[1] * axis[1] + axis[2] * axis[2];
        op->asite.push_back(site);
        for (int a = 0; a < 3; a++) op->apar.push_back(len > 0 ? axis[a] * (1.0 / len) : axis[a]);
        op->apar.push_back(K1);
        op->apar.push_back(K2);
        op->a_dirty = true;
    });
}

int mlb_cubic_add(mlb_op* op, int site, const double a1[3], const double a2[3], const double K[3])
{
    return guard([&] {
        g_version++;
        if (op->kind != MLB_OP_CUBIC) fail(MLB_EINVAL, "not an Anisotropy.Cubic operator");
        check_site(op, site);
        // axis construction of AnisotropyCubic::addAnisotropy (..._cubic.cpp:180-236)
        double u[3] = {a1[0], a1[1], a1[2]}, v[3] = {a2[0], a2[1], a2[2]};
        auto dot = [](const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
        auto cross = [](const double* a, const double* b, double* c) {
            c[0] = a[1] * b[2] - a[2] * b[1];
            c[1] = a[2] * b[0] - a[0] * b[2];
            c[2] = a[0] * b[1] - a[1] * b[0];
        };
        if (dot(u, u) == 0 || dot(v, v) == 0) fail(MLB_EINVAL, "Failed to add anisotropy, are your vectors colinear or empty?");
        double s1 = 1.0 / std::sqrt(dot(u, u));
        for (int a = 0; a < 3; a++) u[a] *= s1;
        double s2 = 1.0 / std::sqrt(dot(v, v));
        for (int a = 0; a < 3; a++) v[a] *= s2;
        if (std::fabs(dot(u, v)) == 1) fail(MLB_EINVAL, "Failed to add anisotropy, are your vectors colinear or empty?");
        if (dot(u, v) != 0) {
            const double d = dot(u, v);
            double p[3] = {u[0] * d, u[1] * d, u[2] * d};
            for (int a = 0; a < 3; a++) v[a] = v[a] + -1 * p[a];
        }
        double ax[9];
        memcpy(ax, u, sizeof(u));
        memcpy(ax + 3, v, sizeof(v));
        cross(ax, ax + 3, ax + 6);
        for (int i = 0; i < 3; i++) {
            const double len = dot(ax + 3 * i, ax + 3 * i);
            if (len > 0) { const double sc = 1.0 / len; for (int a = 0; a < 3; a++) ax[3 * i + a] *= sc; }
        }
        materialize_users(op);
        op->asite.push_back(site);
        for (int a = 0; a < 9; a++) op->apar.push_back(ax[a]);
        for (int a = 0; a < 3; a++) op->apar.push_back(K[a]);
        op->a_dirty = true;
    });
}

int mlb_anisotropy_add_many(mlb_op* op, int n, const int* sites, const double* axes, const double* K)
{
    for (int j = 0; j < n; j++) {
        const int rc = mlb_anisotropy_add(op, sites[j], axes + 3 * j, K[j]);
        if (rc != MLB_OK) return rc;
    }
    return MLB_OK;
}

int mlb_uniaxial_add_many(mlb_op* op, int n, const int* sites, const double* axes, const double* K1,
                          const double* K2)
{
    for (int j = 0; j < n; j++) {
        const int rc = mlb_uniaxial_add(op, sites[j], axes + 3 * j, K1[j], K2[j]);
        if (rc != MLB_OK) return rc;
    }
    return MLB_OK;
}

int mlb_cubic_add_many(mlb_op* op, int n, const int* sites, const double* a1, const double* a2, const double* K)
{
    for (int j = 0; j < n; j++) {
        const int rc = mlb_cubic_add(op, sites[j], a1 + 3 * j, a2 + 3 * j, K + 3 * j);
        if (rc != MLB_OK) return rc;
    }
    return MLB_OK;
}

int mlb_thermal_set_temperature(mlb_op* op, double T)
{
    return guard([&] {
        g_version++;
        if (op->kind != MLB_OP_THERMAL) fail(MLB_EINVAL, "not a Thermal operator");
        op->T = T;
    });
}

int mlb_thermal_get_temperature(const mlb_op* op, double* T) { return guard([&] { *T = op->T; }); }

int mlb_thermal_scale_site(mlb_op* op, int idx, double v)
{
    return guard([&] {
        g_version++;
        if (op->kind != MLB_OP_THERMAL) fail(MLB_EINVAL, "not a Thermal operator");
        const int n = op->nx * op->ny * op->nz;
        if (idx < 0 || idx >= n) return; // scaleSite ignores non-members
        materialize_users(op);
        if (op->tscale.empty()) op->tscale.assign(n, 1.0);
        op->tscale[idx] = v;
        op->tscale_dirty = true;
    });
}

int mlb_thermal_set_seed(mlb_op* op, uint64_t seed)
{
    return guard([&] {
        g_version++;
        materialize_users(op);
        op->seed = seed;
    });
}

int mlb_thermal_set_counter(mlb_op* op, uint64_t counter)
{
    return guard([&] { op->counter = counter; });
}

int mlb_thermal_inject(mlb_op* op, const double* nx, const double* ny, const double* nz)
{
    return guard([&] {
        g_version++;
        if (op->kind != MLB_OP_THERMAL) fail(MLB_EINVAL, "not a Thermal operator");
        const int n = op->nx * op->ny * op->nz;
        const double* src[3] = {nx, ny, nz};
        for (int c = 0; c < 3; c++) {
            op->inj[c].alloc(n);
            CK(cudaMemcpy(op->inj[c].p, src[c], sizeof(double) * n, cudaMemcpyHostToDevice));
        }
        op->inject_pending = true;
    });
}

int mlb_appliedfield_set(mlb_op* op, double bx, double by, double bz)
{
    return guard([&] {
        if (op->kind != MLB_OP_APPLIEDFIELD) fail(MLB_EINVAL, "not an AppliedField operator");
        op->B[0] = bx; op->B[1] = by; op->B[2] = bz;
    });
}

int mlb_appliedfield_get(const mlb_op* op, double out3[3])
{
    return guard([&] { for (int a = 0; a < 3; a++) out3[a] = op->B[a]; });
}

int mlb_appliedfield_set_sweep(mlb_op* op, double dbx, double dby, double dbz)
{
    return guard([&] {
        g_version++; op->dB[0] = dbx; op->dB[1] = dby; op->dB[2] = dbz; });
}

int mlb_longrange_set_strength(mlb_op* op, double g)
{
    return guard([&] {
        g_version++;
        if (!is_conv(op->kind)) fail(MLB_EINVAL, "not a LongRange operator");
        op->g = g;
    });
}

int mlb_longrange_get_strength(const mlb_op* op, double* g) { return guard([&] { *g = op->g; }); }

int mlb_longrange_set_truncation(mlb_op* op, const int gmax[4])
{
    return guard([&] {
        g_version++;
        // l_settrunc (spinoperationlongrange.cpp:505-568): a negative radius
        // is math.huge, stored as -1 in every entry
        if (gmax[0] < 0)
            for (int i = 0; i < 4; i++) op->gmax[i] = -1;
        else
            for (int i = 0; i < 4; i++) op->gmax[i] = gmax[i];
        op->t6_valid = false;
        op->t6_edited = false;
        op->plan_dirty = true;
    });
}

int mlb_dipole_set_huge_rings(mlb_op* op, int rings)
{
    return guard([&] {
        if (!op || op->kind != MLB_OP_DIPOLE) fail(MLB_EINVAL, "not a Dipole operator");
        if (rings < 1) fail(MLB_EINVAL, "at least one ring");
        g_version++;
        op->rings = rings;
        if (op->gmax[0] < 0) { op->t6_valid = false; op->t6_edited = false; op->plan_dirty = true; }
    });
}

int mlb_longrange_get_truncation(const mlb_op* op, int gmax[4])
{
    return guard([&] {
        if (!op || !gmax) fail(MLB_EINVAL, "null argument");
        for (int i = 0; i < 4; i++) gmax[i] = op->gmax[i];
    });
}

int mlb_longrange_set_unit_cell(mlb_op* op, const double ABC[9])
{
    return guard([&] {
        g_version++;
        for (int i = 0; i < 9; i++) op->ABC[i] = ABC[i];
        op->t6_valid = false;
        op->t6_edited = false;
        op->plan_dirty = true;
    });
}

int mlb_magnetostatic_set_cell_dimensions(mlb_op* op, const double d[3])
{
    return guard([&] {
        if (!op || op->kind != MLB_OP_MAGNETOSTATIC) fail(MLB_EINVAL, "not a Magnetostatic operator");
        g_version++;
        for (int a = 0; a < 3; a++) op->mag_prism[a] = d[a];
        op->t6_valid = false;
        op->t6_edited = false;
        op->plan_dirty = true;
    });
}

int mlb_magnetostatic_get_cell_dimensions(const mlb_op* op, double d[3])
{
    return guard([&] {
        if (!op || op->kind != MLB_OP_MAGNETOSTATIC) fail(MLB_EINVAL, "not a Magnetostatic operator");
        for (int a = 0; a < 3; a++) d[a] = op->mag_prism[a];
    });
}

int mlb_magnetostatic_set_crossover_tolerance(mlb_op* op, double tol)
{
    return guard([&] {
        if (!op || op->kind != MLB_OP_MAGNETOSTATIC) fail(MLB_EINVAL, "not a Magnetostatic operator");
        g_version++;
        op->mag_tol = tol;
        op->t6_valid = false;
        op->t6_edited = false;
        op->plan_dirty = true;
    });
}

int mlb_magnetostatic_get_crossover_tolerance(const mlb_op* op, double* tol)
{
    return guard([&] {
        if (!op || op->kind != MLB_OP_MAGNETOSTATIC) fail(MLB_EINVAL, "not a Magnetostatic operator");
        *tol = op->mag_tol;
    });
}

int mlb_longrange_set_open(mlb_op* op, int ox, int oy, int oz)
{
    return guard([&] {
        g_version++;
        if (op->kind != MLB_OP_DIPOLE) fail(MLB_EINVAL, "open boundaries apply to Dipole");
        if (!oz && op->nz > 1) fail(MLB_EUNSUP, "the Dipole layer sum is open in z");
        op->open[0] = ox != 0; op->open[1] = oy != 0; op->open[2] = 1;
        op->t6_valid = false;
        op->plan_dirty = true;
    });
}

static void offset_index(const mlb_op* op, int ox, int oy, int oz, long long* off)
{
    // getsetPattern (spinoperationlongrange.cpp:154-178): wrap in-plane, z in [-nz, nz)
    ox = (ox + 10 * op->nx) % op->nx;
    oy = (oy + 10 * op->ny) % op->ny;
    if (oz < -op->nz || oz >= op->nz) { *off = -1; return; }
    // the reference's offsetOK accepts z = -nz (:144-151), one layer below the
    // stored range; treat it as outside
    if (oz <= -op->nz) { *off = -1; return; }
    *off = ox + (long long)op->nx * (oy + (long long)op->ny * (oz + op->nz - 1));
}

int mlb_longrange_set_matrix(mlb_op* op, int ab, int ox, int oy, int oz, double v)
{
    return guard([&] {
        g_version++;
        if (op->kind != MLB_OP_DIPOLE && op->kind != MLB_OP_LONGRANGE && op->kind != MLB_OP_MAGNETOSTATIC)
            fail(MLB_EINVAL, "not a LongRange operator");
        if (ab < 0 || ab > 5) fail(MLB_EINVAL, "1st argument must be matrix name: XX, XY, XZ, YY, YZ or ZZ");
        if (op->kind == MLB_OP_DIPOLE && (op->open[0] || op->open[1])) fail(MLB_EUNSUP, "open-boundary tensor");
        if (op->kind == MLB_OP_MAGNETOSTATIC && !op->t6_valid) build_magnetostatic_t6(op);
        if (op->kind == MLB_OP_DIPOLE && !op->t6_valid) {
            cudaStream_t st;
            CK(cudaStreamCreate(&st));
            build_plan(op, st, op->plan ? op->plan->rb : 4);
            cudaStreamDestroy(st);
        }
        ensure_t6_layout(op);
        long long off;
        offset_index(op, ox, oy, oz, &off);
        if (off < 0) return;
        materialize_users(op);
        op->t6[ab][off] = v;
        op->t6_valid = true;
        op->t6_edited = true;
        op->plan_dirty = true;
    });
}

int mlb_longrange_get_matrix(mlb_op* op, int ab, int ox, int oy, int oz, double* v)
{
    return guard([&] {
        if (ab < 0 || ab > 5) fail(MLB_EINVAL, "1st argument must be matrix name: XX, XY, XZ, YY, YZ or ZZ");
        if (op->kind == MLB_OP_MAGNETOSTATIC && !op->t6_valid) build_magnetostatic_t6(op);
        if (op->kind == MLB_OP_DIPOLE && !op->t6_valid) {
            cudaStream_t st;
            CK(cudaStreamCreate(&st));
            build_plan(op, st, op->plan ? op->plan->rb : 4);
            cudaStreamDestroy(st);
        }
        ensure_t6_layout(op);
        long long off;
        offset_index(op, ox, oy, oz, &off);
        *v = off < 0 ? 0.0 : op->t6[ab][off];
    });
}

int mlb_longrange_get_tensor(mlb_op* op, double* const t6[6])
{
    return guard([&] {
        if (op->kind == MLB_OP_MAGNETOSTATIC && !op->t6_valid) build_magnetostatic_t6(op);
        if (op->kind == MLB_OP_DIPOLE && !op->t6_valid) {
            if (op->open[0] || op->open[1]) fail(MLB_EUNSUP, "open-boundary tensor has no reference layout");
            cudaStream_t st;
            CK(cudaStreamCreate(&st));
            build_plan(op, st, op->plan ? op->plan->rb : 4);
            cudaStreamDestroy(st);
        }
        ensure_t6_layout(op);
        for (int q = 0; q < 6; q++)
            if (t6[q]) memcpy(t6[q], op->t6[q].data(), sizeof(double) * op->t6[q].size());
    });
}

int mlb_longrange3d_set_tensor(mlb_op* op, int ab, const double* t)
{
    return guard([&] {
        g_version++;
        if (op->kind != MLB_OP_LONGRANGE3D) fail(MLB_EINVAL, "not a LongRange3D operator");
        if (ab < 0 || ab > 8) fail(MLB_EINVAL, "tensor component must be 0..8");
        materialize_users(op);
        const size_t n = (size_t)op->nx * op->ny * op->nz;
        op->t9[ab].assign(t, t + n);
        op->plan_dirty = true;
    });
}

// ---------------------------------------------------------------- LongRange2D / Dipole2D
static void need_lr2d(const mlb_op* op)
{
    if (!op || !is_lr2d(op->kind)) fail(MLB_EINVAL, "not a LongRange2D operator");
}
static void need_layer(const mlb_op* op, int layer)
{
    if (layer < 0 || layer >= op->nz) fail(MLB_EINVAL, "Invalid Layer");
}

int mlb_longrange2d_set_tensor(mlb_op* op, int dest, int src, int ab, const double* t)
{
    return guard([&] {
        g_version++;
        need_lr2d(op);
        need_layer(op, dest);
        need_layer(op, src);
        if (ab < 0 || ab > 8) fail(MLB_EINVAL, "tensor component must be 0..8");
        ensure_t2(op);
        const size_t plane = (size_t)op->nx * op->ny;
        std::copy(t, t + plane, op->t2.begin() + (((size_t)dest * op->nz + src) * 9 + ab) * plane);
    });
}

int mlb_longrange2d_get_tensor(mlb_op* op, int dest, int src, int ab, double* t)
{
    return guard([&] {
        need_lr2d(op);
        need_layer(op, dest);
        need_layer(op, src);
        if (ab < 0 || ab > 8) fail(MLB_EINVAL, "tensor component must be 0..8");
        ensure_t2(op);
        const size_t plane = (size_t)op->nx * op->ny;
        const double* a = op->t2.data() + (((size_t)dest * op->nz + src) * 9 + ab) * plane;
        std::copy(a, a + plane, t);
    });
}

int mlb_longrange2d_set_layer_scales(mlb_op* op, int layer, double src_moment, double dst_field)
{
    return guard([&] {
        g_version++;
        need_lr2d(op);
        need_layer(op, layer);
        op->lr2_src[layer] = src_moment;
        op->lr2_dst[layer] = dst_field;
    });
}

int mlb_longrange2d_get_layer_scales(const mlb_op* op, int layer, double* src_moment, double* dst_field)
{
    return guard([&] {
        need_lr2d(op);
        need_layer(op, layer);
        *src_moment = op->lr2_src[layer];
        *dst_field = op->lr2_dst[layer];
    });
}

int mlb_longrange2d_set_required(mlb_op* op, int new_data, int compile)
{
    return guard([&] {
        g_version++;
        need_lr2d(op);
        if (new_data >= 0) op->lr2_newdata = new_data != 0;
        if (compile >= 0) op->lr2_compile = compile != 0;
    });
}

int mlb_longrange2d_get_required(const mlb_op* op, int* new_data, int* compile)
{
    return guard([&] {
        need_lr2d(op);
        *new_data = op->lr2_newdata ? 1 : 0;
        *compile = op->lr2_compile ? 1 : 0;
    });
}

int mlb_dipole2d_set_unit_cell(mlb_op* op, int layer, const double ABC[9])
{
    return guard([&] {
        need_lr2d(op);
        need_layer(op, layer);
        std::copy(ABC, ABC + 9, op->d2_abc.begin() + (size_t)layer * 9);
    });
}

int mlb_dipole2d_get_unit_cell(const mlb_op* op, int layer, double ABC[9])
{
    return guard([&] {
        need_lr2d(op);
        need_layer(op, layer);
        std::copy(op->d2_abc.begin() + (size_t)layer * 9, op->d2_abc.begin() + (size_t)layer * 9 + 9, ABC);
    });
}

int mlb_dipole2d_set_offset(mlb_op* op, int layer, const double off[3])
{
    return guard([&] {
        need_lr2d(op);
        need_layer(op, layer);
        std::copy(off, off + 3, op->d2_off.begin() + (size_t)layer * 3);
    });
}

int mlb_dipole2d_get_offset(const mlb_op* op, int layer, double off[3])
{
    return guard([&] {
        need_lr2d(op);
        need_layer(op, layer);
        std::copy(op->d2_off.begin() + (size_t)layer * 3, op->d2_off.begin() + (size_t)layer * 3 + 3, off);
    });
}

int mlb_dipole2d_set_truncation(mlb_op* op, const int t[4])
{
    return guard([&] {
        need_lr2d(op);
        for (int i = 0; i < 4; i++) op->d2_trunc[i] = t[i];
    });
}

int mlb_dipole2d_get_truncation(const mlb_op* op, int t[4])
{
    return guard([&] {
        need_lr2d(op);
        for (int i = 0; i < 4; i++) t[i] = op->d2_trunc[i];
    });
}

int mlb_dipole2d_make_data(mlb_op* op)
{
    return guard([&] {
        g_version++;
        if (op && op->kind == MLB_OP_DIPOLE2D) dipole2d_make(op);
        else if (op && op->kind == MLB_OP_MAGNETOSTATICS2D) magnetostatics2d_make(op);
        else fail(MLB_EINVAL, "not a Dipole2D or Magnetostatics2D operator");
    });
}

int mlb_magnetostatics2d_set_grain_size(mlb_op* op, int layer, const double g[3])
{
    return guard([&] {
        need_lr2d(op);
        need_layer(op, layer);
        std::copy(g, g + 3, op->d2_grain.begin() + (size_t)layer * 3);
    });
}

int mlb_magnetostatics2d_get_grain_size(const mlb_op* op, int layer, double g[3])
{
    return guard([&] {
        need_lr2d(op);
        need_layer(op, layer);
        std::copy(op->d2_grain.begin() + (size_t)layer * 3, op->d2_grain.begin() + (size_t)layer * 3 + 3, g);
    });
}

// ---------------------------------------------------------------- LLG
int mlb_llg_create(int kind, mlb_llg** out)
{
    return guard([&] {
        if (kind != MLB_LLG_CARTESIAN && kind != MLB_LLG_QUATERNION) fail(MLB_EINVAL, "unknown LLG type");
        mlb_llg* l = new mlb_llg();
        l->kind = kind;
        *out = l;
    });
}

int mlb_llg_destroy(mlb_llg* l)
{
    return guard([&] {
        g_version++; delete l; });
}

int mlb_llg_set_flags(mlb_llg* l, int tof, int disable_renorm, double precess, double damp)
{
    return guard([&] {
        g_version++;
        l->tof = tof != 0;
        l->disable_renorm = disable_renorm != 0;
        l->precess = precess;
        l->damp = damp;
    });
}

int mlb_llg_apply(mlb_llg* l, mlb_system* from, double scale, mlb_system* dmdt, mlb_system* to, int advance)
{
    return guard([&] {
        if (!from) fail(MLB_EINVAL, "apply requires 1, 2 or 3 SpinSystems");
        if (!dmdt) dmdt = from;
        if (!to) to = from;
        llg_apply(l, from, scale, dmdt, to, advance);
    });
}

// ---------------------------------------------------------------- plans
int mlb_plan_create(mlb_system* s, mlb_op* const* ops, int nops, mlb_llg* l, int timing, mlb_plan** out)
{
    return guard([&] {
        std::unique_ptr<mlb_plan> p(new mlb_plan());
        p->s = s;
        p->ops.assign(ops, ops + nops);
        p->l = l;
        p->timing = timing == 1;
        p->timeline = timing == 2;
        if (p->timeline) {
            p->tl.alloc(4);
            plan_timeline_reset(p.get());
        }
        plan_capture(p.get());
        *out = p.release();
    });
}

int mlb_plan_device_times(mlb_plan* p, double* yz_us, double* xstep_us)
{
    return guard([&] {
        if (!p->timeline) fail(MLB_ESTATE, "not a device-timeline plan (timing = 2)");
        CK(cudaStreamSynchronize(p->s->st));
        unsigned long long t[4];
        CK(cudaMemcpy(t, p->tl.p, sizeof(t), cudaMemcpyDeviceToHost));
        auto span = [](unsigned long long a, unsigned long long b) {
            return (a != ~0ull && b != 0ull && b >= a) ? (double)(b - a) * 1e-3 : -1.0;
        };
        *yz_us = span(t[0], t[1]);
        *xstep_us = span(t[2], t[3]);
        plan_timeline_reset(p);
    });
}

int mlb_plan_launch(mlb_plan* p, int nsteps)
{
    return guard([&] { plan_launch(p, nsteps); });
}

int mlb_plan_kernel_times(mlb_plan* p, int cap, char* names, double* ms, int* count)
{
    return guard([&] {
        CK(cudaStreamSynchronize(p->s->st));
        int k = 0;
        if (p->last)
            for (ProfCaptured& r : *p->last) {
                if (k >= cap) break;
                float t = 0.f;
                CK(cudaEventElapsedTime(&t, r.a, r.b));
                snprintf(names + 48 * k, 48, "%s", r.name);
                ms[k] = t;
                k++;
            }
        *count = k;
    });
}

int mlb_plan_destroy(mlb_plan* p)
{
    return guard([&] {
        if (!p) return;
        plan_release(p);
        delete p;
    });
}

// ---------------------------------------------------------------- fused run
int mlb_run(mlb_system* s, mlb_op* const* ops, int nops, mlb_llg* l, int nsteps)
{
    return guard([&] {
        if (nsteps <= 0) return;
        for (int i = 0; i < nops; i++) check_dims(ops[i], s);
        if (nsteps >= 3) {
            mlb_plan p;
            p.s = s;
            p.ops.assign(ops, ops + nops);
            p.l = l;
            bool ok = true;
            try {
                plan_capture(&p);
            } catch (Err&) {
                ok = false;
            }
            if (ok) {
                plan_launch(&p, nsteps);
                plan_release(&p);
                return;
            }
            plan_release(&p);
        }
        for (int k = 0; k < nsteps; k++) {
            do_step(s, ops, nops, l);
            advance_sweep(ops, nops);
        }
    });
}


// ---------------------------------------------------------------- ensembles
int mlb_ensemble_create(int nrep, const int* dims, mlb_ensemble** out)
{
    return guard([&] {
        if (nrep < 1 || !dims) fail(MLB_EINVAL, "ensemble needs replicas");
        std::unique_ptr<mlb_ensemble> e(new mlb_ensemble());
        e->nrep = nrep;
        // size classes in order of first appearance; replicas packed by class
        std::vector<int> cls_of(nrep);
        for (int r = 0; r < nrep; r++) {
            const int nx = dims[3 * r], ny = dims[3 * r + 1], nz = dims[3 * r + 2];
            if (nx < 1 || ny < 1 || nz < 1) fail(MLB_EINVAL, "dimensions must be positive");
            int k = -1;
            for (size_t j = 0; j < e->cls.size(); j++)
                if (e->cls[j].nx == nx && e->cls[j].ny == ny && e->cls[j].nz == nz) k = (int)j;
            if (k < 0) {
                EnsClass c;
                c.nx = nx; c.ny = ny; c.nz = nz; c.nrep = 0; c.base = 0;
                e->cls.push_back(c);
                k = (int)e->cls.size() - 1;
            }
            cls_of[r] = k;
            e->cls[k].nrep++;
        }
        long long base = 0;
        for (EnsClass& c : e->cls) { c.base = base; base += (long long)c.nx * c.ny * c.nz * c.nrep; }
        if (base > (1LL << 31) - 1) fail(MLB_EUNSUP, "more than 2^31-1 sites in one ensemble");
        e->ntot = base;
        std::vector<int> fill(e->cls.size(), 0);
        e->pos.resize(nrep);
        e->rinfo_h.resize(nrep);
        int packed = 0;
        std::vector<int> first(e->cls.size(), 0);
        for (size_t k = 0; k < e->cls.size(); k++) { first[k] = packed; packed += e->cls[k].nrep; }
        for (int r = 0; r < nrep; r++) {
            const int k = cls_of[r];
            const int p = first[k] + fill[k];
            const EnsClass& c = e->cls[k];
            e->pos[r] = p;
            e->rinfo_h[p] = make_int4(c.nx, c.ny, c.nz, (int)(c.base + (long long)fill[k] * c.nx * c.ny * c.nz));
            fill[k]++;
        }
        CK(cudaStreamCreateWithFlags(&e->own, cudaStreamNonBlocking));
        e->st = e->own;
        for (int b = 0; b < 2; b++)
            for (int c = 0; c < 3; c++) {
                CK(cudaMalloc(&e->sp[b][c], sizeof(float) * e->ntot));
                CK(cudaMemset(e->sp[b][c], 0, sizeof(float) * e->ntot));
            }
        for (int c = 0; c < 3; c++) {
            CK(cudaMalloc(&e->H[c], sizeof(float) * e->ntot));
            CK(cudaMemset(e->H[c], 0, sizeof(float) * e->ntot));
        }
        CK(cudaMalloc(&e->rinfo, sizeof(int4) * nrep));
        CK(cudaMemcpy(e->rinfo, e->rinfo_h.data(), sizeof(int4) * nrep, cudaMemcpyHostToDevice));
        CK(cudaMalloc(&e->dstep, sizeof(DevStep)));
        CK(cudaMemset(e->dstep, 0, sizeof(DevStep)));
        CK(cudaMalloc(&e->mom, sizeof(double) * 6 * nrep));
        CK(cudaMalloc(&e->status, sizeof(unsigned)));
        CK(cudaMemset(e->status, 0, sizeof(unsigned)));
        for (int q = 0; q < 2; q++) {
            CK(cudaMalloc(&e->d_rB[q], sizeof(double) * 3 * nrep));
            CK(cudaMemset(e->d_rB[q], 0, sizeof(double) * 3 * nrep));
        }
        CK(cudaMalloc(&e->d_rdB, sizeof(double) * 3 * nrep));
        CK(cudaMalloc(&e->d_rsig, sizeof(float) * nrep));
        e->rT.assign(nrep, 0.0);
        e->rB.assign(3 * (size_t)nrep, 0.0);
        e->rdB.assign(3 * (size_t)nrep, 0.0);
        CK(cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming));
        for (EnsClass& c : e->cls) {
            CK(cudaStreamCreateWithFlags(&c.st, cudaStreamNonBlocking));
            CK(cudaEventCreateWithFlags(&c.done, cudaEventDisableTiming));
        }
        memset(&e->cfg, 0, sizeof(e->cfg));
        *out = e.release();
    });
}

int mlb_ensemble_destroy(mlb_ensemble* e)
{
    return guard([&] {
        if (!e) return;
        cudaStreamSynchronize(e->st);
        ens_free_graphs(e);
        for (int b = 0; b < 2; b++)
            for (int c = 0; c < 3; c++) cudaFree(e->sp[b][c]);
        for (int c = 0; c < 3; c++) cudaFree(e->H[c]);
        cudaFree(e->rinfo); cudaFree(e->brep); cudaFree(e->bstart); cudaFree(e->dstep); cudaFree(e->mom);
        cudaFree(e->d_rB[0]); cudaFree(e->d_rB[1]); cudaFree(e->d_rdB); cudaFree(e->d_rsig);
        cudaFree(e->status);
        for (EnsClass& c : e->cls) {
            delete c.dip;
            if (c.st) cudaStreamDestroy(c.st);
            if (c.done) cudaEventDestroy(c.done);
        }
        if (e->fork) cudaEventDestroy(e->fork);
        if (e->own) cudaStreamDestroy(e->own);
        delete e;
    });
}

int mlb_ensemble_configure(mlb_ensemble* e, const mlb_ensemble_cfg* cfg)
{
    return guard([&] {
        if (cfg->llg != MLB_LLG_CARTESIAN && cfg->llg != MLB_LLG_QUATERNION) fail(MLB_EINVAL, "unknown LLG type");
        CK(cudaStreamSynchronize(e->st));
        e->cfg = *cfg;
        e->configured = true;
        e->counter = 0;
        for (int r = 0; r < e->nrep; r++) {
            e->rT[r] = cfg->T;
            for (int a = 0; a < 3; a++) { e->rB[3 * r + a] = cfg->B[a]; e->rdB[3 * r + a] = cfg->dB[a]; }
        }
        e->rpar_dirty = true;
        e->tuned = false;
        ens_free_graphs(e);
    });
}

int mlb_ensemble_set_spins(mlb_ensemble* e, int rep, const double* x, const double* y, const double* z)
{
    return guard([&] {
        if (rep < 0 || rep >= e->nrep) fail(MLB_ERANGE, "replica index");
        const int4 ri = e->rinfo_h[e->pos[rep]];
        const int n = ri.x * ri.y * ri.z;
        std::vector<float> f[3];
        const double* src[3] = {x, y, z};
        float m0 = -1.f;
        for (int i = 0; i < n; i++) {
            const float m = (float)std::sqrt(x[i] * x[i] + y[i] * y[i] + z[i] * z[i]);
            if (m0 < 0) m0 = m;
            if (std::fabs(m - m0) > 1e-6f * std::max(1.f, m0)) fail(MLB_EUNSUP, "ensemble spins must share one length");
        }
        if (e->have_ms && std::fabs(m0 - e->ms) > 1e-6f * std::max(1.f, m0))
            fail(MLB_EUNSUP, "ensemble spins must share one length");
        if (!e->have_ms || e->ms != m0) e->rpar_dirty = true;
        ens_download_fields(e);
        e->ms = m0;
        e->have_ms = true;
        CK(cudaStreamSynchronize(e->st));
        for (int c = 0; c < 3; c++) {
            f[c].resize(n);
            for (int i = 0; i < n; i++) f[c][i] = (float)src[c][i];
            CK(cudaMemcpy(e->sp[e->cur][c] + ri.w, f[c].data(), sizeof(float) * n, cudaMemcpyHostToDevice));
        }
    });
}

int mlb_ensemble_get_spins(mlb_ensemble* e, int rep, double* x, double* y, double* z)
{
    return guard([&] {
        if (rep < 0 || rep >= e->nrep) fail(MLB_ERANGE, "replica index");
        const int4 ri = e->rinfo_h[e->pos[rep]];
        const int n = ri.x * ri.y * ri.z;
        std::vector<float> f(n);
        double* dst[3] = {x, y, z};
        CK(cudaStreamSynchronize(e->st));
        for (int c = 0; c < 3; c++) {
            CK(cudaMemcpy(f.data(), e->sp[e->cur][c] + ri.w, sizeof(float) * n, cudaMemcpyDeviceToHost));
            for (int i = 0; i < n; i++) dst[c][i] = f[i];
        }
    });
}

int mlb_ensemble_run(mlb_ensemble* e, int nsteps)
{
    return guard([&] {
        if (nsteps <= 0) return;
        ens_prepare(e);
        DevStep h;
        memset(&h, 0, sizeof(h));
        h.th_counter = e->counter;
        CK(cudaMemcpyAsync(e->dstep, &h, sizeof(h), cudaMemcpyHostToDevice, e->st));
        const bool cart = e->cfg.llg != MLB_LLG_QUATERNION;
        for (int k = 0; k < nsteps; k++) {
            CK(cudaGraphLaunch(e->exec[e->cur], e->st));
            e->cur = 1 - e->cur;
            if (!cart || e->cfg.dt != 0.0) e->time = e->time + e->cfg.dt;
        }
        e->counter += (uint64_t)nsteps;
    });
}

int mlb_ensemble_netmoment(mlb_ensemble* e, double* out8)
{
    return guard([&] {
        const float* s[3] = {e->sp[e->cur][0], e->sp[e->cur][1], e->sp[e->cur][2]};
        CK(mlb::launch_ens_moments(e->rinfo, e->nrep, s, e->mom, e->st));
        std::vector<double> m(6 * (size_t)e->nrep);
        CK(cudaMemcpyAsync(m.data(), e->mom, sizeof(double) * m.size(), cudaMemcpyDeviceToHost, e->st));
        CK(cudaStreamSynchronize(e->st));
        for (int r = 0; r < e->nrep; r++) {
            const double* v = &m[6 * (size_t)e->pos[r]];
            double* o = out8 + 8 * (size_t)r;
            o[0] = v[0]; o[1] = v[1]; o[2] = v[2];
            o[3] = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
            o[4] = v[3]; o[5] = v[4]; o[6] = v[5];
            o[7] = std::sqrt(v[3] * v[3] + v[4] * v[4] + v[5] * v[5]);
        }
    });
}

int mlb_ensemble_info(mlb_ensemble* e, long long* nsites, int* block_size, double* time)
{
    return guard([&] {
        if (nsites) *nsites = e->ntot;
        if (block_size) *block_size = e->bs;
        if (time) *time = e->time;
    });
}

int mlb_ensemble_get_stream(mlb_ensemble* e, void** stream)
{
    return guard([&] { *stream = (void*)e->st; });
}

int mlb_ensemble_status(mlb_ensemble* e, int clear, unsigned* flags)
{
    return guard([&] {
        if (!e || !flags) fail(MLB_EINVAL, "null argument");
        CK(cudaStreamSynchronize(e->st));
        CK(cudaMemcpy(flags, e->status, sizeof(unsigned), cudaMemcpyDeviceToHost));
        if (clear) CK(cudaMemset(e->status, 0, sizeof(unsigned)));
    });
}

int mlb_ensemble_set_replica_params(mlb_ensemble* e, int rep, double T, const double B[3], const double dB[3])
{
    return guard([&] {
        if (!e || !B || !dB) fail(MLB_EINVAL, "null argument");
        if (!e->configured) fail(MLB_ESTATE, "ensemble not configured");
        if (rep < 0 || rep >= e->nrep) fail(MLB_ERANGE, "replica index");
        if (!(T >= 0.0)) fail(MLB_EINVAL, "temperature must be non-negative");
        ens_download_fields(e);
        const int p = e->pos[rep];
        const bool th_before = ens_thermal(e);
        e->rT[p] = T;
        for (int a = 0; a < 3; a++) { e->rB[3 * p + a] = B[a]; e->rdB[3 * p + a] = dB[a]; }
        e->rpar_dirty = true;
        if (ens_thermal(e) != th_before) { e->tuned = false; ens_free_graphs(e); }
    });
}

int mlb_ensemble_get_replica_field(mlb_ensemble* e, int rep, double B[3])
{
    return guard([&] {
        if (!e || !B) fail(MLB_EINVAL, "null argument");
        if (rep < 0 || rep >= e->nrep) fail(MLB_ERANGE, "replica index");
        ens_download_fields(e);
        for (int a = 0; a < 3; a++) B[a] = e->rB[3 * e->pos[rep] + a];
    });
}

int mlb_ensemble_tune_log(mlb_ensemble* e, char* buf, size_t cap, size_t* len)
{
    return guard([&] {
        if (!e || !len) fail(MLB_EINVAL, "null argument");
        *len = e->tune_log.size() + 1;
        if (buf && cap) {
            const size_t n = std::min(cap - 1, e->tune_log.size());
            std::memcpy(buf, e->tune_log.data(), n);
            buf[n] = 0;
        }
    });
}

int mlb_ensemble_config_info(mlb_ensemble* e, int* grid, int* nclasses, int* generic_classes)
{
    return guard([&] {
        if (!e) fail(MLB_EINVAL, "null argument");
        if (grid) *grid = e->grid;
        if (nclasses) *nclasses = (int)e->cls.size();
        if (generic_classes) {
            int g = 0;
            for (EnsClass& c : e->cls) g += c.fast ? 0 : 1;
            *generic_classes = g;
        }
    });
}

} // extern "C"

// ---------------------------------------------------------------- WAB tensor files
// The Dipole tensor cache of the reference (M/cpu/dipole/dipolesupport.cpp:
// 256-643): a Lua file with gmax, nx, ny, nz, the unit cell ABC and, per z
// offset k = -(nz-1) .. nz-1 and component XX, XY, XZ, YY, YZ, ZZ, either
// "NAME[k] = 0" (an all-zero layer) or "NAME[k] = [[" ny lines of nx
// comma-separated numbers "]]", followed by a Lua function parse() that turns
// the strings into tables (the reference's loader runs the file and calls
// it).  The writer here produces that layout with a parse() of its own; the
// reader parses the data lines directly (no Lua needed) and accepts a file
// only when nx, ny, nz, gmax and ABC match the operator, as dipoleParamsMatch
// (:456-560) does.
namespace {

const char* const kWabNames[6] = {"XX", "XY", "XZ", "YY", "YZ", "ZZ"};

void wab_write_layer(FILE* f, const char* name, int k, const double* M, int nx, int ny)
{
    fprintf(f, "\n");
    bool zero = true;
    for (int i = 0; i < nx * ny && zero; i++) zero = M[i] == 0.0;
    if (zero) {
        fprintf(f, "%s[%i] = 0\n", name, k);
        return;
    }
    fprintf(f, "%s[%i] = [[\n", name, k);
    for (int j = 0; j < ny; j++) {
        for (int i = 0; i < nx; i++) {
            const bool last = i == nx - 1 && j == ny - 1;
            const double v = M[i + j * nx];
            if (v == 0.0) fprintf(f, "0%s", last ? "" : ",");
            else fprintf(f, "% .16g%s", v, last ? "" : ",");
        }
        fprintf(f, "\n");
    }
    fprintf(f, "]]\n\n");
}

// Lua that turns each "[[...]]" layer into M[row][col] tables and a "0" layer
// into a table of zeros, written after the data.
const char* const kWabParse =
    "\n"
    "local function rows_of(text)\n"
    "\tlocal M = {}\n"
    "\tfor line in string.gmatch(text, \"[^\\n]+\") do\n"
    "\t\tlocal row = {}\n"
    "\t\tfor v in string.gmatch(line, \"[^,%s]+\") do row[#row + 1] = tonumber(v) end\n"
    "\t\tif #row > 0 then M[#M + 1] = row end\n"
    "\tend\n"
    "\treturn M\n"
    "end\n"
    "\n"
    "local function layer(v)\n"
    "\tif v == 0 then\n"
    "\t\tlocal zrow = setmetatable({}, {__index = function() return 0 end})\n"
    "\t\treturn setmetatable({}, {__index = function() return zrow end})\n"
    "\tend\n"
    "\treturn rows_of(v)\n"
    "end\n"
    "\n"
    "function parse()\n"
    "\tfor _, t in ipairs({XX, XY, XZ, YY, YZ, ZZ}) do\n"
    "\t\tfor k, v in pairs(t) do t[k] = layer(v) end\n"
    "\tend\n"
    "end\n";

bool wab_near(double a, double b) { return fabs(a - b) <= 0.5 * (fabs(a) + fabs(b)) * 1e-6; }

// numbers after `key` up to the end of its statement (a line for scalars, the
// closing braces for tables)
bool wab_numbers_after(const std::string& t, const char* key, std::vector<double>& out, bool& huge)
{
    out.clear();
    huge = false;
    size_t p = t.find(key);
    if (p == std::string::npos) return false;
    p = t.find('=', p);
    if (p == std::string::npos) return false;
    size_t e = t.find('\n', p);
    // tables may span lines: stop at the brace that closes the first one
    size_t q = p + 1;
    while (q < t.size() && (t[q] == ' ' || t[q] == '\t')) q++;
    if (q < t.size() && t[q] == '{') {
        int depth = 0;
        for (size_t r = q; r < t.size(); r++) {
            if (t[r] == '{') depth++;
            else if (t[r] == '}' && --depth == 0) { e = r + 1; break; }
        }
    }
    std::string s = t.substr(p + 1, e == std::string::npos ? std::string::npos : e - p - 1);
    // drop comments
    for (size_t c = s.find("--"); c != std::string::npos; c = s.find("--")) {
        const size_t n = s.find('\n', c);
        s.erase(c, n == std::string::npos ? std::string::npos : n - c);
    }
    if (s.find("math.huge") != std::string::npos) huge = true;
    const char* c = s.c_str();
    while (*c) {
        if ((*c >= '0' && *c <= '9') || *c == '-' || *c == '+' || *c == '.') {
            char* end = nullptr;
            const double v = strtod(c, &end);
            if (end == c) { c++; continue; }
            out.push_back(v);
            c = end;
        } else {
            c++;
        }
    }
    return true;
}

} // namespace

extern "C" {

int mlb_dipole_write_wab(mlb_op* op, const char* filename)
{
    return guard([&] {
        if (!op || !filename) fail(MLB_EINVAL, "null argument");
        if (op->kind != MLB_OP_DIPOLE && op->kind != MLB_OP_LONGRANGE)
            fail(MLB_EINVAL, "not a Dipole or LongRange operator");
        if (op->kind == MLB_OP_DIPOLE && !op->t6_valid) build_plan(op, nullptr, 4);   // the lattice sum
        ensure_t6_layout(op);
        FILE* f = fopen(filename, "w");
        if (!f) fail(MLB_EINVAL, std::string("cannot write ") + filename);
        fprintf(f, "-- This file contains dipole interaction matrices\n\n");
        if (op->gmax[0] < 0)   // dipole_write_matrix (dipolesupport.cpp:360-365)
            fprintf(f, "gmax = {math.huge, math.huge, math.huge, math.huge}  -- radial max, maxX, maxY, maxZ\n");
        else
            fprintf(f, "gmax = {%i, %i, %i, %i} -- radial max, maxX, maxY, maxZ\n", op->gmax[0], op->gmax[1],
                    op->gmax[2], op->gmax[3]);
        fprintf(f, "nx, ny, nz = %i, %i, %i\n", op->nx, op->ny, op->nz);
        const double* A = op->ABC;
        fprintf(f, "ABC = {{%g, %g, %g}, --unit cell\n       {%g, %g, %g},\n       {%g, %g, %g}}\n\n", A[0], A[1],
                A[2], A[3], A[4], A[5], A[6], A[7], A[8]);
        fprintf(f, "XX={} XY={} XZ={} YY={} YZ={} ZZ={}\n");
        const size_t layer = (size_t)op->nx * op->ny;
        for (int c = 0; c < 2 * op->nz - 1; c++)
            for (int q = 0; q < 6; q++)
                wab_write_layer(f, kWabNames[q], c - op->nz + 1, op->t6[q].data() + c * layer, op->nx, op->ny);
        fprintf(f, "%s", kWabParse);
        const bool ok = ferror(f) == 0;
        fclose(f);
        if (!ok) fail(MLB_EINVAL, std::string("error writing ") + filename);
    });
}

int mlb_dipole_read_wab(mlb_op* op, const char* filename)
{
    return guard([&] {
        if (!op || !filename) fail(MLB_EINVAL, "null argument");
        if (op->kind != MLB_OP_DIPOLE && op->kind != MLB_OP_LONGRANGE)
            fail(MLB_EINVAL, "not a Dipole or LongRange operator");
        FILE* f = fopen(filename, "rb");
        if (!f) fail(MLB_ENOTFOUND, std::string("cannot read ") + filename);
        std::string t;
        char buf[65536];
        size_t got;
        while ((got = fread(buf, 1, sizeof(buf), f)) > 0) t.append(buf, got);
        fclose(f);
        // header
        std::vector<double> v;
        bool huge = false;
        if (!wab_numbers_after(t, "nx, ny, nz", v, huge) || v.size() != 3 || (int)v[0] != op->nx ||
            (int)v[1] != op->ny || (int)v[2] != op->nz)
            fail(MLB_EINVAL, "WAB file: nx, ny, nz differ from the operator's");
        if (!wab_numbers_after(t, "gmax", v, huge)) fail(MLB_EINVAL, "WAB file: no gmax");
        if (huge) {
            // gmax = {math.huge, ...}: a file of the extrapolated (ring) sum
            if (op->gmax[0] >= 0) fail(MLB_EINVAL, "WAB file: gmax differs from the operator's");
        } else {
            if (v.size() == 1) v.assign(4, v[0]);   // old files: one radius
            if (v.size() != 4) fail(MLB_EINVAL, "WAB file: malformed gmax");
            for (int i = 0; i < 4; i++)
                if ((int)v[i] != op->gmax[i]) fail(MLB_EINVAL, "WAB file: gmax differs from the operator's");
        }
        if (!wab_numbers_after(t, "ABC", v, huge) || v.size() != 9) fail(MLB_EINVAL, "WAB file: malformed ABC");
        for (int i = 0; i < 9; i++)
            if (!wab_near(v[i], op->ABC[i])) fail(MLB_EINVAL, "WAB file: unit cell differs from the operator's");
        // layers
        const size_t layer = (size_t)op->nx * op->ny;
        std::vector<double> t6[6];
        for (int q = 0; q < 6; q++) t6[q].assign(layer * (2 * op->nz - 1), 0.0);
        std::vector<char> seen((size_t)6 * (2 * op->nz - 1), 0);
        size_t pos = t.find("XX={}");
        if (pos == std::string::npos) fail(MLB_EINVAL, "WAB file: no tensor tables");
        for (;;) {
            size_t best = std::string::npos;
            int q = -1;
            for (int c = 0; c < 6; c++) {
                const std::string key = std::string("\n") + kWabNames[c] + "[";
                const size_t p = t.find(key, pos);
                if (p < best) { best = p; q = c; }
            }
            if (best == std::string::npos) break;
            size_t p = best + 4;   // after "\nXX["
            char* end = nullptr;
            const long k = strtol(t.c_str() + p, &end, 10);
            p = end - t.c_str();
            const size_t eq = t.find('=', p);
            if (eq == std::string::npos || k < -(op->nz - 1) || k > op->nz - 1)
                fail(MLB_EINVAL, "WAB file: malformed layer index");
            const int c = (int)k + op->nz - 1;
            size_t r = eq + 1;
            while (r < t.size() && (t[r] == ' ' || t[r] == '\t')) r++;
            if (t.compare(r, 2, "[[") == 0) {
                const size_t close = t.find("]]", r + 2);
                if (close == std::string::npos) fail(MLB_EINVAL, "WAB file: unterminated layer");
                const char* s = t.c_str() + r + 2;
                const char* stop = t.c_str() + close;
                size_t i = 0;
                while (s < stop) {
                    if (*s == ',' || *s == ' ' || *s == '\n' || *s == '\r' || *s == '\t') { s++; continue; }
                    char* e2 = nullptr;
                    const double x = strtod(s, &e2);
                    if (e2 == s) fail(MLB_EINVAL, "WAB file: malformed number");
                    if (i >= layer) fail(MLB_EINVAL, "WAB file: layer larger than nx*ny");
                    t6[q][c * layer + i++] = x;
                    s = e2;
                }
                if (i != layer) fail(MLB_EINVAL, "WAB file: layer smaller than nx*ny");
                pos = close + 2;
            } else {
                char* e2 = nullptr;
                const double x = strtod(t.c_str() + r, &e2);
                if (e2 == t.c_str() + r || x != 0.0) fail(MLB_EINVAL, "WAB file: malformed zero layer");
                pos = e2 - t.c_str();
            }
            seen[(size_t)q * (2 * op->nz - 1) + c] = 1;
        }
        for (char x : seen)
            if (!x) fail(MLB_EINVAL, "WAB file: missing layers");
        materialize_users(op);
        for (int q = 0; q < 6; q++) op->t6[q].swap(t6[q]);
        op->t6_valid = true;
        op->t6_edited = op->kind == MLB_OP_LONGRANGE;
        op->plan_dirty = true;
        g_version++;
    });
}

} // extern "C"

// ---------------------------------------------------------------- Runge-Kutta integrators
// The reference's make_rk_step_function (M/common/scripts/RungeKutta.lua:
// 57-215) as native host code over the same operations: per step the field
// of the base system, one stage system per Butcher row (a copy of the base
// system, RungeKutta.lua:182-185), each row applied as a chain of
// llg:apply(src, factor, dmdt, dst) calls (istep, :186-193), and the optional
// thermal kick llg:apply(ss, false) (:206-211).  Every call is the library's
// own entry (op_apply, llg_apply), so the time bookkeeping and the arithmetic
// are those of the scripted loop.
struct mlb_rk {
    mlb_system* ss = nullptr;
    std::vector<mlb_system*> k;          // stage systems 2..nstep (owned)
    std::vector<mlb_op*> ops;            // the deterministic field: resetFields, apply each, sumFields
    mlb_llg* l = nullptr;
    mlb_op* temp = nullptr;              // optional Thermal operator
    std::vector<std::vector<double>> bt; // Butcher rows (the c column is not used)
    // Graph steps: a step whose parameters did not change since the previous
    // step is captured (its host logic runs as in an eager step, its kernels
    // are recorded with their dependent-launch edges), the step graph is
    // updated in place and launched.
    bool graph = true;
    cudaGraphExec_t exec = nullptr;
    unsigned long long version = 0;      // g_version at the previous step
    int fail_streak = 0;                 // consecutive captures that failed (3: graph steps off)
    long long graph_steps = 0;           // steps run as graphs
};

namespace {

bool rk_table(const std::string& name, std::vector<std::vector<double>>& bt)
{
    // RungeKutta.lua:100-158
    if (name == "RK1") bt = {{1.0}};
    else if (name == "RK2") bt = {{0.5}, {0.0, 1.0}};
    else if (name == "K3") bt = {{0.5}, {-1.0, 2.0}, {1.0 / 6, 2.0 / 3, 1.0 / 6}};
    else if (name == "RK4") bt = {{0.5}, {0.0, 0.5}, {0.0, 0.0, 1.0}, {1.0 / 6, 1.0 / 3, 1.0 / 3, 1.0 / 6}};
    else if (name == "RK3") bt = {{1.0 / 3}, {0.0, 2.0 / 3}, {0.25, 0.0, 0.75}};
    else if (name == "RK4_38") bt = {{1.0 / 3}, {-1.0 / 3, 1.0}, {1.0, -1.0, 1.0}, {1.0 / 8, 3.0 / 8, 3.0 / 8, 1.0 / 8}};
    else if (name == "RK6")
        bt = {{1.0 / 3},
              {0.0, 2.0 / 3},
              {1.0 / 12, 4.0 / 12, -1.0 / 12},
              {-1.0 / 16, 18.0 / 16, -3.0 / 16, -6.0 / 16},
              {0.0, 9.0 / 8, -3.0 / 8, -6.0 / 8, 4.0 / 8},
              {9.0 / 44, -36.0 / 44, 63.0 / 44, 72.0 / 44, 0.0, -64.0 / 44},
              {11.0 / 120, 0.0, 81.0 / 120, 81.0 / 120, -32.0 / 120, -32.0 / 120, 11.0 / 120}};
    else if (name == "BS3") bt = {{0.5}, {0.0, 0.75}, {2.0 / 9, 1.0 / 3, 4.0 / 9}, {7.0 / 24, 0.25, 1.0 / 3, 1.0 / 8}};
    else return false;
    return true;
}

void rk_field(mlb_rk* r, mlb_system* s)
{
    reset_fields(s);
    for (mlb_op* op : r->ops) op_apply(op, s);
    sum_fields(s);
}

// istep (RungeKutta.lua:186-193): one Butcher row into dst
void rk_row(mlb_rk* r, mlb_system* src, const std::vector<double>& f, mlb_system* dst)
{
    const int nstep = (int)r->bt.size();
    llg_apply(r->l, src, f[0], src, dst, 1);
    for (int i = 2; i <= nstep; i++)
        if (i <= (int)f.size() && f[i - 1] != 0.0) llg_apply(r->l, dst, f[i - 1], r->k[i - 2], dst, 1);
}

// sfunc (RungeKutta.lua:194-213) on the base system ss (the script's
// ss_input, default the system the scheme was made for)
void rk_step(mlb_rk* r, mlb_system* ss, bool skip_temperature)
{
    const int nstep = (int)r->bt.size();
    rk_field(r, ss);
    for (int i = 1; i <= nstep - 1; i++) {
        mlb_system* d = r->k[i - 1];   // ss_k[i+1]
        d->dt = ss->dt;
        rk_row(r, ss, r->bt[i - 1], d);
        rk_field(r, d);
    }
    rk_row(r, ss, r->bt[nstep - 1], ss);
    if (r->temp && !skip_temperature) {
        reset_fields(ss);
        op_apply(r->temp, ss);
        sum_fields(ss);
        llg_apply(r->l, ss, 1.0, ss, ss, 0);
    }
}

// One step of r on its own system as a graph (see mlb_rk): false when it
// must run eagerly (parameters changed since the previous step, injected
// noise pending, a surrogate attached, graph steps off or failing).
bool rk_graph_ok(mlb_rk* r)
{
    if (!r->graph || r->fail_streak >= 3 || r->version != g_version || r->ss->sur) return false;
    for (mlb_system* c : r->k)
        if (c->st != r->ss->st) return false;
    for (mlb_op* o : r->ops)
        if (o->inject_pending) return false;
    if (r->temp && r->temp->inject_pending) return false;
    return true;
}

void rk_step_graph(mlb_rk* r)
{
    mlb_system* ss = r->ss;
    std::vector<mlb_op*> all = r->ops;
    if (r->temp) all.push_back(r->temp);
    std::vector<mlb_system*> sys = {ss};
    for (mlb_system* c : r->k) sys.push_back(c);
    std::vector<HostState> saved;
    for (mlb_system* x : sys) saved.push_back(save_state(x, all));
    for (mlb_system* x : sys) nm_guard(x, -1);   // no waits on outside events inside the capture
    cudaStream_t st = ss->st;
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    bool ok = true;
    try {
        rk_step(r, ss, false);
        for (mlb_system* x : sys) flush_pending(x);
    } catch (Err&) {
        ok = false;
    }
    const cudaError_t e = cudaStreamEndCapture(st, &g);
    if (!ok || e != cudaSuccess || !g) {
        // nothing was launched: put the bookkeeping back and run the step eagerly
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        for (size_t i = 0; i < sys.size(); i++) {
            load_state(sys[i], all, saved[i]);
            sys[i]->spec_token = 0;
        }
        r->fail_streak++;
        rk_step(r, ss, false);
        return;
    }
    if (r->exec) {
        cudaGraphExecUpdateResultInfo info;
        if (cudaGraphExecUpdate(r->exec, g, &info) != cudaSuccess) {
            cudaGetLastError();
            cudaGraphExecDestroy(r->exec);
            r->exec = nullptr;
        }
    }
    cudaError_t ie = cudaSuccess;
    if (!r->exec) ie = cudaGraphInstantiate(&r->exec, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) {
        r->exec = nullptr;
        fail(MLB_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(ie));
    }
    CK(cudaGraphLaunch(r->exec, st));
    r->fail_streak = 0;
    r->graph_steps++;
}

} // namespace

extern "C" {

int mlb_rk_create(mlb_system* ss, const char* type, mlb_op* const* ops, int nops, mlb_llg* l, mlb_op* temp,
                  mlb_rk** out)
{
    return guard([&] {
        if (!ss || !l || !out || !type || (nops > 0 && !ops)) fail(MLB_EINVAL, "null argument");
        std::unique_ptr<mlb_rk> r(new mlb_rk());
        if (!rk_table(type, r->bt))
            fail(MLB_EINVAL, "RK type must be one of \"RK1\", \"RK2\", \"K3\", \"RK4\", \"RK3\", \"RK4_38\", \"RK6\", \"BS3\"");
        for (int i = 0; i < nops; i++) {
            check_dims(ops[i], ss);
            r->ops.push_back(ops[i]);
        }
        if (temp) {
            if (temp->kind != MLB_OP_THERMAL) fail(MLB_EINVAL, "the optional operator must be a Thermal");
            check_dims(temp, ss);
        }
        r->ss = ss;
        r->l = l;
        r->temp = temp;
        // stage systems: copies of the base system on its stream (ss_k[i] = ss_k[1]:copy())
        const int nstep = (int)r->bt.size();
        try {
            for (int i = 2; i <= nstep; i++) {
                mlb_system* c = make_system(ss->nx, ss->ny, ss->nz, ss->rb);
                r->k.push_back(c);
                int rc = mlb_system_copy(c, ss, 1);
                if (rc) fail(rc, g_err);
                c->st = ss->st;
                c->internal = true;
            }
        } catch (...) {
            for (mlb_system* c : r->k) free_system(c);
            throw;
        }
        *out = r.release();
    });
}

int mlb_rk_step(mlb_rk* r, int nsteps)
{
    return guard([&] {
        for (int k = 0; k < nsteps; k++) {
            if (rk_graph_ok(r)) rk_step_graph(r);
            else rk_step(r, r->ss, false);
            r->version = g_version;
        }
    });
}

int mlb_rk_set_graph(mlb_rk* r, int on)
{
    return guard([&] {
        if (!r) fail(MLB_EINVAL, "null scheme");
        r->graph = on != 0;
        r->fail_streak = 0;
    });
}

int mlb_rk_graph_steps(mlb_rk* r, long long* steps)
{
    return guard([&] {
        if (!r || !steps) fail(MLB_EINVAL, "null argument");
        *steps = r->graph_steps;
    });
}

int mlb_rk_step_on(mlb_rk* r, mlb_system* ss, int skip_temperature)
{
    return guard([&] {
        if (ss->nx != r->ss->nx || ss->ny != r->ss->ny || ss->nz != r->ss->nz || ss->rb != r->ss->rb)
            fail(MLB_EINVAL, "SpinSystem differs in size or precision from the scheme's");
        rk_step(r, ss, skip_temperature != 0);
    });
}

int mlb_rk_destroy(mlb_rk* r)
{
    return guard([&] {
        if (!r) return;
        if (r->exec) cudaGraphExecDestroy(r->exec);
        for (mlb_system* c : r->k) free_system(c);
        delete r;
    });
}

} // extern "C"

// ---------------------------------------------------------------- adaptive time step
// make_adapt_step_function (M/common/scripts/AdaptiveTimeStep.lua:9-110)
// over a Runge-Kutta scheme: a full step of dt on one copy and two steps of
// dt/2 on another, compared with SpinSystem::diff; accepted when the
// difference is below the tolerance (the half-step result is kept, the time
// step grows by 1 + clamp(e^2, 0.1, 0.5) - 0.1 with e = (tol - diff)/tol),
// otherwise the time step halves.  The optional dynamics function of the
// script is not part of this entry.
struct mlb_adapt {
    mlb_system* ss = nullptr;
    mlb_system* s2 = nullptr;   // full step (owned copy)
    mlb_system* s3 = nullptr;   // two half steps (owned copy)
    mlb_rk* step = nullptr;
    double tol = 0.0;
    mlb_llg* l = nullptr;
    mlb_op* temp = nullptr;
};

namespace {

bool adapt_step(mlb_adapt* a)
{
    mlb_system* s = a->ss;
    mlb_system* s2 = a->s2;
    mlb_system* s3 = a->s3;
    s2->time = s->time;
    s3->time = s->time;
    s2->dt = s->dt;
    s3->dt = s->dt / 2;
    copy_spins(s2, s);
    copy_spins(s3, s);
    rk_step(a->step, s2, true);
    rk_step(a->step, s3, true);
    rk_step(a->step, s3, true);
    double d4[4];
    system_diff(s2, s3, d4);
    const bool same = d4[3] < a->tol;
    double ee = (a->tol - d4[3]) / a->tol;
    if (same) {
        copy_spins(s, s3);
        if (a->temp) {
            reset_fields(s);
            op_apply(a->temp, s);
            sum_fields(s);
            llg_apply(a->l, s, 1.0, s, s, 0);
        }
        s->time = s3->time;
        ee = ee * ee;
        if (ee > 0.5) ee = 0.5;
        if (ee < 0.1) ee = 0.1;
        s->dt = s->dt * (1 + ee - 0.1);
    } else {
        s->dt = s->dt * 0.5;
    }
    return same;
}

} // namespace

extern "C" {

int mlb_adapt_create(mlb_system* ss, mlb_rk* step, double tolerance, mlb_llg* l, mlb_op* temp, mlb_adapt** out)
{
    return guard([&] {
        if (!ss || !step || !out) fail(MLB_EINVAL, "null argument");
        if (ss->nx != step->ss->nx || ss->ny != step->ss->ny || ss->nz != step->ss->nz || ss->rb != step->ss->rb)
            fail(MLB_EINVAL, "SpinSystem differs in size or precision from the scheme's");
        if (temp && (temp->kind != MLB_OP_THERMAL || !l)) fail(MLB_EINVAL, "a Thermal operator needs the LLG operator");
        std::unique_ptr<mlb_adapt> a(new mlb_adapt());
        a->ss = ss;
        a->step = step;
        a->tol = tolerance;
        a->l = l;
        a->temp = temp;
        for (mlb_system** c : {&a->s2, &a->s3}) {
            *c = make_system(ss->nx, ss->ny, ss->nz, ss->rb);
            int rc = mlb_system_copy(*c, ss, 1);
            if (rc) {
                free_system(a->s2);
                free_system(a->s3);
                fail(rc, g_err);
            }
            (*c)->st = ss->st;
            (*c)->internal = true;
        }
        *out = a.release();
    });
}

int mlb_adapt_step(mlb_adapt* a, int* accepted)
{
    return guard([&] {
        const bool ok = adapt_step(a);
        if (accepted) *accepted = ok ? 1 : 0;
    });
}

int mlb_adapt_destroy(mlb_adapt* a)
{
    return guard([&] {
        if (!a) return;
        free_system(a->s2);
        free_system(a->s3);
        delete a;
    });
}

} // extern "C"

// ---------------------------------------------------------------- learned surrogate
struct mlb_surrogate {
    mlb_op* op = nullptr;
    int nx = 0, ny = 0, nz = 0, n = 0;
    SurK k{};
    int nw = 0, nr = 0;
    double g_train = 0.0;       // operator strength x global scale the parameters were trained at
    int adam_step = 0;
    int kint = 10;              // exact evaluation every kint steps
    double tol = 1e-3;          // bound on the estimated relative field error
    double eps = 0.1;           // validated relative error of the predicted update
    DBuf<float> w, r, gw, gr, mw, vw, mr, vr;
    DBuf<uint8_t> wc, Fc;
    DBuf<__nv_bfloat16> F;
    DBuf<float2> twy, Xp, Yh, Zh, Gh;
    DBuf<uint4> Xb;             // BF16 input records [CP/8][ny][nx] for the output kernel
    DBuf<uint8_t> Zb;           // per-row B tiles of the mixed spectrum [ny][CP x 32 BF16]
    DBuf<unsigned int> ycnt;    // per-kx arrival counters of the y-DFT
    DBuf<float> m0[3], h0[3], P[3], G[3], part;
    DBuf<double> lpart, lsum;
    DBuf<int> err;
    DBuf<SurDev> dev;
    DBuf<double> rpart;         // per-CTA residual sums of the output kernel
    int rnp = 0;
    int lnb = 1;
    long long stats[3] = {0, 0, 0};
    double last_bound = 0.0;
};

namespace {

uint16_t host_bf16(float f)
{
    uint32_t u;
    memcpy(&u, &f, 4);
    if ((u & 0x7f800000u) == 0x7f800000u) return (uint16_t)(u >> 16);
    const uint32_t lsb = (u >> 16) & 1u;
    u += 0x7fffu + lsb;           // round to nearest even
    return (uint16_t)(u >> 16);
}

void sur_upload_w(mlb_surrogate* S, const std::vector<float>& w)
{
    const int C = S->k.C, CP = S->k.CP, no = (2 * S->k.rad + 1) * (2 * S->k.rad + 1);
    std::vector<uint16_t> t((size_t)no * CP * CP, 0);
    for (int o = 0; o < no; o++)
        for (int co = 0; co < C; co++)
            for (int ci = 0; ci < C; ci++) {
                const size_t byte = (size_t)(co >> 3) * (CP / 8) * 128 + (ci >> 3) * 128 + (co & 7) * 16 + (ci & 7) * 2;
                t[(size_t)o * CP * CP + byte / 2] = host_bf16(w[((size_t)o * C + co) * C + ci]);
            }
    CK(cudaMemcpy(S->wc.p, t.data(), t.size() * 2, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(S->w.p, w.data(), sizeof(float) * w.size(), cudaMemcpyHostToDevice));
}

void sur_check_err(mlb_surrogate* S)
{
    int e = 0;
    CK(cudaMemcpy(&e, S->err.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) {
        CK(cudaMemset(S->err.p, 0, sizeof(int)));
        fail(MLB_ECUDA, "tensor-core completion wait gave up (results of that launch are invalid)");
    }
}

// dH (mode 1) or H0 + ratio dH (mode 0, with residual statistics in dev) for
// a = m, b = m0 (b may be null: the input is a itself).
void sur_forward(mlb_surrogate* S, const float* const a[3], const float* const b[3], int mode,
                 const float* const h0[3], float* const out[3], SurDev* dev, const int* skip, float ratio,
                 cudaStream_t st)
{
    SurK k = S->k;
    k.skip_if = skip;
    k.ratio = ratio;
    CK(mlb::launch_sur_xdft(k, a, b, S->F.p, S->Xp.p, S->Xb.p, S->err.p, st));
    CK(mlb::launch_sur_ydft(k, S->Xp.p, S->twy.p, reinterpret_cast<const float2*>(S->r.p), S->Yh.p, S->Zh.p,
                            S->ycnt.p, st));
    CK(mlb::launch_sur_zrows(k, S->Zh.p, S->twy.p, S->Zb.p, st));
    CK(mlb::launch_sur_out(k, S->Xb.p, h0, out, S->wc.p, S->Fc.p, S->Zb.p, dev, mode == 1 ? nullptr : S->rpart.p,
                           S->err.p, mode, st));
}

// Loss, gradients and one Adam step for the pair (a - b, hx - h0) (h0 may be
// null: target hx); leaves sum T^2, sum (P - T)^2, sum hx^2 in lsum.
void sur_train_iter(mlb_surrogate* S, const float* const a[3], const float* const b[3], const float* const hx[3],
                    const float* const h0[3], double lr, bool update, cudaStream_t st)
{
    float* P[3] = {S->P[0].p, S->P[1].p, S->P[2].p};
    float* G[3] = {S->G[0].p, S->G[1].p, S->G[2].p};
    const float* Gc[3] = {G[0], G[1], G[2]};
    sur_forward(S, a, b, 1, nullptr, P, nullptr, nullptr, 1.f, st);
    const float* Pc[3] = {P[0], P[1], P[2]};
    CK(mlb::launch_sur_loss(S->n, Pc, hx, h0, G, S->lpart.p, S->lnb, S->lsum.p, st));
    SurK k = S->k;
    k.skip_if = nullptr;
    CK(mlb::launch_sur_xdft(k, Gc, nullptr, S->F.p, S->Xp.p, nullptr, S->err.p, st));
    CK(mlb::launch_sur_ydft(k, S->Xp.p, S->twy.p, nullptr, S->Gh.p, nullptr, S->ycnt.p, st));
    CK(mlb::launch_sur_grad_r(k, S->Gh.p, S->Yh.p, reinterpret_cast<float2*>(S->gr.p), st));
    CK(mlb::launch_sur_grad_w(k, a, b, Gc, S->part.p, S->gw.p, st));
    if (!update) return;
    S->adam_step++;
    CK(mlb::launch_sur_adam(S->w.p, S->r.p, S->gw.p, S->gr.p, S->mw.p, S->vw.p, S->mr.p, S->vr.p, S->wc.p,
                            S->lsum.p, (float)lr, S->adam_step, S->nw, S->nr, S->k.C, S->k.CP, st));
}

void sur_check_use(mlb_surrogate* S, mlb_system* ss, mlb_op* const* ops, int nops)
{
    if (ss->rb != 4) fail(MLB_EUNSUP, "the surrogate runs on FP32 systems");
    if (ss->nx != S->nx || ss->ny != S->ny || ss->nz != S->nz) fail(MLB_EINVAL, "surrogate and SpinSystem sizes differ");
    bool found = false;
    for (int i = 0; i < nops; i++) {
        check_dims(ops[i], ss);
        if (ops[i] == S->op) found = true;
    }
    if (!found) fail(MLB_EINVAL, "the surrogate's operator is not among the step's operators");
}

void sur_snapshot_now(mlb_surrogate* S, mlb_system* ss, const Slot& sl)
{
    for (int c = 0; c < 3; c++) {
        CK(cudaMemcpyAsync(S->m0[c].p, ss->sp[ss->cur][c], sizeof(float) * S->n, cudaMemcpyDeviceToDevice, ss->st));
        CK(cudaMemcpyAsync(S->h0[c].p, sl.h[c], sizeof(float) * S->n, cudaMemcpyDeviceToDevice, ss->st));
    }
}

// One canonical step with the hook point after the operators: f(step) runs
// with the surrogate operator's exact field in its slot.
template <class Fn>
void plain_step_with(mlb_system* ss, mlb_op* const* ops, int nops, mlb_llg* l, mlb_surrogate* S, Fn&& f)
{
    reset_fields(ss);
    for (int i = 0; i < nops; i++) op_apply(ops[i], ss);
    const int si = slot_find(ss, S->op->slot.c_str());
    materialize(ss, si);
    f(ss->slots[si]);
    sum_fields(ss);
    llg_apply(l, ss, 1.0, ss, ss, 1);
    advance_sweep(ops, nops);
}

} // namespace

namespace {

// The surrogate's operator field of this step: the network's field (skipped
// on exact steps), the exact passes (run on exact steps only), and the
// snapshot m0 = m, H0 = H after an exact evaluation; the device schedule
// decides which, so a captured step holds both.
bool sur_hook(mlb_op* op, mlb_system* s, Slot& sl)
{
    mlb_surrogate* S = s->sur;
    if (S->op != op || s->rb != 4) return false;
    SurDev* d = S->dev.p;
    const float* a[3];
    const float* b[3] = {S->m0[0].p, S->m0[1].p, S->m0[2].p};
    const float* h0[3] = {S->h0[0].p, S->h0[1].p, S->h0[2].p};
    float* out[3];
    for (int c = 0; c < 3; c++) {
        a[c] = static_cast<const float*>(s->sp[s->cur][c]);
        out[c] = static_cast<float*>(sl.h[c]);
    }
    const float ratio = S->g_train > 0 ? (float)(op->g * op->gs / S->g_train) : 1.f;
    sur_forward(S, a, b, 0, h0, out, d, &d->exact, ratio, s->st);
    ConvPlan& P = *op->plan;
    if (!s->capturing) P.spec_token = 0;
    ConvK kk = P.k;
    kk.run_if = &d->exact;
    if (mlb::conv_fast_ok(kk)) {
        CK(mlb::launch_conv_fast(kk, P.L, reinterpret_cast<const float2*>(P.tw.p), a,
                                 reinterpret_cast<float2*>(P.spec.p), reinterpret_cast<const float*>(P.ten6.p), out,
                                 s->st));
    } else {
        const void* av[3] = {a[0], a[1], a[2]};
        void* ov[3] = {out[0], out[1], out[2]};
        CK(mlb::launch_conv(kk, P.L[0], P.L[1], P.L[2], P.tw.p, av, P.spec.p, P.ten6.p, P.ten9.p, ov, 4, s->st));
    }
    const float* hc[3] = {out[0], out[1], out[2]};
    float* sm[3] = {S->m0[0].p, S->m0[1].p, S->m0[2].p};
    float* sh[3] = {S->h0[0].p, S->h0[1].p, S->h0[2].p};
    CK(mlb::launch_sur_snapshot(d, S->n, a, hc, sm, sh, s->st));
    return true;
}

void sur_advance(mlb_system* s)
{
    CK(mlb::launch_sur_advance(s->sur->dev.p, s->sur->rpart.p, s->sur->rnp, s->st));
}

} // namespace

extern "C" {

int mlb_surrogate_set_wait_limit(mlb_surrogate* s, unsigned polls)
{
    return guard([&] {
        if (!s) fail(MLB_EINVAL, "null surrogate");
        g_version++;   // captured steps carry the limit: capture again
        s->k.wait_polls = polls;
    });
}

int mlb_surrogate_create(mlb_op* op, int mx, int my, int rad, mlb_surrogate** out)
{
    return guard([&] {
        if (!op || !out) fail(MLB_EINVAL, "null argument");
        if (op->kind != MLB_OP_DIPOLE && op->kind != MLB_OP_LONGRANGE)
            fail(MLB_EINVAL, "the surrogate stands in for a Dipole or LongRange operator");
        const int nx = op->nx, ny = op->ny, nz = op->nz, C = 3 * nz;
        if (C > 32) fail(MLB_EUNSUP, "more than 10 layers in z");
        const int CP = C <= 16 ? 16 : 32;
        if (nx % 128 != 0) fail(MLB_EUNSUP, "nx must be a multiple of 128");
        if (ny % (128 / CP) != 0 || ny % 4 != 0) fail(MLB_EUNSUP, "ny must be a multiple of 8 (of 4 above 16 channels)");
        if (mx < 1 || mx > 16 || mx > nx / 2) fail(MLB_EINVAL, "modes_x must be in 1..16 and at most nx/2");
        if (my < 2 || my > 16 || my % 2 || my > ny) fail(MLB_EINVAL, "modes_y must be even, in 2..16, at most ny");
        if (rad < 0 || rad > 3) fail(MLB_EINVAL, "radius must be in 0..3");
        if (mlb::sur_out_smem(CP, rad) > 226 * 1024) fail(MLB_EUNSUP, "stencil too large for shared memory");
        std::unique_ptr<mlb_surrogate> S(new mlb_surrogate());
        S->op = op;
        S->nx = nx; S->ny = ny; S->nz = nz; S->n = nx * ny * nz;
        SurK& k = S->k;
        k.nx = nx; k.ny = ny; k.nz = nz; k.C = C; k.CP = CP; k.mx = mx; k.my = my; k.rad = rad;
        k.nxc = nx / 64; k.skip_if = nullptr; k.ratio = 1.f; k.wait_polls = 1u << 24;
        const int dia = 2 * rad + 1;
        S->nw = dia * dia * C * C;
        S->nr = mx * my * C * C * 2;
        for (DBuf<float>* b : {&S->w, &S->gw, &S->mw, &S->vw}) { b->alloc(S->nw); CK(cudaMemset(b->p, 0, sizeof(float) * S->nw)); }
        for (DBuf<float>* b : {&S->r, &S->gr, &S->mr, &S->vr}) { b->alloc(S->nr); CK(cudaMemset(b->p, 0, sizeof(float) * S->nr)); }
        S->wc.alloc((size_t)dia * dia * CP * CP * 2);
        CK(cudaMemset(S->wc.p, 0, S->wc.n));
        // forward x-DFT rows [2 kx + ri][x] and inverse rows in the canonical A layout
        std::vector<uint16_t> F((size_t)32 * nx, 0), Fc((size_t)nx * 32, 0);
        for (int kx = 0; kx < mx; kx++)
            for (int x = 0; x < nx; x++) {
                const double th = 2.0 * M_PI * (double)((long long)kx * x % nx) / nx;
                const uint16_t c = host_bf16((float)std::cos(th)), s = host_bf16((float)-std::sin(th));
                F[(size_t)(2 * kx) * nx + x] = c;
                F[(size_t)(2 * kx + 1) * nx + x] = s;
                for (int ri = 0; ri < 2; ri++) {
                    const int kk = 2 * kx + ri;
                    const size_t byte = (size_t)(x >> 3) * 512 + (kk >> 3) * 128 + (x & 7) * 16 + (kk & 7) * 2;
                    Fc[byte / 2] = ri ? s : c;
                }
            }
        S->F.alloc(F.size());
        CK(cudaMemcpy(S->F.p, F.data(), F.size() * 2, cudaMemcpyHostToDevice));
        S->Fc.alloc(Fc.size() * 2);
        CK(cudaMemcpy(S->Fc.p, Fc.data(), Fc.size() * 2, cudaMemcpyHostToDevice));
        std::vector<float2> twy((size_t)my * ny);
        for (int j = 0; j < my; j++) {
            const int ky = j < my / 2 ? j : ny - my + j;
            for (int y = 0; y < ny; y++) {
                const double th = 2.0 * M_PI * (double)((long long)ky * y % ny) / ny;
                twy[(size_t)j * ny + y] = make_float2((float)std::cos(th), (float)-std::sin(th));
            }
        }
        S->twy.alloc(twy.size());
        CK(cudaMemcpy(S->twy.p, twy.data(), sizeof(float2) * twy.size(), cudaMemcpyHostToDevice));
        S->Xp.alloc((size_t)k.nxc * mx * C * ny);
        S->Yh.alloc((size_t)mx * my * C);
        S->Gh.alloc((size_t)mx * my * C);
        S->Zh.alloc((size_t)mx * my * C);
        S->Xb.alloc((size_t)(CP / 8) * nx * ny);
        S->Zb.alloc((size_t)ny * CP * 64);
        CK(cudaMemset(S->Zb.p, 0, S->Zb.n));
        S->ycnt.alloc(16);
        CK(cudaMemset(S->ycnt.p, 0, sizeof(unsigned int) * 16));
        if (mlb::sur_ydft_smem(k) > 128 * 1024) fail(MLB_EUNSUP, "ny too large for the y-DFT of this build");
        if (sizeof(float2) * (mx * my * C + my * 4) > 128 * 1024) fail(MLB_EUNSUP, "too many retained modes");
        for (int c = 0; c < 3; c++) {
            for (DBuf<float>* b : {&S->m0[c], &S->h0[c], &S->P[c], &S->G[c]}) {
                b->alloc(S->n);
                CK(cudaMemset(b->p, 0, sizeof(float) * S->n));
            }
        }
        S->part.alloc((size_t)(nx / 128) * (ny / 4) * S->nw);
        S->lnb = (int)std::min<long long>(1024, std::max<long long>(1, (3LL * S->n + 255) / 256));
        S->lpart.alloc((size_t)S->lnb * 3);
        S->lsum.alloc(3);
        S->err.alloc(1);
        CK(cudaMemset(S->err.p, 0, sizeof(int)));
        S->dev.alloc(1);
        S->rnp = mlb::sur_out_ctas(nx, ny);
        S->rpart.alloc((size_t)2 * S->rnp);

        SurDev h{};
        h.exact = 1;
        h.k = S->kint;
        h.eps = (float)S->eps;
        h.tol = (float)S->tol;
        CK(cudaMemcpy(S->dev.p, &h, sizeof(h), cudaMemcpyHostToDevice));
        CK(cudaDeviceSynchronize());
        *out = S.release();
    });
}

int mlb_surrogate_destroy(mlb_surrogate* s)
{
    return guard([&] {
        for (mlb_system* x : g_systems)
            if (x->sur == s) x->sur = nullptr;
        cudaDeviceSynchronize();
        delete s;
    });
}

int mlb_surrogate_sizes(const mlb_surrogate* s, int out[7])
{
    return guard([&] {
        out[0] = s->k.C; out[1] = s->k.CP; out[2] = s->k.mx; out[3] = s->k.my; out[4] = s->k.rad;
        out[5] = s->nw; out[6] = s->nr;
    });
}

int mlb_surrogate_get_params(mlb_surrogate* s, float* w, float* r)
{
    return guard([&] {
        if (w) CK(cudaMemcpy(w, s->w.p, sizeof(float) * s->nw, cudaMemcpyDeviceToHost));
        if (r) CK(cudaMemcpy(r, s->r.p, sizeof(float) * s->nr, cudaMemcpyDeviceToHost));
    });
}

int mlb_surrogate_set_params(mlb_surrogate* s, const float* w, const float* r)
{
    return guard([&] {
        g_version++;
        if (w) sur_upload_w(s, std::vector<float>(w, w + s->nw));
        if (r) CK(cudaMemcpy(s->r.p, r, sizeof(float) * s->nr, cudaMemcpyHostToDevice));
        if (s->g_train == 0.0) s->g_train = s->op->g * s->op->gs;
        CK(cudaDeviceSynchronize());
    });
}

int mlb_surrogate_set_schedule(mlb_surrogate* s, int k, double tol, double eps)
{
    return guard([&] {
        g_version++;
        if (k < 1) fail(MLB_EINVAL, "k must be at least 1");
        s->kint = k;
        s->tol = tol;
        if (eps > 0) s->eps = eps;
    });
}

int mlb_surrogate_forward(mlb_surrogate* s, const float* const x[3], float* const dh[3])
{
    return guard([&] {
        const size_t bytes = sizeof(float) * s->n;
        for (int c = 0; c < 3; c++) CK(cudaMemcpy(s->m0[c].p, x[c], bytes, cudaMemcpyHostToDevice));
        const float* a[3] = {s->m0[0].p, s->m0[1].p, s->m0[2].p};
        float* P[3] = {s->P[0].p, s->P[1].p, s->P[2].p};
        sur_forward(s, a, nullptr, 1, nullptr, P, nullptr, nullptr, 1.f, 0);
        CK(cudaDeviceSynchronize());
        sur_check_err(s);
        for (int c = 0; c < 3; c++) CK(cudaMemcpy(dh[c], P[c], bytes, cudaMemcpyDeviceToHost));
    });
}

int mlb_surrogate_gradients(mlb_surrogate* s, const float* const x[3], const float* const t[3], float* dw, float* dr,
                            float* const p[3], double* loss)
{
    return guard([&] {
        const size_t bytes = sizeof(float) * s->n;
        for (int c = 0; c < 3; c++) {
            CK(cudaMemcpy(s->m0[c].p, x[c], bytes, cudaMemcpyHostToDevice));
            CK(cudaMemcpy(s->h0[c].p, t[c], bytes, cudaMemcpyHostToDevice));
        }
        const float* a[3] = {s->m0[0].p, s->m0[1].p, s->m0[2].p};
        const float* hx[3] = {s->h0[0].p, s->h0[1].p, s->h0[2].p};
        sur_train_iter(s, a, nullptr, hx, nullptr, 0.0, false, 0);
        CK(cudaDeviceSynchronize());
        sur_check_err(s);
        double sums[3];
        CK(cudaMemcpy(sums, s->lsum.p, sizeof(sums), cudaMemcpyDeviceToHost));
        const double sc = sums[0] > 0 ? 1.0 / sums[0] : 0.0;
        if (dw) {
            CK(cudaMemcpy(dw, s->gw.p, sizeof(float) * s->nw, cudaMemcpyDeviceToHost));
            for (int i = 0; i < s->nw; i++) dw[i] = (float)(dw[i] * sc);
        }
        if (dr) {
            CK(cudaMemcpy(dr, s->gr.p, sizeof(float) * s->nr, cudaMemcpyDeviceToHost));
            for (int i = 0; i < s->nr; i++) dr[i] = (float)(dr[i] * sc);
        }
        if (p)
            for (int c = 0; c < 3; c++)
                if (p[c]) CK(cudaMemcpy(p[c], s->P[c].p, bytes, cudaMemcpyDeviceToHost));
        if (loss) *loss = sums[1] * sc;
    });
}

int mlb_surrogate_train(mlb_surrogate* S, mlb_system* ss, mlb_op* const* ops, int nops, mlb_llg* l, int nsteps,
                        int window, double lr, double* loss_out)
{
    return guard([&] {
        sur_check_use(S, ss, ops, nops);
        if (window < 2) fail(MLB_EINVAL, "window must be at least 2");
        g_version++;
        S->g_train = S->op->g * S->op->gs;
        std::vector<double> hist;
        DBuf<double> dh;
        dh.alloc((size_t)3 * std::max(1, nsteps));
        int it = 0;
        for (int step = 0; step < nsteps; step++) {
            plain_step_with(ss, ops, nops, l, S, [&](Slot& sl) {
                if (step % window == 0) {
                    sur_snapshot_now(S, ss, sl);
                    return;
                }
                const float* a[3];
                const float* b[3] = {S->m0[0].p, S->m0[1].p, S->m0[2].p};
                const float* hx[3];
                const float* h0[3] = {S->h0[0].p, S->h0[1].p, S->h0[2].p};
                for (int c = 0; c < 3; c++) {
                    a[c] = static_cast<const float*>(ss->sp[ss->cur][c]);
                    hx[c] = static_cast<const float*>(sl.h[c]);
                }
                sur_train_iter(S, a, b, hx, h0, lr, true, ss->st);
                CK(cudaMemcpyAsync(dh.p + 3 * (size_t)it, S->lsum.p, sizeof(double) * 3, cudaMemcpyDeviceToDevice,
                                   ss->st));
                it++;
            });
        }
        CK(cudaStreamSynchronize(ss->st));
        sur_check_err(S);
        hist.resize((size_t)3 * it);
        if (it) CK(cudaMemcpy(hist.data(), dh.p, sizeof(double) * hist.size(), cudaMemcpyDeviceToHost));
        double acc = 0;
        int cnt = 0;
        for (int i = it - std::max(1, it / 4); i < it; i++) {
            if (i < 0 || hist[3 * i] <= 0) continue;
            acc += hist[3 * i + 1] / hist[3 * i];
            cnt++;
        }
        if (loss_out) *loss_out = cnt ? acc / cnt : 0.0;
    });
}

int mlb_surrogate_validate(mlb_surrogate* S, mlb_system* ss, mlb_op* const* ops, int nops, mlb_llg* l, int nsteps,
                           int window, double out[6])
{
    return guard([&] {
        sur_check_use(S, ss, ops, nops);
        if (window < 2) fail(MLB_EINVAL, "window must be at least 2");
        double sum[3] = {0, 0, 0}, mx[3] = {0, 0, 0};
        int cnt = 0;
        const float ratio = S->g_train > 0 ? (float)(S->op->g * S->op->gs / S->g_train) : 1.f;
        for (int step = 0; step < nsteps; step++) {
            plain_step_with(ss, ops, nops, l, S, [&](Slot& sl) {
                if (step % window == 0) {
                    sur_snapshot_now(S, ss, sl);
                    return;
                }
                const float* a[3];
                const float* b[3] = {S->m0[0].p, S->m0[1].p, S->m0[2].p};
                const float* hx[3];
                const float* h0[3] = {S->h0[0].p, S->h0[1].p, S->h0[2].p};
                float* P[3] = {S->P[0].p, S->P[1].p, S->P[2].p};
                float* G[3] = {S->G[0].p, S->G[1].p, S->G[2].p};
                for (int c = 0; c < 3; c++) {
                    a[c] = static_cast<const float*>(ss->sp[ss->cur][c]);
                    hx[c] = static_cast<const float*>(sl.h[c]);
                }
                sur_forward(S, a, b, 1, nullptr, P, nullptr, nullptr, ratio, ss->st);
                const float* Pc[3] = {P[0], P[1], P[2]};
                CK(mlb::launch_sur_loss(S->n, Pc, hx, h0, G, S->lpart.p, S->lnb, S->lsum.p, ss->st));
                double s3[3];
                CK(cudaMemcpyAsync(s3, S->lsum.p, sizeof(s3), cudaMemcpyDeviceToHost, ss->st));
                CK(cudaStreamSynchronize(ss->st));
                if (s3[0] <= 0 || s3[2] <= 0) return;
                const double e[3] = {std::sqrt(s3[1] / s3[0]), std::sqrt(s3[1] / s3[2]), std::sqrt(s3[0] / s3[2])};
                for (int q = 0; q < 3; q++) { sum[q] += e[q]; mx[q] = std::max(mx[q], e[q]); }
                cnt++;
            });
        }
        sur_check_err(S);
        for (int q = 0; q < 3; q++) {
            out[2 * q] = cnt ? sum[q] / cnt : 0.0;
            out[2 * q + 1] = mx[q];
        }
        if (cnt) S->eps = mx[0];
    });
}

int mlb_surrogate_attach(mlb_surrogate* S, mlb_system* ss)
{
    return guard([&] {
        if (ss->rb != 4) fail(MLB_EUNSUP, "the surrogate runs on FP32 systems");
        if (ss->nx != S->nx || ss->ny != S->ny || ss->nz != S->nz)
            fail(MLB_EINVAL, "surrogate and SpinSystem sizes differ");
        if (ss->sur && ss->sur != S) fail(MLB_ESTATE, "another surrogate is attached to this system");
        // the tensor spectrum is built outside any capture
        if (!S->op->plan || S->op->plan_dirty || S->op->plan->rb != 4) build_plan(S->op, ss->st, 4);
        SurDev h{};
        h.exact = 1;
        h.k = S->kint;
        h.eps = (float)S->eps;
        h.tol = (float)S->tol;
        CK(cudaMemcpyAsync(S->dev.p, &h, sizeof(h), cudaMemcpyHostToDevice, ss->st));
        CK(cudaStreamSynchronize(ss->st));
        ss->sur = S;
        g_version++;
    });
}

int mlb_surrogate_detach(mlb_system* ss)
{
    return guard([&] {
        mlb_surrogate* S = ss->sur;
        if (!S) return;
        ss->sur = nullptr;
        g_version++;
        CK(cudaStreamSynchronize(ss->st));
        SurDev h;
        CK(cudaMemcpy(&h, S->dev.p, sizeof(h), cudaMemcpyDeviceToHost));
        S->stats[0] = h.nexact;
        S->stats[1] = h.nsur;      // steps that used the network's field
        S->stats[2] = h.nfail;     // of those, checks that sent the next step to the exact field
        S->last_bound = h.last_bound;
        sur_check_err(S);
    });
}

int mlb_surrogate_run(mlb_surrogate* S, mlb_system* ss, mlb_op* const* ops, int nops, mlb_llg* l, int nsteps)
{
    return guard([&] {
        sur_check_use(S, ss, ops, nops);
        if (nsteps <= 0) return;
        int rc = mlb_surrogate_attach(S, ss);
        if (rc) fail(rc, g_err);
        try {
            bool done = false;
            if (nsteps >= 3) {
                mlb_plan p;
                p.s = ss;
                p.ops.assign(ops, ops + nops);
                p.l = l;
                bool ok = true;
                try {
                    plan_capture(&p);
                } catch (Err&) {
                    ok = false;
                }
                if (ok) {
                    plan_launch(&p, nsteps);
                    done = true;
                }
                plan_release(&p);
            }
            if (!done)
                for (int k = 0; k < nsteps; k++) {
                    do_step(ss, ops, nops, l);
                    advance_sweep(ops, nops);
                }
        } catch (...) {
            ss->sur = nullptr;
            g_version++;
            throw;
        }
        rc = mlb_surrogate_detach(ss);
        if (rc) fail(rc, g_err);
    });
}

int mlb_surrogate_stats(mlb_surrogate* s, long long out[3], double* last_bound)
{
    return guard([&] {
        for (int q = 0; q < 3; q++) out[q] = s->stats[q];
        if (last_bound) *last_bound = s->last_bound;
    });
}

} // extern "C"

// ---------------------------------------------------------------- no-allocation dipole field
// Spectrum scratch of mlb_dipole_field_noalloc: a file-scope device array,
// so the call allocates nothing.  Nothing in it needs to start at zero: the
// forward x pass writes every spectrum element (kx < Px/2+1, all three
// components, every data row) before the (y,z) pass and the inverse x pass
// read it.
static __device__ __align__(256) unsigned char g_noalloc_spec[MLB_NOALLOC_SCRATCH_BYTES];

namespace {
constexpr int kNoallocMaxDevices = 64;
void* g_noalloc_addr[kNoallocMaxDevices] = {};   // device address of g_noalloc_spec per device
std::mutex g_noalloc_mu;

// Address of the scratch on device dev (the current device), looked up on
// the first call made with that device current (the lookup may load this
// library's device code, so that first call belongs before any stream
// capture).  The address is kept for the life of the process: it does not
// survive a cudaDeviceReset.
void* noalloc_scratch(int dev)
{
    if (dev < 0 || dev >= kNoallocMaxDevices) fail(MLB_EUNSUP, "device ordinal beyond the scratch table");
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_spec);
        if (e != cudaSuccess || !p)
            fail(MLB_ECUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
        g_noalloc_addr[dev] = p;
    }
    return g_noalloc_addr[dev];
}
} // namespace

extern "C" int mlb_dipole_field_noalloc(mlb_op* op, const float* sx, const float* sy, const float* sz, float* hx,
                                        float* hy, float* hz, void* stream)
{
    return guard([&] {
        if (!op) fail(MLB_EINVAL, "null operator");
        if (op->kind != MLB_OP_DIPOLE && op->kind != MLB_OP_LONGRANGE)
            fail(MLB_EINVAL, "not a Dipole or LongRange operator");
        // size check first, from the plan geometry alone (nothing allocated)
        ConvPlan geo;
        geo.rb = 4;
        plan_sizes(op, geo);
        if (geo.k.split)
            fail(MLB_EUNSUP, "a (y,z) plane larger than shared memory needs the split passes' second spectrum "
                             "buffer, which mlb_dipole_field_noalloc does not provide");
        const size_t need = (size_t)geo.k.Kx * 3 * op->nz * op->ny * sizeof(float2);
        if (need > (size_t)MLB_NOALLOC_SCRATCH_BYTES)
            fail(MLB_ERANGE, "spectrum of " + std::to_string(need) + " bytes for " + std::to_string(op->nx) + "x" +
                                 std::to_string(op->ny) + "x" + std::to_string(op->nz) + " exceeds the " +
                                 std::to_string((unsigned long long)MLB_NOALLOC_SCRATCH_BYTES) +
                                 "-byte static scratch of mlb_dipole_field_noalloc");
        if (!op->plan || op->plan_dirty || op->plan->rb != 4)
            fail(MLB_ESTATE, "tensor spectrum not built for FP32: apply the operator to an FP32 SpinSystem once "
                             "(that call allocates) before calling mlb_dipole_field_noalloc");
        if (!sx || !sy || !sz || !hx || !hy || !hz) fail(MLB_EINVAL, "null spin or field array");
        int dev = -1;
        CK(cudaGetDevice(&dev));
        if (dev != op->plan->device)
            fail(MLB_EINVAL, "current device " + std::to_string(dev) + " is not the device " +
                                 std::to_string(op->plan->device) + " that holds the operator's tensor spectrum");
        void* scratch = noalloc_scratch(dev);
        const ConvPlan& P = *op->plan;
        ConvK k = P.k;
        k.nrep = 1;
        k.g = op->g * op->gs / ((double)k.Px * k.Py * k.Pz);
        cudaStream_t st = (cudaStream_t)stream;
        const float* sp[3] = {sx, sy, sz};
        float* h[3] = {hx, hy, hz};
        if (mlb::conv_fast_ok(k)) {
            CK(mlb::launch_conv_fast(k, P.L, reinterpret_cast<const float2*>(P.tw.p), sp,
                                     static_cast<float2*>(scratch), reinterpret_cast<const float*>(P.ten6.p), h, st));
        } else {
            const void* spv[3] = {sx, sy, sz};
            void* hv[3] = {hx, hy, hz};
            CK(mlb::launch_conv(k, P.L[0], P.L[1], P.L[2], P.tw.p, spv, scratch, P.ten6.p, P.ten9.p, hv, 4, st));
        }
    });
}

// ====================================================================== GAB / MAB tensor files
// Dipole2D and Magnetostatics2D data files (dip2d_luafuncs.lua:278-500,
// mag2d_luafuncs.lua:278-480): a Lua file holding the system size, the
// builder state and the nine arrays of every (destination, source) layer
// pair, `% 16.15E` numbers with `0` for exact zeros, ending in a loader that
// the reference's makeData runs (`return sameInternals, load`).  The layout
// is the reference's so that either side can read the other's files; the
// loader text below is this library's own.
namespace {

const char* const kLr2dLoader = R"LUA(
-- loader: rows of comma-separated numbers -> tables indexed [y][x]
local function rows_of(block)
    if block == 0 then
        local zero_row = setmetatable({}, {__index = function() return 0 end})
        return setmetatable({}, {__index = function() return zero_row end})
    end
    local out = {}
    for line in string.gmatch(block, "[^\n]+") do
        local row = {}
        for w in string.gmatch(line, "[^,]+") do
            local v = tonumber(w)
            if v then row[#row + 1] = v end
        end
        if #row > 0 then out[#out + 1] = row end
    end
    return out
end

local names = {"XX", "XY", "XZ", "YX", "YY", "YZ", "ZX", "ZY", "ZZ"}
local blocks = {XX = XX, XY = XY, XZ = XZ, YX = YX, YY = YY, YZ = YZ, ZX = ZX, ZY = ZY, ZZ = ZZ}

local function close(a, b)
    if a == b then return true end
    if a == nil or b == nil or a == 0 or b == 0 then return false end
    return math.abs(a - b) / math.abs(a + b) < 1e-8
end

local function matches(op)
    local id = op:internalData()
    if id == nil then return false end
    if op:nx() ~= nx or op:ny() ~= ny or op:nz() ~= nz then return false end
    for k = 1, nz do
        for i = 1, 3 do
            for j = 1, 3 do
                if not close(id.ABC[k][i][j], internal.ABC[k][i][j]) then return false end
            end
            local mine = (internal.offset or internal.grainSize)[k][i]
            local theirs = ((internal.offset and id.offset) or id.grainSize)[k][i]
            if not close(theirs, mine) then return false end
        end
    end
    for _, key in ipairs({"truncation", "truncationX", "truncationY", "truncationZ"}) do
        if not close(id[key], internal[key]) then return false end
    end
    return true
end

local function load(op)
    if op:nx() ~= nx or op:ny() ~= ny or op:nz() ~= nz then
        error("Size Mismatch", 2)
    end
    op:setInternalData(internal)
    op:setNewDataRequired(false)
    for d = 1, nz do
        for s = 1, nz do
            for _, ab in ipairs(names) do
                local r = rows_of(blocks[ab][d][s])
                local t = op:tensorArray(d, s, ab)
                for x = 1, nx do
                    for y = 1, ny do
                        t:set(x, y, r[y][x])
                    end
                end
            end
        end
    end
    op:setCompileRequired(true)
end

return matches, load
)LUA";

const char* const kNames9[9] = {"XX", "XY", "XZ", "YX", "YY", "YZ", "ZX", "ZY", "ZZ"};

std::string num14(double v)
{
    char b[64];
    snprintf(b, sizeof(b), "%.14g", v);
    return b;
}

bool same_number(double a, double b)
{
    if (a == b) return true;
    if (a == 0 || b == 0) return false;
    return std::fabs(a - b) / std::fabs(a + b) < 1e-8;
}

// numbers following `key` up to the end of its line (or of a {...} group)
std::vector<double> numbers_on_line(const std::string& t, size_t at)
{
    std::vector<double> v;
    const size_t end = t.find('\n', at);
    const std::string line = t.substr(at, end == std::string::npos ? std::string::npos : end - at);
    const char* p = line.c_str();
    while (*p) {
        if ((*p >= '0' && *p <= '9') || *p == '-' || *p == '+' || *p == '.') {
            char* e;
            const double x = strtod(p, &e);
            if (e == p) { p++; continue; }
            v.push_back(x);
            p = e;
        } else {
            p++;
        }
    }
    return v;
}

} // namespace

extern "C" {

int mlb_lr2d_write_data_file(mlb_op* op, const char* filename)
{
    return guard([&] {
        if (!op || !filename) fail(MLB_EINVAL, "null argument");
        if (op->kind != MLB_OP_DIPOLE2D && op->kind != MLB_OP_MAGNETOSTATICS2D)
            fail(MLB_EINVAL, "not a Dipole2D or Magnetostatics2D operator");
        const bool mag = op->kind == MLB_OP_MAGNETOSTATICS2D;
        if (op->lr2_newdata) {
            if (mag) magnetostatics2d_make(op);
            else dipole2d_make(op);
        }
        ensure_t2(op);
        const int nx = op->nx, ny = op->ny, nz = op->nz;
        FILE* f = fopen(filename, "w");
        if (!f) fail(MLB_EINVAL, std::string("cannot write ") + filename);
        fprintf(f, "-- %s Data File\n--\nMagLua_Version = %d\n\n", mag ? "Magnetostatics2D" : "Dipole2D", mlb_version());
        fprintf(f, "-- system size\nlocal nx, ny, nz = %d, %d, %d\n\t\n-- internal state\nlocal internal = {}\n", nx, ny,
                nz);
        fprintf(f, "internal.ABC = {}\ninternal.%s = {}\n", mag ? "grainSize" : "offset");
        for (int z = 0; z < nz; z++) {
            const double* a = &op->d2_abc[z * 9];
            fprintf(f, "internal.ABC[%d] = {{%s, %s, %s}, {%s, %s, %s}, {%s, %s, %s}}\n", z + 1, num14(a[0]).c_str(),
                    num14(a[1]).c_str(), num14(a[2]).c_str(), num14(a[3]).c_str(), num14(a[4]).c_str(),
                    num14(a[5]).c_str(), num14(a[6]).c_str(), num14(a[7]).c_str(), num14(a[8]).c_str());
        }
        fprintf(f, "\n");
        for (int z = 0; z < nz; z++) {
            const double* v = mag ? &op->d2_grain[z * 3] : &op->d2_off[z * 3];
            fprintf(f, "internal.%s[%d] = {%s, %s, %s}\n", mag ? "grainSize" : "offset", z + 1, num14(v[0]).c_str(),
                    num14(v[1]).c_str(), num14(v[2]).c_str());
        }
        fprintf(f, "internal.truncation  = %d\ninternal.truncationX = %d\ninternal.truncationY = %d\n"
                   "internal.truncationZ = %d\n\n",
                op->d2_trunc[0], op->d2_trunc[1], op->d2_trunc[2], op->d2_trunc[3]);
        fprintf(f, "-- interaction tensors. Format is AB[destination_layer][source_layer]\n");
        std::string tt = "{";
        for (int d = 0; d < nz; d++) tt += d ? ", {}" : "{}";
        tt += "}";
        for (int ab = 0; ab < 9; ab++) fprintf(f, "local %s = %s\n", kNames9[ab], tt.c_str());
        fprintf(f, "\n");
        const size_t plane = (size_t)nx * ny;
        for (int ab = 0; ab < 9; ab++)
            for (int d = 0; d < nz; d++)
                for (int s = 0; s < nz; s++) {
                    fprintf(f, "%s[%d][%d] = [[\n", kNames9[ab], d + 1, s + 1);
                    const double* a = op->t2.data() + (((size_t)d * nz + s) * 9 + ab) * plane;
                    for (int y = 0; y < ny; y++) {
                        for (int x = 0; x < nx; x++) {
                            const double v = a[(size_t)y * nx + x];
                            if (x) fputs(", ", f);
                            if (v == 0) fputs("0", f);
                            else fprintf(f, "% 16.15E", v);
                        }
                        fputc('\n', f);
                    }
                    fprintf(f, "]]\n");
                }
        fputs(kLr2dLoader, f);
        const bool ok = ferror(f) == 0;
        fclose(f);
        if (!ok) fail(MLB_EINVAL, std::string("error writing ") + filename);
    });
}

int mlb_lr2d_read_data_file(mlb_op* op, const char* filename, int* loaded)
{
    return guard([&] {
        if (!op || !filename || !loaded) fail(MLB_EINVAL, "null argument");
        if (op->kind != MLB_OP_DIPOLE2D && op->kind != MLB_OP_MAGNETOSTATICS2D)
            fail(MLB_EINVAL, "not a Dipole2D or Magnetostatics2D operator");
        *loaded = 0;
        const bool mag = op->kind == MLB_OP_MAGNETOSTATICS2D;
        FILE* f = fopen(filename, "rb");
        if (!f) fail(MLB_ENOTFOUND, std::string("cannot read ") + filename);
        std::string t;
        char buf[65536];
        size_t got;
        while ((got = fread(buf, 1, sizeof(buf), f)) > 0) t.append(buf, got);
        fclose(f);
        const int nx = op->nx, ny = op->ny, nz = op->nz;
        // kind and size
        if (t.find(mag ? "-- Magnetostatics2D Data File" : "-- Dipole2D Data File") == std::string::npos) return;
        size_t at = t.find("local nx, ny, nz =");
        if (at == std::string::npos) fail(MLB_EINVAL, "no system size in " + std::string(filename));
        std::vector<double> dims = numbers_on_line(t, at + 18);
        if (dims.size() < 3 || dims[0] != nx || dims[1] != ny || dims[2] != nz) return;
        // builder state (sameInternals)
        for (int z = 0; z < nz; z++) {
            at = t.find("internal.ABC[" + std::to_string(z + 1) + "] =");
            if (at == std::string::npos) return;
            std::vector<double> a = numbers_on_line(t, t.find('=', at) + 1);
            if (a.size() < 9) return;
            for (int q = 0; q < 9; q++)
                if (!same_number(a[q], op->d2_abc[z * 9 + q])) return;
            const std::string key = mag ? "internal.grainSize[" : "internal.offset[";
            at = t.find(key + std::to_string(z + 1) + "] =");
            if (at == std::string::npos) return;
            std::vector<double> v = numbers_on_line(t, t.find('=', at) + 1);
            if (v.size() < 3) return;
            const double* mine = mag ? &op->d2_grain[z * 3] : &op->d2_off[z * 3];
            for (int q = 0; q < 3; q++)
                if (!same_number(v[q], mine[q])) return;
        }
        const char* tkeys[4] = {"internal.truncation ", "internal.truncationX", "internal.truncationY",
                                "internal.truncationZ"};
        for (int q = 0; q < 4; q++) {
            at = t.find(tkeys[q]);
            if (at == std::string::npos) return;
            std::vector<double> v = numbers_on_line(t, t.find('=', at) + 1);
            if (v.empty() || !same_number(v[0], op->d2_trunc[q])) return;
        }
        // the arrays
        const size_t plane = (size_t)nx * ny;
        std::vector<double> all((size_t)nz * nz * 9 * plane, 0.0);
        for (int ab = 0; ab < 9; ab++)
            for (int d = 0; d < nz; d++)
                for (int s = 0; s < nz; s++) {
                    const std::string key =
                        std::string(kNames9[ab]) + "[" + std::to_string(d + 1) + "][" + std::to_string(s + 1) + "] =";
                    at = t.find(key);
                    if (at == std::string::npos) fail(MLB_EINVAL, "no " + key + " block in " + filename);
                    size_t p = at + key.size();
                    while (p < t.size() && (t[p] == ' ' || t[p] == '\t')) p++;
                    double* out = all.data() + (((size_t)d * nz + s) * 9 + ab) * plane;
                    if (t.compare(p, 2, "[[") != 0) continue;   // `= 0`: an all-zero array
                    const size_t e = t.find("]]", p + 2);
                    if (e == std::string::npos) fail(MLB_EINVAL, "unterminated " + key + " block in " + filename);
                    const char* c = t.c_str() + p + 2;
                    const char* stop = t.c_str() + e;
                    size_t n = 0;
                    while (c < stop && n < plane) {
                        char* endp;
                        const double v = strtod(c, &endp);
                        if (endp == c) { c++; continue; }
                        out[n++] = v;   // row y, column x
                        c = endp;
                    }
                    if (n != plane) fail(MLB_EINVAL, key + " block of " + filename + " is not nx*ny numbers");
                }
        g_version++;
        op->t2.swap(all);
        op->lr2_newdata = false;
        op->lr2_compile = true;
        *loaded = 1;
    });
}

} // extern "C"

namespace mlb {
// The message mlb_last_error returns, for entry points defined in other
// translation units (ewald.cu).
void set_last_error(const std::string& msg) { g_err = msg; }
} // namespace mlb
