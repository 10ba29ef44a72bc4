// kparams.h -- plain-old-data launch parameters shared by the host layer
// (capi.cu) and the kernels (kernels.cu, conv_fast.cu).  Device pointers
// only.
#pragma once
#include <stdint.h>

#define MLB_MAX_ADDENDS 6

// Exchange in one of two forms (see exchange compile in capi.cu):
//   STENCIL: six lattice directions, J per direction, per-axis periodicity;
//   CSR:     pathways grouped by target site (insertion order kept).
enum { EX_NONE = 0, EX_STENCIL = 1, EX_CSR = 2 };
// Anisotropy: uniform (same axis/constants on every site, one op per site)
// or a per-site op list in CSR form.
enum { ANI_NONE = 0, ANI_UNIFORM = 1, ANI_CSR = 2 };
enum { TH_NONE = 0, TH_PHILOX = 1, TH_INJECT = 2 };
enum { LLG_CART = 0, LLG_QUAT = 1 };

// Operator parameters are FP64 (host values); kernels compute in the
// system's precision R (float or double) and convert on use.  State arrays
// (spins, ms, slots, per-site alpha/gamma) are untyped device pointers of R.
struct ExchangeK {
    int mode;
    int normalize;
    double J[6];           // (+x,-x,+y,-y,+z,-z): source offset from target
    int pbc[3];
    const int* ptr;        // CSR (n+1)
    const int* col;        // source sites
    const double* val;     // J per pathway
};

// Generic Anisotropy (H = 2K (s.n)/ms^2 n)
struct AniK {
    int mode;
    double axis[3]; double K;                    // uniform (K times global_scale)
    const int* ptr; const double* axes; const double* Ks;   // CSR: axes 3/op, K 1/op
};
// Uniaxial (H = [2K1 u + 4K2 u^3] n, u from unit spin)
struct UniK {
    int mode; int quirk;
    double axis[3]; double K1, K2;
    const int* ptr; const double* axes; const double* K12;  // axes 3/op, K 2/op
};
// Cubic
struct CubK {
    int mode; int quirk;
    double axes[9]; double K[3];
    const int* ptr; const double* axs; const double* Ks;    // axes 9/op, K 3/op
};
struct ThermalK {
    int mode;
    double T;                 // temperature * global_scale
    const double* scale;      // per-site scale or null
    uint64_t seed;
    uint64_t counter;         // host part of the Philox counter
    const uint64_t* dctr;     // device step counter added to it (null = 0)
    const double* nx; const double* ny; const double* nz;   // injected normals
};
struct ZeemanK {
    int on;
    double B[3];              // times global_scale
    const double* Bdev;       // captured steps: B read from the device step block
};

// Parameters a captured step reads on the device and advances once per step
// (k_advance_step): the Thermal counter and the applied field with its sweep.
struct DevStep {
    uint64_t th_counter;
    double B[3];
    double dB[3];
};

struct SysK {
    int nx, ny, nz, n;
    const void* x; const void* y; const void* z;   // spins read (R)
    const void* ms; double ms_u; int ms_uniform;
    const void* site_alpha; const void* site_gamma;
    double alpha, gamma;
};

// Which terms a kernel evaluates, in slot order for the sum.
struct TermsK {
    ExchangeK ex; double ex_gs;   // exchange scale (global_scale x applies)
    AniK ani;
    UniK uni;
    CubK cub;
    ThermalK th;
    ZeemanK zee;
    int nadd;
    const void* add[MLB_MAX_ADDENDS][3];   // materialised slot arrays added to Total (R)
    double addw[MLB_MAX_ADDENDS];
    int add_is_thermal[MLB_MAX_ADDENDS];   // this addend is the Thermal slot
};

struct LlgK {
    unsigned* status;         // bit 0 set when a new spin is not finite (null: not checked)
    int type;
    int thermal_only_first_term;
    int renorm;
    double precess, damp;
    double dt;                // scale * dmdt->dt
    int dt_zero;
};

// One fused step: read spins (sys), evaluate terms, LLG, write spins (out).
struct FusedK {
    SysK sys;
    TermsK terms;
    LlgK llg;
    void* ox; void* oy; void* oz;
};

// ------------------------------------------------------------- dipole
// Convolution plan: padded grid P, data grid n, R2C along x (Kx = Px/2+1).
// Spectrum layout SPEC[kx][c][z][y] (y fastest, data rows only).
struct ConvK {
    int nx, ny, nz;
    int Px, Py, Pz;
    int Kx;
    int ty;                  // rows per CTA in the x passes
    int general;             // 0: 6 real tensor entries per k, 1: 9 complex
    double g;                // strength * global_scale / (Px*Py*Pz)
    int fx, fy, fz;          // FftLen indices
    int nrep;                // replicas of this size packed back to back (1 for a system)
    const int* run_if;       // when set, the passes run only while *run_if != 0
    int yz_variant = 0;      // (y,z) pass of the fast path: 0 automatic, 1 shared-memory Stockham, 2 register
    // Planes too large for one CTA's shared memory: the (y,z) pass runs as
    // three passes (y, z with the tensor multiply, inverse y) through spec2,
    // S2[kx][ky][comp][z] (data layers only), and the tensor is stored
    // ky-major, TEN[kx][ky][kz][q].
    int split;
    void* spec2;
    // Split FP32 passes of a tensor with the per-axis parities of a
    // point-dipole tensor on an orthogonal lattice (XY and YZ odd in ky, XZ
    // and YZ odd in kz, checked on the FP64 transform): the tensor is stored
    // for ky <= Py/2 and kz <= Pz/2 only, TEN[kx][ky][kz][q], and each z-pass
    // CTA takes mirrored ky columns together.
    int quarter = 0;
    // Device timeline of a timing plan (null otherwise): the single-CTA-plane
    // (y,z) kernels write tl[0] = first CTA released from the dependency
    // wait, tl[1] = last CTA finished; the fused x pass tl[2], tl[3]
    // (%globaltimer, ns)
    unsigned long long* tl = nullptr;
};

// LongRange2D layer scales (spinoperationlongrange2d.cpp:430-530): the
// source-moment scale of each source layer and the destination-field scale
// of each destination layer times the operator's global scale.
#define MLB_LR2D_MAXZ 64
struct LR2DScale {
    double src[MLB_LR2D_MAXZ];
    double dst[MLB_LR2D_MAXZ];
};

// Fused step for uniform-parameter systems (k_fused_fast): every constant
// folded on the host.
template <typename R>
struct FastKT {
    int nx, ny, nz;
    int ex;                   // six-direction stencil present
    R J[6];                   // J * scale / ms^2 (normalised) or / ms
    int pbc[3];
    int ani;                  // 0 none, 1 uniaxial (axis, ani_c), 2 cubic (cub_*)
    R axis[3];
    R ani_c;                  // 2 K scale / ms^2
    R cub_n[9];               // cubic axes n1, n2, n3
    R cub_K[3];               // cubic K1, K2, K3 (times the global scale)
    int cub_quirk;
    R cub_ims;                // 1 / ms (the reduced moment S / ms)
    int th;
    R sigma;                  // sqrt(2 alpha T scale / (ms dt gamma))
    uint64_t seed, counter;
    const uint64_t* dctr;
    R B[3];                   // Zeeman (Bdev when read from the device step block)
    const double* Bdev;
    R addw;
    int llg_type, tof, renorm, dt_zero;
    R dt, precess, c_prec, c_damp, c_rot, ms;
    unsigned* status;         // bit 0 set when a new spin is not finite (null: not checked)
    // captured steps of the fused x pass: the step reads adv_cur (through
    // dctr and Bdev) and the pass writes the next step's block into adv_next
    // (null: the step block is advanced by a kernel of its own)
    DevStep* adv_cur;
    DevStep* adv_next;
};
// FP32 state (every fused kernel); FastKT<double> for FP64 state
typedef FastKT<float> FastK;

// ------------------------------------------------------------- learned surrogate
// Linear spectral-conv network on the in-plane grid (ny x nx) with the
// (component, z) pairs as channels: ch = c * nz + z, C = 3 nz real channels
// padded to CP.  Output channel co at site s:
//   sum_{o, ci} W[o][co][ci] X[ci][s + o]                      (stencil, |o_x|,|o_y| <= rad)
// + sum_{kx < mx, ky} w_kx / (nx ny) Re(e^{i k.s} sum_ci R_k[co][ci] Xhat_k[ci])
// with Xhat the 2D DFT of X restricted to the retained modes.
struct SurK {
    int nx, ny, nz;
    int C, CP;
    int mx, my;               // kx < mx; ky in {0..my/2-1} and {ny-my/2..ny-1}
    int rad;
    int nxc;                  // 128-wide x chunks of the x-DFT (nx / 128)
    const int* skip_if;       // kernels return at once while *skip_if != 0
    float ratio;              // strength now / strength at training
    unsigned wait_polls;      // polls of a tensor-core completion wait before it gives up
};

// Device state of a surrogate-driven run (one block per surrogate).
struct SurDev {
    int exact;                // this step evaluates the exact convolution
    int cycle;                // steps since the last exact evaluation
    int k;                    // exact evaluation every k steps
    int nexact, nfail, nsur;  // counters: exact steps, failed residual checks, surrogate steps
    float eps;                // validation relative error of the predicted update
    float tol;                // bound on the estimated relative field error
    float last_bound;
    int fail;                 // this step's residual check failed: the next step is exact
    unsigned int arrivals;    // CTAs of the output kernel done this step
    double sums[2];           // sum dH^2, sum H^2 of this step
};

// Block table of the packed-ensemble fused kernel.
// Packed ensemble step: the work table (replica, first site) of nblk
// tiles of bs sites walked by `grid` CTAs (grid < nblk: persistent CTAs,
// each taking every grid-th tile); per packed replica r the applied field
// B[3r..3r+2] of this step (rB), its sweep (rdB) and thermal deviation
// (rsig); the CTA holding tile 0 of a replica writes the next step's field
// to rBn.
struct EnsLaunch {
    int nblk, bs;
    const int* brep;
    const int* bstart;
    const int4* rinfo;
    int grid;
    const double* rB;
    double* rBn;
    const double* rdB;
    const float* rsig;
};
