/*
 * oracle.h -- FP64 CPU restatement of MagLua's spin-dynamics step.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA
 * product path is compared against.  Only tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline leg may load it.  Nothing in maglua_b200/
 * links, loads or calls it.
 *
 * Parity status: the reference CPU modules cannot be compiled in this
 * environment (no Lua 5.1, no FFTW3, no MPI headers), so this is a
 * restatement ("port"), not the reference binary.  It is pinned by:
 *   - the published MT19937 known-answer outputs (mt19937ar.out vectors),
 *   - numpy.fft (pocketfft, float64) for the FFT,
 *   - the closed-form dipole tensor elements,
 *   - a physical O(N^2) direct dipole sum,
 *   - the reference's own LongRange3D-vs-Exchange equivalence script
 *     (src/modules/cpu/longrange3d/test.lua), made quantitative.
 * The rest of the arithmetic follows the cited reference lines
 * statement by statement and is otherwise "parity unpinned".
 *
 * Every function names the reference file:line it restates; paths are
 * relative to the reference project root, with src/modules abbreviated M/.
 */
#ifndef MLB200_ORACLE_H
#define MLB200_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAX_SLOTS 32
#define ORC_SLOT_NAME 32

/* SpinSystem: SoA x,y,z,ms; named field slots, "Total" = slot 0.
 * M/cpu/core/spinsystem.h:33-140, init spinsystem.cpp:502-566. */
typedef struct orc_ss {
    int nx, ny, nz, n;
    double *x, *y, *z, *ms;
    double alpha, gamma, dt, time;        /* defaults 1,1,1,0 (spinsystem.cpp:29-34) */
    double *site_alpha, *site_gamma;      /* NULL when uniform */
    int nslots;
    char names[ORC_MAX_SLOTS][ORC_SLOT_NAME];
    double *hx[ORC_MAX_SLOTS], *hy[ORC_MAX_SLOTS], *hz[ORC_MAX_SLOTS];
    int used[ORC_MAX_SLOTS];
} orc_ss;

orc_ss* orc_ss_new(int nx, int ny, int nz);
void    orc_ss_free(orc_ss* ss);
void    orc_ss_copy(orc_ss* dst, const orc_ss* src);          /* spins + scalars */
int     orc_ss_slot(orc_ss* ss, const char* name);            /* register (spinsystem.cpp:603-625) */
int     orc_ss_find_slot(const orc_ss* ss, const char* name); /* getSlot (:889-905), -1 if absent */
double* orc_ss_field(orc_ss* ss, const char* name, int comp); /* registers when absent */
void    orc_ss_set_spin(orc_ss* ss, int i, double sx, double sy, double sz);  /* set(i,..) :1090 */
void    orc_ss_set_site_alpha(orc_ss* ss, const double* a);   /* NULL clears */
void    orc_ss_set_site_gamma(orc_ss* ss, const double* g);
void    orc_ss_reset_fields(orc_ss* ss);                      /* zeroFields :968-980 */
void    orc_ss_sum_fields(orc_ss* ss);                        /* sumFields :853-871 */
void    orc_ss_sum_fields_weighted(orc_ss* ss, const char* dest, int nsrc,
                                   const char* const* src, const double* w);
void    orc_ss_netmoment(const orc_ss* ss, double m, double out[8]);

/* Mersenne Twister, M/common/random/mersennetwister.h:82-360. */
typedef struct orc_mt { unsigned long long state[624]; int pnext; int left; } orc_mt;
void     orc_mt_seed(orc_mt* mt, unsigned long long seed);
unsigned long long orc_mt_randint(orc_mt* mt);
double   orc_mt_rand(orc_mt* mt);
double   orc_mt_randnorm(orc_mt* mt, double mean, double stddev);
void     orc_mt_seed_array(orc_mt* mt, const unsigned long long* key, int len);

/* Field operators (each writes its slot; names as in the reference). */
void orc_exchange_apply(orc_ss* ss, const int* from, const int* to, const double* J,
                        int npath, int normalize, double gscale);
void orc_anisotropy_apply(orc_ss* ss, const int* site, const double* axis, const double* K,
                          int nops, double gscale);
void orc_anisotropy_uniaxial_apply(orc_ss* ss, const int* site, const double* axis,
                                   const double* K1, const double* K2, int nops,
                                   double gscale, int quirk);
void orc_anisotropy_cubic_apply(orc_ss* ss, const int* site, const double* axes,
                                const double* K, int nops, double gscale, int quirk);
int  orc_cubic_axes(const double* a1_in, const double* a2_in, double out9[9]);
void orc_uniaxial_axis(const double* a_in, double out3[3]);
int  orc_thermal_apply(orc_ss* ss, double T, const double* scale, double gscale, orc_mt* rng);
void orc_thermal_apply_noise(orc_ss* ss, double T, const double* scale, double gscale,
                             const double* nx, const double* ny, const double* nz);
void orc_thermal_draw(const orc_ss* ss, double T, orc_mt* rng, double* nx, double* ny, double* nz);
void orc_zeeman_apply(orc_ss* ss, const double B[3], double gscale);

/* Dipole tensor: periodic-in-plane lattice sum, dipolesupport.cpp:34-240,717-851.
 * Output arrays have nx*ny*(2nz-1) entries, index i + nx*(j + ny*(k+nz-1)). */
/* The math.huge Dipole tensor: images summed in rings of lstep lattices,
 * nrings rings (the reference: 1000 rings of 5). */
void orc_dipole_tensor_rings(int nx, int ny, int nz, const double ABC[9], int nrings, int lstep,
                             double* XX, double* XY, double* XZ, double* YY, double* YZ, double* ZZ);
/* The Magnetostatic tensor of a finite truncation: prism-prism
 * demagnetising elements (gamma_ab_v.cpp) with the crossover to the point
 * dipole of getGAB_range. */
void orc_magnetostatic_tensor(int nx, int ny, int nz, const int gmax[4], const double ABC[9], const double prism[3],
                              double tol, double* XX, double* XY, double* XZ, double* YY, double* YZ, double* ZZ);
void orc_dipole_tensor(int nx, int ny, int nz, const int gmax[4], const double ABC[9],
                       double* XX, double* XY, double* XZ, double* YY, double* YZ, double* ZZ);
/* LongRange::apply, spinoperationlongrange.cpp:275-312,354-440.
 * T6 = {XX,XY,XZ,YY,YZ,ZZ} in the layout above. */
void orc_longrange_apply(orc_ss* ss, const char* slot, double* const T6[6], double g, double gscale);
typedef struct orc_lr orc_lr;   /* cached tensor transforms (updateData) */
orc_lr* orc_lr_new(int nx, int ny, int nz, double* const T6[6]);
void    orc_lr_apply(orc_lr* c, orc_ss* ss, const char* slot, double g, double gscale);
void    orc_lr_free(orc_lr* c);
/* LongRange3D::apply/compile, spinoperationlongrange3d.cpp:331-424.
 * T9 = {XX,XY,XZ,YX,YY,YZ,ZX,ZY,ZZ}, each nx*ny*nz, cyclic. */
void orc_longrange3d_apply(orc_ss* ss, double* const T9[9], double g, double gscale);
/* Physical open-boundary direct sum h_t = g * sum_s Gamma(r_t - r_s) s_s (no images). */
void orc_dipole_direct_sites(int nx, int ny, int nz, const double* x, const double* y, const double* z,
                             const double ABC[9], double g, const long long* sites, int nsites, double* out);
/* Gamma(r) of every offset of an open lattice (six arrays, XX..ZZ, of
 * (2nx-1)(2ny-1)(2nz-1) values, offset (dx+nx-1) + (2nx-1)((dy+ny-1) +
 * (2ny-1)(dz+nz-1))), the kernel of orc_dipole_direct_sites. */
void orc_dipole_open_tensor(int nx, int ny, int nz, const double ABC[9], double* out6);
void orc_dipole_direct(const orc_ss* ss, const double ABC[9], double g,
                       int px, int py, int pz, double* hx, double* hy, double* hz);

/* LLG, llgcartesian.cpp:90-278, llgquat.cpp:126-378. */
typedef struct orc_llg {
    int thermal_only_first_term;   /* default 1, llg.cpp:25 */
    int disable_renormalization;   /* default 0 */
    double precess_scale, damp_scale;
} orc_llg;
void orc_llg_default(orc_llg* l);
void orc_llg_cart_apply(const orc_llg* l, orc_ss* from, double scale, orc_ss* dmdt,
                        orc_ss* to, int advance);
void orc_llg_quat_apply(const orc_llg* l, orc_ss* from, double scale, orc_ss* dmdt,
                        orc_ss* to, int advance);

/* FFT: unnormalised, sign -1 forward / +1 inverse (FFTW convention,
 * M/cpu/array/fourier.cpp:40-232).  data is interleaved re,im. */
void orc_fft1d(double* data, int n, int stride, int sign);
void orc_fft2d_layers(double* data, int nx, int ny, int nz, int sign);
void orc_fft3d(double* data, int nx, int ny, int nz, int sign);

/* Canonical step driver used to time the CPU path:
 * resetFields; ops in order; sumFields; llg:apply(ss).  Mirrors
 * doc/manual/BasicMicromagneticSimulation.lua:84-94. */
typedef struct orc_step_cfg {
    /* exchange */
    int npath; const int* from; const int* to; const double* J; int ex_normalize;
    /* anisotropy (generic) */
    int nani; const int* ani_site; const double* ani_axis; const double* ani_K;
    /* cubic anisotropy */
    int ncub; const int* cub_site; const double* cub_axes; const double* cub_K; int cub_quirk;
    /* thermal */
    double T; orc_mt* rng;
    /* zeeman */
    int zeeman; double B[3];
    /* dipole (LongRange with reference tensor) */
    int dipole; orc_lr* lr; double g;
    /* llg */
    int llg_type; /* 0 cartesian, 1 quaternion */
    orc_llg llg;
} orc_step_cfg;
void orc_run_steps(orc_ss* ss, const orc_step_cfg* cfg, int nsteps);

#ifdef __cplusplus
}
#endif
#endif
