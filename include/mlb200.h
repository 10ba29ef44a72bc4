/*
 * mlb200.h -- C ABI of the B200-native MagLua spin-dynamics step.
 *
 * Plain C types only (ints, doubles, pointers, sizes); every function returns
 * MLB_OK (0) or a negative MLB_E* code and never throws, exits or traps.  The
 * message of the last failure on the calling thread is mlb_last_error().
 *
 * Each entry point names the reference interface it replaces (paths relative
 * to the MagLua project root; M/ = src/modules/).  In MagLua those are Lua
 * methods of C++ classes registered by luaT_register<T>
 * (M/common/luabaseobject/luabaseobject.h:643-700); a Lua 5.1 glue module
 * maps each method onto one call below.
 *
 * State lives on the GPU in FP32, or FP64 per system (SoA x, y, z, ms; one
 * stream per system); host-facing values are FP64 like the reference.
 * Reductions are FP64.
 */
#ifndef MLB200_H
#define MLB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MLB_OK 0
#define MLB_EINVAL -1     /* bad argument (luaL_error "invalid ..." in the reference) */
#define MLB_ENOMEM -2     /* device allocation failed */
#define MLB_ECUDA -3      /* CUDA runtime error */
#define MLB_ESTATE -4     /* operation not possible in this state ("Missing RNG", ...) */
#define MLB_ENOTFOUND -5  /* unknown slot name ("Unknown field type") */
#define MLB_ERANGE -6     /* site or size outside the system */
#define MLB_EUNSUP -7     /* size/configuration this build does not support */

typedef struct mlb_system mlb_system;
typedef struct mlb_op mlb_op;
typedef struct mlb_llg mlb_llg;

/* ---------------------------------------------------------------- library */
const char* mlb_last_error(void);
int mlb_version(void);
/* Select the CUDA device (the cuda core's lib_main / "-gpu N" option,
 * M/cuda/core_cuda/maglua.cpp:50-93). */
int mlb_init(int device);
/* Per-kernel timing (no reference counterpart; the reference has only the
 * wall-clock Timer, M/common/timer/mtimer.cpp:219-350).  Between begin and
 * end every kernel launched outside a graph capture is bracketed by CUDA
 * events on its stream; end synchronises and returns per kernel name
 * (48-byte slots in names) the summed milliseconds and launch counts. */
int mlb_profile_begin(void);
int mlb_profile_end(int cap, char* names, double* ms, int* launches, int* count);
/* The counter-based generator behind Thermal (no reference counterpart: the
 * reference uses Mersenne Twister on the host, Random.HybridTaus on the GPU,
 * M/cuda/random_cuda/hybridtaus.cu:32-88).  Host-callable; for checks. */
int mlb_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* ---------------------------------------------------------------- SpinSystem
 * M/cpu/core/spinsystem.h:33-140; methods spinsystem.cpp:3233-3318 and
 * spinsystem_luafuncs.lua. */
int mlb_system_create(int nx, int ny, int nz, mlb_system** out);      /* SpinSystem.new(nx,ny,nz) */
/* The same with the state precision chosen: real_bytes 4 (FP32, the
 * default and the only width the specialised step kernels take) or 8 (FP64
 * state, fields and LLG, as the reference's CPU build computes them; the
 * general kernels only).  No counterpart in the reference, whose CPU build
 * is FP64 and whose cuda32 build is FP32 by compile-time choice
 * (M/cuda32 versus M/cpu). */
int mlb_system_create_ex(int nx, int ny, int nz, int real_bytes, mlb_system** out);
int mlb_system_real_bytes(const mlb_system* s, int* real_bytes);
int mlb_system_destroy(mlb_system* s);                                 /* __gc */
int mlb_system_dims(const mlb_system* s, int out[3]);                  /* nx(), ny(), nz() */
/* Launch on this stream from now on (NULL = the system's own stream). */
int mlb_system_set_stream(mlb_system* s, void* cuda_stream);
int mlb_system_get_stream(const mlb_system* s, void** cuda_stream);
int mlb_system_synchronize(mlb_system* s);
/* B200 extension (the reference only prints CUDA errors): the system's
 * status word after the work queued so far -- bit 0 (MLB_STATUS_NONFINITE)
 * is set once any LLG step of this system wrote a spin component that is not
 * finite (NaN or infinity).  Synchronises the system's stream; clear != 0
 * resets the word. */
#define MLB_STATUS_NONFINITE 1u
int mlb_system_status(mlb_system* s, int clear, unsigned* flags);
/* setSpin(i,j,k, sx,sy,sz[, m]) for one site (l_setspin :1312-1361); idx is
 * the 0-based x + nx*(y + ny*z). */
int mlb_system_set_spin(mlb_system* s, int idx, double sx, double sy, double sz);
int mlb_system_get_spin(mlb_system* s, int idx, double out4[4]);       /* spin(i,j,k) */
/* Whole arrays (setSpinArrayX/Y/Z/M, spinArrayX/Y/Z/M :2164-2305).  With
 * ms == NULL every ms becomes |s| (SpinSystem::set). */
int mlb_system_set_spins(mlb_system* s, const double* x, const double* y, const double* z,
                         const double* ms);
int mlb_system_get_spins(mlb_system* s, double* x, double* y, double* z, double* ms);
/* FP32 host buffers (pinned memory recommended) for bulk I/O. */
int mlb_system_upload_f32(mlb_system* s, const float* x, const float* y, const float* z,
                          const float* ms);
int mlb_system_download_f32(mlb_system* s, float* x, float* y, float* z);
/* Scalars: setAlpha/alpha, setGamma/gamma, setTimeStep/timeStep, setTime/time. */
#define MLB_ALPHA 0
#define MLB_GAMMA 1
#define MLB_DT 2
#define MLB_TIME 3
int mlb_system_set_param(mlb_system* s, int which, double v);
int mlb_system_get_param(const mlb_system* s, int which, double* v);
/* setSiteAlphaArray / setSiteGammaArray (NULL clears: setAlpha resets). */
int mlb_system_set_site_alpha(mlb_system* s, const double* a);
int mlb_system_set_site_gamma(mlb_system* s, const double* g);
/* resetFields (zeroFields :968-980), sumFields (:853-871). */
int mlb_system_reset_fields(mlb_system* s);
int mlb_system_sum_fields(mlb_system* s);
/* sumFields(dest, {{w, name}, ...}) (spinsystem_luafuncs.lua:298-360). */
int mlb_system_sum_fields_custom(mlb_system* s, const char* dest, int n, const char* const* src,
                                 const double* w);
/* fieldArrayX/Y/Z(name) (:1656-1690); any of hx/hy/hz may be NULL. */
int mlb_system_get_field(mlb_system* s, const char* slot, double* hx, double* hy, double* hz);
/* setFieldArrayX/Y/Z (:1692-1728); NULL components are left unchanged. */
int mlb_system_set_field(mlb_system* s, const char* slot, const double* hx, const double* hy,
                         const double* hz);
int mlb_system_slot_used(mlb_system* s, const char* slot, int* used);  /* _slotUsed */
int mlb_system_set_slot_used(mlb_system* s, const char* slot, int used);
int mlb_system_ensure_slot(mlb_system* s, const char* slot);          /* _ensureSlotExists */
/* netMoment(m): 8 numbers as the Lua method (spinsystem_luafuncs.lua:17-54). */
int mlb_system_netmoment(mlb_system* s, double m, double out8[8]);
/* B200 extension (no reference counterpart): netMoment without waiting.
 * _async enqueues the reduction of the current spins and its copy into
 * pinned slot 0..3 and returns: the reduction waits for the work already on
 * the system's stream and runs on a stream of its own, next to the steps
 * enqueued after it (the system's stream waits for it before it next writes
 * the spin buffer it reads); _wait blocks until that slot's copy has landed
 * and fills out8 as mlb_system_netmoment does (the same sums up to the
 * order of the FP64 additions: the side-stream read runs on at most 16
 * blocks, so that most SMs stay free for the following steps).  A caller
 * can launch the next steps before reading this step's result. */
int mlb_system_netmoment_async(mlb_system* s, double m, int slot);
int mlb_system_netmoment_wait(mlb_system* s, int slot, double out8[8]);
/* sum_i s_i . h_slot,i in FP64 (the fieldArray:dot(spinArray) energy pattern). */
int mlb_system_field_dot(mlb_system* s, const char* slot, double* out);
/* copyTo (with_fields: spins, ms, per-site alpha/gamma, alpha, gamma, dt,
 * time and the fields; SpinSystem::copyFrom, spinsystem.cpp:310-391) or
 * copySpinsTo (without: spins and ms only; copySpinsFrom, :393-409). */
int mlb_system_copy(mlb_system* dst, mlb_system* src, int with_fields);
/* diff (spinsystem.cpp:301-307, l_getdiff :2145-2160): sum_i |a_i - b_i| of
 * each component and the length of that vector, FP64. */
int mlb_system_diff(mlb_system* a, mlb_system* b, double out4[4]);
/* encode / decode (SpinSystem::encode / decode, spinsystem.cpp:669-851, as
 * exported as a Lua value, luamigrate.cpp:265-275): the byte stream the
 * reference's CPU build writes for a SpinSystem inside a checkpoint, so that
 * either side reads the other's.  encode writes it into buf when cap holds
 * it (*len = its size; buf == NULL asks for the size alone); first_index is
 * the object index the system takes in the stream (0 for a stream of its
 * own, else the count of objects the enclosing buffer has encoded so far),
 * its arrays take the next ones.  decode makes a new system of that state
 * with real_bytes 4 or 8; with used != NULL the stream may continue after
 * the system and *used = the bytes read, with used == NULL it must end
 * there.  *objects (when not NULL) = the objects the stream holds: the
 * system and its 4 to 6 arrays, each an entry of the enclosing buffer's
 * object list.  Streams whose sites carry extra data (Lua values) give
 * MLB_EUNSUP. */
int mlb_system_encode(mlb_system* s, int first_index, void* buf, size_t cap, size_t* len, int* objects);
int mlb_system_decode(const void* buf, size_t len, int real_bytes, mlb_system** out, size_t* used,
                      int* objects);

/* ---------------------------------------------------------------- operators
 * SpinOperation base, M/cpu/core/spinoperation.h:28-72. */
#define MLB_OP_EXCHANGE 1       /* M/cpu/exchange */
#define MLB_OP_ANISOTROPY 2     /* M/cpu/anisotropy (generic) */
#define MLB_OP_UNIAXIAL 3       /* Anisotropy.Uniaxial */
#define MLB_OP_CUBIC 4          /* Anisotropy.Cubic */
#define MLB_OP_THERMAL 5        /* M/cpu/thermal */
#define MLB_OP_APPLIEDFIELD 6   /* M/cpu/appliedfield */
#define MLB_OP_DIPOLE 7         /* M/cpu/dipole */
#define MLB_OP_LONGRANGE 8      /* M/cpu/longrange (user tensor) */
#define MLB_OP_LONGRANGE3D 9    /* M/cpu/longrange3d */
#define MLB_OP_LONGRANGE2D 10   /* M/cpu/longrange2d (layer-pair tensors) */
#define MLB_OP_DIPOLE2D 11      /* M/cpu/dipole2d (LongRange2D + tensor builder) */
#define MLB_OP_MAGNETOSTATICS2D 12 /* M/cpu/magnetostatics2d (LongRange2D + prism tensors) */
#define MLB_OP_MAGNETOSTATIC 13 /* M/cpu/magnetostatics (LongRange + volume-averaged prism tensors; deprecated there) */
int mlb_op_create(int kind, int nx, int ny, int nz, mlb_op** out);     /* X.new(nx,ny,nz) */
int mlb_op_destroy(mlb_op* op);
int mlb_op_kind(const mlb_op* op, int* kind);
int mlb_op_set_scale(mlb_op* op, double global_scale);                 /* setScale */
int mlb_op_get_scale(const mlb_op* op, double* global_scale);
int mlb_op_set_slot_name(mlb_op* op, const char* name);                /* setSlotName */
int mlb_op_get_slot_name(const mlb_op* op, char* buf, size_t len);     /* slotName */
/* Reproduce the reference's arithmetic quirks (default on): Uniaxial sz*nx
 * (..._uniaxial.cpp:287), Cubic n3s3 (..._cubic.cpp:372-374), LongRange
 * interlayer z-sign (spinoperationlongrange.cpp:377-384). */
int mlb_op_set_quirks(mlb_op* op, int on);
/* op:apply(ss) and op:apply({ss1, ss2, ...}) (spinoperation.cpp:423-446). */
int mlb_op_apply(mlb_op* op, mlb_system* s);
int mlb_op_apply_many(mlb_op* op, mlb_system* const* s, int n);

/* Exchange: ex:add(from, to, J) after pbc wrapping (l_addpath :368-420),
 * normalizeMoments (:283-292, exchange_luafuncs.lua:10-17). */
int mlb_exchange_add_path(mlb_op* op, int from, int to, double J);
int mlb_exchange_add_paths(mlb_op* op, const int* from, const int* to, const double* J, int n);
int mlb_exchange_set_normalize(mlb_op* op, int on);
/* setPeriodicXYZ / periodicXYZ (spinoperationexchange.cpp:560-580): the
 * flags the Lua add() wraps sites by, kept for getPeriodicXYZ and encode. */
int mlb_exchange_set_pbc(mlb_op* op, int px, int py, int pz);
int mlb_exchange_get_pbc(const mlb_op* op, int pbc[3]);
int mlb_exchange_num_paths(const mlb_op* op, int* n);
/* Anisotropy: ani:add(site, axis, K) (axis normalised, spinoperationanisotropy.cpp:367-410). */
int mlb_anisotropy_add(mlb_op* op, int site, const double axis[3], double K);
/* Anisotropy.Uniaxial: add(site, axis, K1, K2) (..._uniaxial.cpp:158-179). */
int mlb_uniaxial_add(mlb_op* op, int site, const double axis[3], double K1, double K2);
/* Anisotropy.Cubic: add(site, a1, a2, K1, K2, K3) (..._cubic.cpp:180-236);
 * MLB_EINVAL for zero-length or colinear axes. */
int mlb_cubic_add(mlb_op* op, int site, const double a1[3], const double a2[3], const double K[3]);
/* Bulk forms of the three add calls (one call per site in the reference's
 * setup loops; n sites, axes 3 per site, K 1 (generic), K1/K2 (uniaxial),
 * a1/a2 3 per site and K 3 per site (cubic)). */
int mlb_anisotropy_add_many(mlb_op* op, int n, const int* sites, const double* axes, const double* K);
int mlb_uniaxial_add_many(mlb_op* op, int n, const int* sites, const double* axes, const double* K1,
                          const double* K2);
int mlb_cubic_add_many(mlb_op* op, int n, const int* sites, const double* a1, const double* a2, const double* K);
/* Thermal (spinoperationthermal.cpp:135-387): temperature, per-site scale,
 * counter-based Philox stream (seed), or injected normals for the next apply
 * (three arrays of nxyz standard normals, as drawn by the reference RNG). */
int mlb_thermal_set_temperature(mlb_op* op, double T);
int mlb_thermal_get_temperature(const mlb_op* op, double* T);
int mlb_thermal_scale_site(mlb_op* op, int idx, double v);
int mlb_thermal_set_seed(mlb_op* op, uint64_t seed);        /* keeps the counter */
int mlb_thermal_set_counter(mlb_op* op, uint64_t counter);
int mlb_thermal_inject(mlb_op* op, const double* nx, const double* ny, const double* nz);
/* AppliedField set/get (appliedfield_luafuncs.lua), plus a per-step linear
 * sweep used by mlb_run (B += dB each step). */
int mlb_appliedfield_set(mlb_op* op, double bx, double by, double bz);
int mlb_appliedfield_get(const mlb_op* op, double out3[3]);
int mlb_appliedfield_set_sweep(mlb_op* op, double dbx, double dby, double dbz);
/* LongRange / Dipole (spinoperationlongrange.cpp:460-875): strength,
 * truncation gmax {r, x, y, z}, unit cell, tensor elements. */
int mlb_longrange_set_strength(mlb_op* op, double g);
int mlb_longrange_get_strength(const mlb_op* op, double* g);
/* setTruncation (spinoperationlongrange.cpp:505-568): gmax[0] < 0 is
 * math.huge (every entry becomes -1).  A Dipole of truncation math.huge takes
 * the reference's extrapolated lattice sum (dipoleLoad,
 * M/cpu/dipole/dipolesupport.cpp:771-835), which in the reference always
 * ends as the image sum over 1000 rings of 5 lattices (|X|, |Y| <= 4999):
 * its C side reads a second return value from the Lua extrapolate() that
 * the function never gives, so convergence is never reported.  FP64 on the
 * GPU, one warp per tensor element. */
int mlb_longrange_set_truncation(mlb_op* op, const int gmax[4]);
int mlb_longrange_get_truncation(const mlb_op* op, int gmax[4]);     /* getTruncation (-1 = math.huge) */
/* B200 extension (no reference counterpart): the number of 5-lattice rings
 * of the math.huge sum (the reference's fixed 1000), for checks on small
 * ring counts. */
int mlb_dipole_set_huge_rings(mlb_op* op, int rings);
int mlb_longrange_set_unit_cell(mlb_op* op, const double ABC[9]);
/* Magnetostatic (M/cpu/magnetostatics/spinoperationmagnetostatics.cpp:
 * 99-160; slot "Magnetostatic"): a LongRange whose tensor is the
 * demagnetising interaction of rectangular prisms of the cell dimensions
 * (gamma_ab_v.cpp), switching per component to the point dipole (times the
 * prism volume / 4 pi) from the first image, nearest first, where the two
 * agree within the crossover tolerance (magnetostaticssupport.cpp:81-187;
 * default 1e-5); built on host threads at first use.  A truncation of
 * math.huge gives MLB_EUNSUP: the reference's ring sum for it keeps only the
 * last of each ring's eight ranges. */
int mlb_magnetostatic_set_cell_dimensions(mlb_op* op, const double d[3]);     /* setCellDimensions */
int mlb_magnetostatic_get_cell_dimensions(const mlb_op* op, double d[3]);     /* cellDimensions */
int mlb_magnetostatic_set_crossover_tolerance(mlb_op* op, double tol);        /* setCrossoverTolerance */
int mlb_magnetostatic_get_crossover_tolerance(const mlb_op* op, double* tol);
/* B200 extension: open (zero-padded) boundaries per axis for Dipole; the
 * reference Dipole is periodic in x and y and open in z. */
int mlb_longrange_set_open(mlb_op* op, int open_x, int open_y, int open_z);
/* setMatrix/getMatrix(AB, {ox,oy,oz}) with AB in XX,XY,XZ,YY,YZ,ZZ = 0..5 */
int mlb_longrange_set_matrix(mlb_op* op, int ab, int ox, int oy, int oz, double v);
int mlb_longrange_get_matrix(mlb_op* op, int ab, int ox, int oy, int oz, double* v);
/* The six tensor arrays, each nx*ny*(2nz-1), layout i + nx*(j + ny*(k+nz-1)). */
int mlb_longrange_get_tensor(mlb_op* op, double* const t6[6]);
/* LongRange3D (spinoperationlongrange3d.cpp:312-424, setMatrix): component
 * ab = 3*a + b in XX..ZZ order, array nx*ny*nz. */
int mlb_longrange3d_set_tensor(mlb_op* op, int ab, const double* t);
/* LongRange2D (spinoperationlongrange2d.cpp:201-230 getLAB/setLAB, :430-530
 * apply, :532-590 layer scales, :605-640 flags).  Layers are 0-based here
 * (1-based in the Lua API); ab = 3*a + b in XX..ZZ order; each array is
 * nx*ny, element (x, y) at x + nx*y.  The arrays are copied in and out.
 * apply reads the arrays set for (dest s, src d) to make the field of layer
 * d from layer s, as the reference's apply does (qAB[s][d]); the field of
 * layer d is scaled by dst_field[d] * global scale and each source layer's
 * moments by src_moment[s].  At apply, new data required fails with
 * MLB_ESTATE ("make data function not set") for LongRange2D and runs the
 * builder for Dipole2D; compile required re-transforms the arrays (setting
 * an array alone does not mark it, as in the reference).  At most 64 layers;
 * 6*nz*ny complex values of the state precision must fit 227 KB. */
int mlb_longrange2d_set_tensor(mlb_op* op, int dest, int src, int ab, const double* t);   /* setTensorArray */
int mlb_longrange2d_get_tensor(mlb_op* op, int dest, int src, int ab, double* t);         /* tensorArray */
int mlb_longrange2d_set_layer_scales(mlb_op* op, int layer, double src_moment, double dst_field);
int mlb_longrange2d_get_layer_scales(const mlb_op* op, int layer, double* src_moment, double* dst_field);
/* setNewDataRequired / setCompileRequired (a negative value leaves a flag) */
int mlb_longrange2d_set_required(mlb_op* op, int new_data, int compile);
int mlb_longrange2d_get_required(const mlb_op* op, int* new_data, int* compile);
/* Dipole2D builder state (dip2d_luafuncs.lua:6-26 defaults, :48-162
 * setUnitCell / setOffset / setTruncation) and makeData (:540-660).  As in
 * the reference, changing the builder state does not mark new data
 * required. */
int mlb_dipole2d_set_unit_cell(mlb_op* op, int layer, const double ABC[9]);
int mlb_dipole2d_get_unit_cell(const mlb_op* op, int layer, double ABC[9]);
int mlb_dipole2d_set_offset(mlb_op* op, int layer, const double off[3]);
int mlb_dipole2d_get_offset(const mlb_op* op, int layer, double off[3]);
int mlb_dipole2d_set_truncation(mlb_op* op, const int t[4]);     /* radial, x, y, z */
int mlb_dipole2d_get_truncation(const mlb_op* op, int t[4]);
int mlb_dipole2d_make_data(mlb_op* op);
/* Magnetostatics2D: the same unit-cell and truncation state (the mlb_dipole2d
 * calls, offsets unused) plus a grain size per layer (mag2d_luafuncs.lua:
 * 93-122, default 1 x 1 x 1); mlb_dipole2d_make_data runs its builder
 * (:598-744): minus the demagnetising tensor of a source and a destination
 * prism (Newell's f and g, demag.cpp:196-350), summed over the in-plane
 * images within the truncations. */
int mlb_magnetostatics2d_set_grain_size(mlb_op* op, int layer, const double g[3]);
int mlb_magnetostatics2d_get_grain_size(const mlb_op* op, int layer, double g[3]);
/* Dipole2D / Magnetostatics2D tensor data files, the GAB_<nx>x<ny>x<nz>.<n>.lua
 * and MAB_... files of dip2d_luafuncs.lua:278-500 (dip2d_save, dip2d_load)
 * and mag2d_luafuncs.lua:278-480: write builds the arrays if new data is
 * required and writes the reference's layout (system size, builder state,
 * `% 16.15E` arrays [dest][src], a Lua loader); read sets the arrays, clears
 * new data required and marks compile required only when the file's kind,
 * size, unit cells, offsets or grain sizes and truncations match the
 * operator's (relative 1e-8, as sameInternals); *loaded says whether it did. */
int mlb_lr2d_write_data_file(mlb_op* op, const char* filename);
int mlb_lr2d_read_data_file(mlb_op* op, const char* filename, int* loaded);

/* ---------------------------------------------------------------- DipoleEwald3D
 * M/cpu/ewald3d/ewald3d.cpp: the dipolar tensor G_ab(r) of a periodic
 * lattice of nx x ny x nz unit cells by Ewald summation in FP64 (the
 * tensor source of LongRange3D in make_tensor.lua, which stores -G).
 * Defaults: cubic unit cell, NSites 10, tau 1e-3.  eta (the real/reciprocal
 * split) is searched at the first element after the geometry, tau or NSites
 * changed, as calcTensorElement does it: G_xx's N -> N + 1 shell at r = a1
 * minimised by golden sections with the shell count taken from the integer
 * part of tau (findEta(a1, tau), ewald3d.cpp:30) and tolerance 1e-3;
 * MLB_ESTATE when the search does not converge.  setTau ignores tau <= 0 and
 * setNSites n <= 1, as the reference.  ab = 3*a + b in XX..ZZ order. */
typedef struct mlb_ewald3d mlb_ewald3d;
int mlb_ewald3d_create(int nx, int ny, int nz, mlb_ewald3d** out);       /* DipoleEwald3D.new(nx,ny,nz) */
int mlb_ewald3d_destroy(mlb_ewald3d* e);
int mlb_ewald3d_set_unit_cell(mlb_ewald3d* e, const double a[3], const double b[3], const double c[3]);
int mlb_ewald3d_get_unit_cell(const mlb_ewald3d* e, double abc[9]);
int mlb_ewald3d_set_lattice_size(mlb_ewald3d* e, int nx, int ny, int nz);
int mlb_ewald3d_get_lattice_size(const mlb_ewald3d* e, int n3[3]);
int mlb_ewald3d_set_tau(mlb_ewald3d* e, double tau);
int mlb_ewald3d_get_tau(const mlb_ewald3d* e, double* tau);
int mlb_ewald3d_set_nsites(mlb_ewald3d* e, int n);
int mlb_ewald3d_get_nsites(const mlb_ewald3d* e, int* n);
int mlb_ewald3d_get_eta(const mlb_ewald3d* e, double* eta);
int mlb_ewald3d_get_volume(const mlb_ewald3d* e, double* v);           /* volume: supercell |u1.(u2 x u3)| */
/* calculateTensorElement(AB, {x,y,z}) at r = x a + y b + z c (host) */
int mlb_ewald3d_element(mlb_ewald3d* e, int ab, const int r3[3], double* out);
/* calculateTensorElementRealR(AB, {rx,ry,rz}) (host) */
int mlb_ewald3d_element_real(mlb_ewald3d* e, int ab, const double r[3], double* out);
/* B200 extension: every element of the lattice, out9[ab][x + nx*(y + ny*z)]
 * = calculateTensorElement(ab, {x,y,z}), one GPU thread per element (FP64). */
int mlb_ewald3d_tensor(mlb_ewald3d* e, double* out9);

/* ---------------------------------------------------------------- LLG
 * M/cpu/llg/llg.cpp:91-171, llgcartesian.cpp:90-278, llgquat.cpp:126-378. */
#define MLB_LLG_CARTESIAN 0
#define MLB_LLG_QUATERNION 1
int mlb_llg_create(int kind, mlb_llg** out);                            /* LLG.new("Cartesian") */
int mlb_llg_destroy(mlb_llg* l);
int mlb_llg_kind(const mlb_llg* l, int* kind);                          /* MLB_LLG_CARTESIAN or _QUATERNION */
/* thermalOnlyFirstTerm (default 1), disableRenormalization (0),
 * unphysical precession / damping scales (1, 1). */
int mlb_llg_set_flags(mlb_llg* l, int thermal_only_first_term, int disable_renormalization,
                      double precess_scale, double damp_scale);
/* llg:apply(from[, scale], dmdt, to[, advance]) */
int mlb_llg_apply(mlb_llg* l, mlb_system* from, double scale, mlb_system* dmdt, mlb_system* to,
                  int advance);

/* ---------------------------------------------------------------- operator and LLG streams
 * encode / decode of operators and integrators: the bytes the reference's
 * CPU build writes for them inside a checkpoint, as exported Lua values
 * (LUA_TUSERDATA, type id, char 111 and the object index, then the class's
 * encode): Exchange (M/cpu/exchange/spinoperationexchange.cpp:52-112),
 * Anisotropy (M/cpu/anisotropy/spinoperationanisotropy.cpp:191-236),
 * Anisotropy.Uniaxial (..._uniaxial.cpp:181-230), Anisotropy.Cubic
 * (..._cubic.cpp:239-290), Thermal (M/cpu/thermal/spinoperationthermal.cpp:
 * 51-77, its scale array an object of its own), AppliedField
 * (M/cpu/appliedfield/spinoperationappliedfield.cpp:33-58), Dipole
 * (M/cpu/dipole/spinoperationdipole.cpp:35-59 over LongRange's,
 * M/cpu/longrange/spinoperationlongrange.cpp:55-95), LLG.Cartesian and
 * LLG.Quaternion (M/cpu/llg/llg.cpp:50-88).  Arguments as for
 * mlb_system_encode / mlb_system_decode; *objects = the objects the stream
 * holds (2 for Thermal).  A plain LongRange gives MLB_EUNSUP: the
 * reference's LongRange::encode writes no object header, so its stream
 * cannot be read back.  Tensors, RNG state and injected noise are not part
 * of the streams (as in the reference); a decoded Dipole builds its tensor
 * on first use. */
int mlb_op_encode(mlb_op* op, int first_index, void* buf, size_t cap, size_t* len, int* objects);
int mlb_op_decode(const void* buf, size_t len, mlb_op** out, size_t* used, int* objects);
int mlb_llg_encode(mlb_llg* l, int first_index, void* buf, size_t cap, size_t* len, int* objects);
int mlb_llg_decode(const void* buf, size_t len, mlb_llg** out, size_t* used, int* objects);

/* ---------------------------------------------------------------- plans
 * B200 extension (the reference steps from Lua, one operator call at a time):
 * a plan captures the canonical step of a system (resetFields; each op's
 * apply; sumFields; llg:apply) as CUDA graphs so that one host call
 * enqueues a whole step.  Once a step leaves the convolution's x spectrum
 * carried, runs of four or more steps go four to a graph (dependent launches
 * across the step boundaries).  The Thermal counter and the applied field
 * (with its sweep) advance on the device; any other parameter change makes
 * the next launch capture again.  With timing = 1, every kernel of the step is
 * bracketed by graph event nodes and mlb_plan_kernel_times returns the
 * milliseconds of the last launched step per kernel (48-byte name slots).
 * With timing = 2 the step keeps its dependent launches and the fused (y,z)
 * and x passes of an FP32 dipole convolution record a device timeline
 * (%globaltimer): mlb_plan_device_times returns, in microseconds, each
 * pass's span over the steps launched since the previous call (one step:
 * that step's span) from its first CTA released from the dependency wait to
 * its last CTA's end (-1 where a pass did not run), and resets the stamps. */
typedef struct mlb_plan mlb_plan;
int mlb_plan_create(mlb_system* s, mlb_op* const* ops, int nops, mlb_llg* l, int timing, mlb_plan** out);
int mlb_plan_launch(mlb_plan* p, int nsteps);
int mlb_plan_kernel_times(mlb_plan* p, int cap, char* names, double* ms, int* count);
int mlb_plan_device_times(mlb_plan* p, double* yz_us, double* xstep_us);
int mlb_plan_destroy(mlb_plan* p);

/* ---------------------------------------------------------------- ensembles
 * B200 extension for the reference's batched form op:apply({ss1, ss2, ...})
 * (SpinOperation::apply(SpinSystem**, n), spinoperation.cpp:288-300; the
 * CUDA build's *_N kernels need equal sizes, e.g. cuda_llg_cart_apply_N,
 * M/cuda/llg_cuda/llgcartesian.cu:133): nrep independent replicas of uneven
 * sizes packed by size class.  One step is one captured CUDA graph: every
 * class's dipole passes (all its replicas per launch; classes outside the
 * power-of-two fast sizes run the generic passes replica by replica) on a
 * branch of its own, the branches concurrent, then one fused step kernel
 * whose CTAs walk a packed (replica, tile) table across all classes
 * (persistent when the tuner finds it faster).  All replicas share the
 * operator set of mlb_ensemble_cfg: nearest-neighbour Exchange (normalised
 * moments), uniform Anisotropy, Thermal (Philox), AppliedField with a
 * per-step sweep, Dipole (open or periodic in-plane images), LLG;
 * temperature and applied field (start and sweep) may differ per replica
 * (mlb_ensemble_set_replica_params).  Replica spins must share one length.
 * dims holds nx, ny, nz per replica.  The first run tunes the (y,z) pass of
 * every class and the fused kernel's tile size and grid by timing the
 * candidates, and keeps the choices per process and in a cache file
 * (MLB_TUNE_CACHE = its path or "off"; default
 * $XDG_CACHE_HOME/maglua_b200/tune.txt or ~/.cache/maglua_b200/tune.txt). */
typedef struct mlb_ensemble mlb_ensemble;
typedef struct mlb_ensemble_cfg {
    double alpha, gamma, dt;
    double J;                 /* exchange with the six neighbours */
    int pbc[3];               /* periodic x, y, z */
    double K;                 /* anisotropy strength along axis */
    double axis[3];
    double T;                 /* temperature */
    uint64_t seed;            /* Philox seed */
    double B[3];              /* applied field at the first step */
    double dB[3];             /* added after every step */
    double g;                 /* dipole strength (0: off) */
    int open_xy;              /* 1: zero-padded open in-plane boundaries */
    int llg;                  /* MLB_LLG_CARTESIAN or MLB_LLG_QUATERNION */
} mlb_ensemble_cfg;
int mlb_ensemble_create(int nrep, const int* dims, mlb_ensemble** out);
int mlb_ensemble_destroy(mlb_ensemble* e);
int mlb_ensemble_configure(mlb_ensemble* e, const mlb_ensemble_cfg* cfg);
int mlb_ensemble_set_spins(mlb_ensemble* e, int rep, const double* x, const double* y, const double* z);
int mlb_ensemble_get_spins(mlb_ensemble* e, int rep, double* x, double* y, double* z);
int mlb_ensemble_run(mlb_ensemble* e, int nsteps);
/* netMoment of every replica (8 numbers each, as mlb_system_netmoment with m = 1). */
int mlb_ensemble_netmoment(mlb_ensemble* e, double* out8);
int mlb_ensemble_info(mlb_ensemble* e, long long* nsites, int* block_size, double* time);
int mlb_ensemble_get_stream(mlb_ensemble* e, void** stream);
/* The ensemble's status word, as mlb_system_status (any replica). */
int mlb_ensemble_status(mlb_ensemble* e, int clear, unsigned* flags);
/* Temperature, applied field at the next step and its per-step sweep of
 * replica rep (mlb_ensemble_configure sets every replica to the cfg's
 * values); the per-replica form of Thermal:set and AppliedField:set
 * (spinoperationthermal.cpp:379-387, appliedfield_luafuncs.lua:46-60). */
int mlb_ensemble_set_replica_params(mlb_ensemble* e, int rep, double T, const double B[3], const double dB[3]);
/* The applied field replica rep takes at its next step. */
int mlb_ensemble_get_replica_field(mlb_ensemble* e, int rep, double B[3]);
/* The tuner's report of the last tuning (NUL-terminated text; *len = its
 * size with the NUL; buf == NULL asks for the size alone). */
int mlb_ensemble_tune_log(mlb_ensemble* e, char* buf, size_t cap, size_t* len);
/* The fused kernel's grid (0: one CTA per tile), the number of size classes
 * and how many of them run the generic (non power-of-two) passes. */
int mlb_ensemble_config_info(mlb_ensemble* e, int* grid, int* nclasses, int* generic_classes);

/* ---------------------------------------------------------------- fused run
 * B200 extension: nsteps repetitions of the canonical script step
 * (doc/manual/BasicMicromagneticSimulation.lua:84-94):
 *   ss:resetFields(); for op in ops: op:apply(ss); ss:sumFields(); llg:apply(ss)
 * with the per-step work captured in a CUDA graph.  The end state equals
 * issuing those calls one by one. */
int mlb_run(mlb_system* s, mlb_op* const* ops, int nops, mlb_llg* l, int nsteps);

/* The Dipole tensor cache files WAB_<nx>x<ny>.<v>.lua of the reference
 * (M/cpu/dipole/dipolesupport.cpp:256-643; written by dipole_write_matrix,
 * checked by dipoleParamsMatch, loaded by dipoleLoad :717-851).  write: the
 * operator's reference-layout tensor (computed first for a Dipole);
 * read: a file whose nx, ny, nz, gmax and unit cell match the operator
 * (MLB_EINVAL otherwise) becomes its tensor, so the lattice sum is skipped. */
int mlb_dipole_write_wab(mlb_op* op, const char* filename);
int mlb_dipole_read_wab(mlb_op* op, const char* filename);

/* ---------------------------------------------------------------- Runge-Kutta integrators
 * Replaces the script M/common/scripts/RungeKutta.lua:57-215
 * (make_rk_step_function(ss, type, {ops}, llg, temp) and its step function):
 * type is one of "RK1", "RK2", "K3", "RK4", "RK3", "RK4_38", "RK6", "BS3"
 * (the script's Butcher tables; another name is MLB_EINVAL with the script's
 * message).  ops make the deterministic field (resetFields, apply each,
 * sumFields); temp (may be NULL) is a Thermal operator applied after the
 * stages with llg:apply(ss, false).  The stage systems are copies of ss made
 * here (fields included), on ss's stream.  mlb_rk_step runs nsteps steps;
 * a step whose parameters did not change since the previous step runs as
 * a CUDA graph (the same kernels and arguments as the eager step, recorded
 * with their dependent-launch edges, the step graph updated in place), so
 * its results are those of eager steps bit for bit.  mlb_rk_set_graph(r, 0)
 * keeps every step eager; mlb_rk_graph_steps counts the graph steps run. */
typedef struct mlb_rk mlb_rk;
int mlb_rk_create(mlb_system* ss, const char* type, mlb_op* const* ops, int nops, mlb_llg* l, mlb_op* temp,
                  mlb_rk** out);
int mlb_rk_step(mlb_rk* r, int nsteps);
int mlb_rk_set_graph(mlb_rk* r, int on);
int mlb_rk_graph_steps(mlb_rk* r, long long* steps);
/* The step function called on another system of the same size, as the
 * script's step(ss_input, skip_temperature) (RungeKutta.lua:194-213). */
int mlb_rk_step_on(mlb_rk* r, mlb_system* ss, int skip_temperature);
int mlb_rk_destroy(mlb_rk* r);

/* Replaces M/common/scripts/AdaptiveTimeStep.lua:9-110
 * (make_adapt_step_function(ss, step, tolerance, llg, temp) and its step
 * function) over a Runge-Kutta scheme: one step of dt against two of dt/2
 * on copies of ss, compared with SpinSystem:diff; *accepted = 1 when the
 * difference is below tolerance (ss takes the half-step result and dt grows),
 * else 0 (ss unchanged, dt halves).  temp (may be NULL, then l may be NULL)
 * is the Thermal kick applied after an accepted step. */
typedef struct mlb_adapt mlb_adapt;
int mlb_adapt_create(mlb_system* ss, mlb_rk* step, double tolerance, mlb_llg* l, mlb_op* temp, mlb_adapt** out);
int mlb_adapt_step(mlb_adapt* a, int* accepted);
int mlb_adapt_destroy(mlb_adapt* a);

/* ---------------------------------------------------------------- learned dipolar surrogate
 * B200 extension, no counterpart in the reference.  A linear spectral-conv
 * network on the in-plane grid, with the (component, z) pairs as 3*nz
 * channels, predicts the Dipole/LongRange field change dH from the spin
 * change m - m0 since the last exact evaluation (M/cpu/longrange/
 * spinoperationlongrange.cpp:354-440 computes the exact field):
 *   dH[co](s) = sum_{|ox|,|oy| <= radius} sum_ci W[o][co][ci] (m - m0)[ci](s + o)
 *             + sum_{kx < modes_x, ky in the modes_y lowest |ky|}
 *                 w_kx/(nx ny) Re(e^{i k.s} sum_ci R_k[co][ci] (m - m0)^_k[ci])
 * evaluated in BF16 on the tcgen05 tensor cores with FP32 accumulation.
 * Needs an FP32 system, periodic in-plane lattice, nx a multiple of 128, ny
 * a multiple of 8 (of 4 when 3*nz > 16), 3*nz <= 32, modes_x, modes_y <= 16,
 * radius <= 3.  Parameters: W [(2r+1)^2][C][C], R [modes_x][modes_y][C][C][2]
 * (C = 3*nz), FP32 on the host side. */
typedef struct mlb_surrogate mlb_surrogate;
int mlb_surrogate_create(mlb_op* dipole, int modes_x, int modes_y, int radius, mlb_surrogate** out);
int mlb_surrogate_destroy(mlb_surrogate* s);
/* out: C, CP (padded channels), modes_x, modes_y, radius, number of W values, number of R values (floats) */
int mlb_surrogate_sizes(const mlb_surrogate* s, int out[7]);
int mlb_surrogate_get_params(mlb_surrogate* s, float* w, float* r);
int mlb_surrogate_set_params(mlb_surrogate* s, const float* w, const float* r);
/* Exact evaluation every k steps and whenever the estimated relative field
 * error eps * |dH| / |H| exceeds tol (eps: the validated relative error of
 * the predicted update, set by mlb_surrogate_validate or here when > 0). */
int mlb_surrogate_set_schedule(mlb_surrogate* s, int k, double tol, double eps);
/* Online training on the plain method: nsteps canonical steps of ss with
 * ops (which hold the surrogate's operator) and l; every step that is not
 * the first of a window of `window` steps is one Adam step on the pair
 * (m - m0, H - H0) with learning rate lr.  loss_out[0]: mean relative loss
 * |dH_pred - dH|^2 / |dH|^2 over the last quarter of the iterations. */
int mlb_surrogate_train(mlb_surrogate* s, mlb_system* ss, mlb_op* const* ops, int nops, mlb_llg* l, int nsteps,
                        int window, double lr, double* loss_out);
/* nsteps plain steps; at every step inside a window of `window` steps the
 * surrogate's field is compared with the exact one.  out: mean and max of
 * |dH_pred - dH|/|dH|, mean and max of |H_pred - H|/|H|, mean and max of
 * |H0 - H|/|H| (the field without the surrogate).  Sets eps to the max of
 * the first pair. */
int mlb_surrogate_validate(mlb_surrogate* s, mlb_system* ss, mlb_op* const* ops, int nops, mlb_llg* l, int nsteps,
                           int window, double out[6]);
/* nsteps canonical steps (captured) with the surrogate standing in for its
 * operator between exact evaluations: attach, run, detach. */
int mlb_surrogate_run(mlb_surrogate* s, mlb_system* ss, mlb_op* const* ops, int nops, mlb_llg* l, int nsteps);
/* From attach to detach every step of ss (eager calls, mlb_run, plans
 * captured meanwhile) takes the surrogate's operator field from the
 * surrogate, with the device schedule restarted (first step exact).  detach
 * collects the statistics of mlb_surrogate_stats. */
int mlb_surrogate_attach(mlb_surrogate* s, mlb_system* ss);
int mlb_surrogate_detach(mlb_system* ss);
/* out: exact evaluations, surrogate evaluations, failed residual checks of
 * the last run; *last_bound: the last estimated relative field error. */
int mlb_surrogate_stats(mlb_surrogate* s, long long out[3], double* last_bound);
/* Polls of each tensor-core completion wait (mbarrier try_wait) before it
 * gives up (default 2^24, about 0.1 s).  A wait that gives up sets the
 * surrogate's error flag, then waits (bounded again) for the launch's own
 * MMAs before its TMEM is read and freed, so the kernel always returns; the
 * next host call that reads the flag (forward, gradients, train, validate,
 * run) returns MLB_ECUDA and clears it.  0 makes every wait give up at once:
 * a way to exercise that path. */
int mlb_surrogate_set_wait_limit(mlb_surrogate* s, unsigned polls);
/* Host-array forms for checks: x (3 arrays of nx*ny*nz, SpinSystem layout)
 * -> dh = net(x); and the gradients of L = |net(x) - t|^2 / |t|^2 with
 * respect to W and R (p: the prediction the gradients used; may be NULL). */
int mlb_surrogate_forward(mlb_surrogate* s, const float* const x[3], float* const dh[3]);
int mlb_surrogate_gradients(mlb_surrogate* s, const float* const x[3], const float* const t[3], float* dw, float* dr,
                            float* const p[3], double* loss);

/* ---------------------------------------------------------------- no-allocation dipole field
 * No counterpart in the reference (LongRange::init allocates the FFT work
 * arrays per operator, M/cpu/longrange/spinoperationlongrange.cpp:98-139).
 * The Dipole / LongRange field of FP32 device spin arrays (sx, sy, sz: nx*ny*nz
 * each, layout x + nx*(y + ny*z)) into FP32 device field arrays (hx, hy, hz),
 * scaled by the operator's strength, on `stream` (NULL = the legacy default
 * stream), with no device or host allocation: the spectrum scratch is a
 * static device array of MLB_NOALLOC_SCRATCH_BYTES (16 MiB), enough for
 * Kx*3*nz*ny complex FP32 values with Kx = Px/2+1 (256x256x8 needs 6.3 MB).
 * Larger lattices return MLB_ERANGE.  The operator's tensor spectrum must
 * already exist (apply the operator once to an FP32 SpinSystem of its size;
 * that call allocates), else MLB_ESTATE.  It is for callers that cannot
 * allocate in the middle of a run: a host whose caching allocator already
 * holds the GPU's memory (a PyTorch job sized to the whole device), where a
 * cudaMalloc fails for want of memory or a cudaFree stalls the device, and
 * loops over trial configurations that must not pay an allocation per
 * evaluation.  The first call on each device looks
 * up the scratch's address with cudaGetSymbolAddress with that device
 * current; make it before any stream capture.  That address is kept for the
 * life of the process and does not survive a cudaDeviceReset.  The current
 * device must be the one the operator's tensor spectrum was built on, else
 * MLB_EINVAL before any launch.  Every call shares the one scratch: calls
 * that overlap in time (two streams, two threads) race on it and must be
 * serialised by the caller.  The scratch is part of this library's device
 * code: every device on which the library's kernels are loaded holds its
 * 16 MiB until the process exits, whether or not this call is used. */
#define MLB_NOALLOC_SCRATCH_BYTES 16777216u
int mlb_dipole_field_noalloc(mlb_op* op, const float* sx, const float* sy, const float* sz, float* hx, float* hy,
                             float* hz, void* stream);

#ifdef __cplusplus
}
#endif
#endif
