"""ctypes wrapper around the FP64 oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: the checker the CUDA path is compared against.
Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg import
this package; the product (maglua_b200) never does.
"""
import ctypes as C
import math
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")

MAX_SLOTS = 32
SLOT_NAME = 32


def build():
    """Compile oracle.c into liboracle.so (gcc -O2, as the reference's CFLAGS)."""
    subprocess.check_call(["make", "-s", "-C", _HERE, "liboracle.so"])


def _load():
    src = os.path.join(_HERE, "oracle.c")
    if (not os.path.exists(_LIB)) or os.path.getmtime(_LIB) < os.path.getmtime(src):
        build()
    return C.CDLL(_LIB)


class _SS(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("n", C.c_int),
        ("x", C.POINTER(C.c_double)), ("y", C.POINTER(C.c_double)),
        ("z", C.POINTER(C.c_double)), ("ms", C.POINTER(C.c_double)),
        ("alpha", C.c_double), ("gamma", C.c_double), ("dt", C.c_double), ("time", C.c_double),
        ("site_alpha", C.POINTER(C.c_double)), ("site_gamma", C.POINTER(C.c_double)),
        ("nslots", C.c_int),
        ("names", (C.c_char * SLOT_NAME) * MAX_SLOTS),
        ("hx", C.POINTER(C.c_double) * MAX_SLOTS),
        ("hy", C.POINTER(C.c_double) * MAX_SLOTS),
        ("hz", C.POINTER(C.c_double) * MAX_SLOTS),
        ("used", C.c_int * MAX_SLOTS),
    ]


class _MT(C.Structure):
    _fields_ = [("state", C.c_ulonglong * 624), ("pnext", C.c_int), ("left", C.c_int)]


class _LLG(C.Structure):
    _fields_ = [("thermal_only_first_term", C.c_int), ("disable_renormalization", C.c_int),
                ("precess_scale", C.c_double), ("damp_scale", C.c_double)]


class _StepCfg(C.Structure):
    _fields_ = [
        ("npath", C.c_int), ("from_", C.POINTER(C.c_int)), ("to", C.POINTER(C.c_int)),
        ("J", C.POINTER(C.c_double)), ("ex_normalize", C.c_int),
        ("nani", C.c_int), ("ani_site", C.POINTER(C.c_int)), ("ani_axis", C.POINTER(C.c_double)),
        ("ani_K", C.POINTER(C.c_double)),
        ("ncub", C.c_int), ("cub_site", C.POINTER(C.c_int)), ("cub_axes", C.POINTER(C.c_double)),
        ("cub_K", C.POINTER(C.c_double)), ("cub_quirk", C.c_int),
        ("T", C.c_double), ("rng", C.POINTER(_MT)),
        ("zeeman", C.c_int), ("B", C.c_double * 3),
        ("dipole", C.c_int), ("lr", C.c_void_p), ("g", C.c_double),
        ("llg_type", C.c_int), ("llg", _LLG),
    ]


lib = _load()
_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)
_PSS = C.POINTER(_SS)

lib.orc_ss_new.restype = _PSS
lib.orc_ss_new.argtypes = [C.c_int, C.c_int, C.c_int]
lib.orc_ss_free.argtypes = [_PSS]
lib.orc_ss_copy.argtypes = [_PSS, _PSS]
lib.orc_ss_slot.argtypes = [_PSS, C.c_char_p]
lib.orc_ss_find_slot.argtypes = [_PSS, C.c_char_p]
lib.orc_ss_field.restype = _D
lib.orc_ss_field.argtypes = [_PSS, C.c_char_p, C.c_int]
lib.orc_ss_set_spin.argtypes = [_PSS, C.c_int, C.c_double, C.c_double, C.c_double]
lib.orc_ss_set_site_alpha.argtypes = [_PSS, _D]
lib.orc_ss_set_site_gamma.argtypes = [_PSS, _D]
lib.orc_ss_reset_fields.argtypes = [_PSS]
lib.orc_ss_sum_fields.argtypes = [_PSS]
lib.orc_ss_sum_fields_weighted.argtypes = [_PSS, C.c_char_p, C.c_int, C.POINTER(C.c_char_p), _D]
lib.orc_ss_netmoment.argtypes = [_PSS, C.c_double, _D]
lib.orc_mt_seed.argtypes = [C.POINTER(_MT), C.c_ulonglong]
lib.orc_mt_seed_array.argtypes = [C.POINTER(_MT), C.POINTER(C.c_ulonglong), C.c_int]
lib.orc_mt_randint.restype = C.c_ulonglong
lib.orc_mt_randint.argtypes = [C.POINTER(_MT)]
lib.orc_mt_rand.restype = C.c_double
lib.orc_mt_rand.argtypes = [C.POINTER(_MT)]
lib.orc_mt_randnorm.restype = C.c_double
lib.orc_mt_randnorm.argtypes = [C.POINTER(_MT), C.c_double, C.c_double]
lib.orc_exchange_apply.argtypes = [_PSS, _I, _I, _D, C.c_int, C.c_int, C.c_double]
lib.orc_anisotropy_apply.argtypes = [_PSS, _I, _D, _D, C.c_int, C.c_double]
lib.orc_anisotropy_uniaxial_apply.argtypes = [_PSS, _I, _D, _D, _D, C.c_int, C.c_double, C.c_int]
lib.orc_anisotropy_cubic_apply.argtypes = [_PSS, _I, _D, _D, C.c_int, C.c_double, C.c_int]
lib.orc_cubic_axes.argtypes = [_D, _D, _D]
lib.orc_uniaxial_axis.argtypes = [_D, _D]
lib.orc_thermal_apply.argtypes = [_PSS, C.c_double, _D, C.c_double, C.POINTER(_MT)]
lib.orc_thermal_apply_noise.argtypes = [_PSS, C.c_double, _D, C.c_double, _D, _D, _D]
lib.orc_thermal_draw.argtypes = [_PSS, C.c_double, C.POINTER(_MT), _D, _D, _D]
lib.orc_zeeman_apply.argtypes = [_PSS, _D, C.c_double]
lib.orc_dipole_tensor.argtypes = [C.c_int, C.c_int, C.c_int, _I, _D, _D, _D, _D, _D, _D, _D]
lib.orc_magnetostatic_tensor.argtypes = [C.c_int, C.c_int, C.c_int, _I, _D, _D, C.c_double, _D, _D, _D, _D, _D, _D]
lib.orc_dipole_tensor_rings.argtypes = [C.c_int, C.c_int, C.c_int, _D, C.c_int, C.c_int, _D, _D, _D, _D, _D, _D]
lib.orc_longrange_apply.argtypes = [_PSS, C.c_char_p, _D * 6, C.c_double, C.c_double]
lib.orc_lr_new.restype = C.c_void_p
lib.orc_lr_new.argtypes = [C.c_int, C.c_int, C.c_int, _D * 6]
lib.orc_lr_apply.argtypes = [C.c_void_p, _PSS, C.c_char_p, C.c_double, C.c_double]
lib.orc_lr_free.argtypes = [C.c_void_p]
lib.orc_longrange3d_apply.argtypes = [_PSS, _D * 9, C.c_double, C.c_double]
lib.orc_dipole_direct.argtypes = [_PSS, _D, C.c_double, C.c_int, C.c_int, C.c_int, _D, _D, _D]
lib.orc_dipole_open_tensor.argtypes = [C.c_int, C.c_int, C.c_int, _D, _D]
lib.orc_dipole_direct_sites.argtypes = [C.c_int, C.c_int, C.c_int, _D, _D, _D, _D, C.c_double,
                                        C.POINTER(C.c_longlong), C.c_int, _D]
lib.orc_llg_default.argtypes = [C.POINTER(_LLG)]
lib.orc_llg_cart_apply.argtypes = [C.POINTER(_LLG), _PSS, C.c_double, _PSS, _PSS, C.c_int]
lib.orc_llg_quat_apply.argtypes = [C.POINTER(_LLG), _PSS, C.c_double, _PSS, _PSS, C.c_int]
lib.orc_fft1d.argtypes = [_D, C.c_int, C.c_int, C.c_int]
lib.orc_fft2d_layers.argtypes = [_D, C.c_int, C.c_int, C.c_int, C.c_int]
lib.orc_fft3d.argtypes = [_D, C.c_int, C.c_int, C.c_int, C.c_int]
lib.orc_run_steps.argtypes = [_PSS, C.POINTER(_StepCfg), C.c_int]


def _dp(a):
    return a.ctypes.data_as(_D)


def _ip(a):
    return a.ctypes.data_as(_I)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class MT:
    """Random.MersenneTwister restatement."""

    def __init__(self, seed=None, key=None):
        self.s = _MT()
        if key is not None:
            k = (C.c_ulonglong * len(key))(*key)
            lib.orc_mt_seed_array(C.byref(self.s), k, len(key))
        else:
            lib.orc_mt_seed(C.byref(self.s), seed)

    def randint(self):
        return lib.orc_mt_randint(C.byref(self.s))

    def rand(self):
        return lib.orc_mt_rand(C.byref(self.s))

    def normal(self):
        return lib.orc_mt_randnorm(C.byref(self.s), 0.0, 1.0)

    def ptr(self):
        return C.pointer(self.s)


class LLG:
    def __init__(self, kind="Cartesian", **kw):
        self.kind = kind
        self.s = _LLG()
        lib.orc_llg_default(C.byref(self.s))
        for k, v in kw.items():
            setattr(self.s, k, v)

    def apply(self, frm, scale=1.0, dmdt=None, to=None, advance=True):
        dmdt = dmdt or frm
        to = to or frm
        f = lib.orc_llg_cart_apply if self.kind == "Cartesian" else lib.orc_llg_quat_apply
        f(C.byref(self.s), frm.p, scale, dmdt.p, to.p, int(bool(advance)))


class SpinSystem:
    """FP64 SpinSystem with numpy views of its arrays."""

    def __init__(self, nx, ny=1, nz=1):
        self.p = lib.orc_ss_new(nx, ny, nz)
        self.nx, self.ny, self.nz = nx, ny, nz
        self.n = nx * ny * nz
        s = self.p.contents
        self.x = np.ctypeslib.as_array(s.x, shape=(self.n,))
        self.y = np.ctypeslib.as_array(s.y, shape=(self.n,))
        self.z = np.ctypeslib.as_array(s.z, shape=(self.n,))
        self.ms = np.ctypeslib.as_array(s.ms, shape=(self.n,))

    def __del__(self):
        try:
            lib.orc_ss_free(self.p)
        except Exception:
            pass

    def __getattr__(self, k):
        if k in ("alpha", "gamma", "dt", "time"):
            return getattr(self.p.contents, k)
        raise AttributeError(k)

    def __setattr__(self, k, v):
        if k in ("alpha", "gamma", "dt", "time"):
            setattr(self.p.contents, k, float(v))
        else:
            object.__setattr__(self, k, v)

    def set_spins(self, x, y, z):
        """SpinSystem::set(i, sx, sy, sz) for every site (ms = |s|)."""
        x, y, z = _f64(x), _f64(y), _f64(z)
        self.x[:] = x
        self.y[:] = y
        self.z[:] = z
        self.ms[:] = np.sqrt(x * x + y * y + z * z)

    def spins(self):
        return np.stack([self.x.copy(), self.y.copy(), self.z.copy()])

    def field(self, name):
        ptrs = [lib.orc_ss_field(self.p, name.encode(), c) for c in range(3)]
        return np.stack([np.ctypeslib.as_array(q, shape=(self.n,)).copy() for q in ptrs])

    def field_views(self, name):
        ptrs = [lib.orc_ss_field(self.p, name.encode(), c) for c in range(3)]
        return [np.ctypeslib.as_array(q, shape=(self.n,)) for q in ptrs]

    def slot_used(self, name):
        s = lib.orc_ss_find_slot(self.p, name.encode())
        return s >= 0 and bool(self.p.contents.used[s])

    def set_slot_used(self, name, used=True):
        s = lib.orc_ss_slot(self.p, name.encode())
        self.p.contents.used[s] = int(bool(used))

    def set_site_alpha(self, a):
        self._sa = None if a is None else _f64(a)
        lib.orc_ss_set_site_alpha(self.p, None if a is None else _dp(self._sa))

    def set_site_gamma(self, g):
        self._sg = None if g is None else _f64(g)
        lib.orc_ss_set_site_gamma(self.p, None if g is None else _dp(self._sg))

    def reset_fields(self):
        lib.orc_ss_reset_fields(self.p)

    def sum_fields(self):
        lib.orc_ss_sum_fields(self.p)

    def sum_fields_weighted(self, dest, names, weights):
        arr = (C.c_char_p * len(names))(*[n.encode() for n in names])
        w = _f64(weights)
        lib.orc_ss_sum_fields_weighted(self.p, dest.encode(), len(names), arr, _dp(w))

    def netmoment(self, m=1.0):
        out = np.zeros(8)
        lib.orc_ss_netmoment(self.p, m, _dp(out))
        return out

    def copy_from(self, other):
        lib.orc_ss_copy(self.p, other.p)


# ---------------------------------------------------------------- operators
def exchange_apply(ss, frm, to, J, normalize=True, gscale=1.0):
    f, t, j = _i32(frm), _i32(to), _f64(J)
    lib.orc_exchange_apply(ss.p, _ip(f), _ip(t), _dp(j), len(f), int(normalize), gscale)


def anisotropy_apply(ss, site, axis, K, gscale=1.0):
    s, a, k = _i32(site), _f64(axis).reshape(-1), _f64(K)
    lib.orc_anisotropy_apply(ss.p, _ip(s), _dp(a), _dp(k), len(s), gscale)


def anisotropy_uniaxial_apply(ss, site, axis, K1, K2, gscale=1.0, quirk=True):
    s, a, k1, k2 = _i32(site), _f64(axis).reshape(-1), _f64(K1), _f64(K2)
    lib.orc_anisotropy_uniaxial_apply(ss.p, _ip(s), _dp(a), _dp(k1), _dp(k2), len(s), gscale, int(quirk))


def anisotropy_cubic_apply(ss, site, axes, K, gscale=1.0, quirk=True):
    s, a, k = _i32(site), _f64(axes).reshape(-1), _f64(K).reshape(-1)
    lib.orc_anisotropy_cubic_apply(ss.p, _ip(s), _dp(a), _dp(k), len(s), gscale, int(quirk))


def cubic_axes(a1, a2):
    a, b, out = _f64(a1), _f64(a2), np.zeros(9)
    rc = lib.orc_cubic_axes(_dp(a), _dp(b), _dp(out))
    return rc, out


def uniaxial_axis(a):
    a, out = _f64(a), np.zeros(3)
    lib.orc_uniaxial_axis(_dp(a), _dp(out))
    return out


def thermal_apply(ss, T, rng, scale=None, gscale=1.0):
    sc = None if scale is None else _f64(scale)
    return lib.orc_thermal_apply(ss.p, T, None if sc is None else _dp(sc), gscale, rng.ptr())


def thermal_draw(ss, T, rng):
    nx, ny, nz = np.zeros(ss.n), np.zeros(ss.n), np.zeros(ss.n)
    lib.orc_thermal_draw(ss.p, T, rng.ptr(), _dp(nx), _dp(ny), _dp(nz))
    return nx, ny, nz


def thermal_apply_noise(ss, T, noise, scale=None, gscale=1.0):
    nx, ny, nz = (_f64(a) for a in noise)
    sc = None if scale is None else _f64(scale)
    lib.orc_thermal_apply_noise(ss.p, T, None if sc is None else _dp(sc), gscale,
                                _dp(nx), _dp(ny), _dp(nz))


def zeeman_apply(ss, B, gscale=1.0):
    b = _f64(B)
    lib.orc_zeeman_apply(ss.p, _dp(b), gscale)


def dipole_tensor(nx, ny, nz, gmax=(1000, 1000, 1000, 1000), ABC=(1, 0, 0, 0, 1, 0, 0, 0, 1)):
    """Six arrays of shape (2nz-1, ny, nx): XX, XY, XZ, YY, YZ, ZZ."""
    g = _i32(gmax)
    abc = _f64(ABC)
    n = nx * ny * (2 * nz - 1)
    arrs = [np.zeros(n) for _ in range(6)]
    lib.orc_dipole_tensor(nx, ny, nz, _ip(g), _dp(abc), *[_dp(a) for a in arrs])
    return [a.reshape(2 * nz - 1, ny, nx) for a in arrs]


def magnetostatic_tensor(nx, ny, nz, gmax=(1000, 1000, 1000, 1000), ABC=(1, 0, 0, 0, 1, 0, 0, 0, 1),
                         prism=(1.0, 1.0, 1.0), tol=1e-5):
    """The Magnetostatic tensor (orc_magnetostatic_tensor): six arrays of
    shape (2nz-1, ny, nx), XX, XY, XZ, YY, YZ, ZZ."""
    g = _i32(gmax)
    abc, pr = _f64(ABC), _f64(prism)
    n = nx * ny * (2 * nz - 1)
    arrs = [np.zeros(n) for _ in range(6)]
    lib.orc_magnetostatic_tensor(nx, ny, nz, _ip(g), _dp(abc), _dp(pr), float(tol), *[_dp(a) for a in arrs])
    return [a.reshape(2 * nz - 1, ny, nx) for a in arrs]


def dipole_tensor_rings(nx, ny, nz, nrings=1000, lstep=5, ABC=(1, 0, 0, 0, 1, 0, 0, 0, 1)):
    """The Dipole tensor of truncation math.huge (orc_dipole_tensor_rings):
    six arrays of shape (2nz-1, ny, nx)."""
    abc = _f64(ABC)
    n = nx * ny * (2 * nz - 1)
    arrs = [np.zeros(n) for _ in range(6)]
    lib.orc_dipole_tensor_rings(nx, ny, nz, _dp(abc), int(nrings), int(lstep), *[_dp(a) for a in arrs])
    return [a.reshape(2 * nz - 1, ny, nx) for a in arrs]


class LongRange:
    """LongRange/Dipole with cached tensor transforms."""

    def __init__(self, nx, ny, nz, T6):
        self.T6 = [_f64(t).reshape(-1) for t in T6]
        arr = (_D * 6)(*[_dp(t) for t in self.T6])
        self.c = lib.orc_lr_new(nx, ny, nz, arr)

    def apply(self, ss, g, slot="Dipole", gscale=1.0):
        lib.orc_lr_apply(self.c, ss.p, slot.encode(), g, gscale)

    def __del__(self):
        try:
            lib.orc_lr_free(self.c)
        except Exception:
            pass


def longrange3d_apply(ss, T9, g, gscale=1.0):
    T9 = [_f64(t).reshape(-1) for t in T9]
    arr = (_D * 9)(*[_dp(t) for t in T9])
    lib.orc_longrange3d_apply(ss.p, arr, g, gscale)


def dipole_direct_sites(dims, spins, g, sites, ABC=(1, 0, 0, 0, 1, 0, 0, 0, 1)):
    """Open-boundary direct dipole sum at the listed target sites only
    (3 x len(sites)); spins are 3 arrays of nx*ny*nz in SpinSystem order."""
    nx, ny, nz = dims
    x, y, z = (_f64(a) for a in spins)
    st = np.ascontiguousarray(sites, dtype=np.int64)
    out = np.zeros(3 * len(st))
    lib.orc_dipole_direct_sites(nx, ny, nz, _dp(x), _dp(y), _dp(z), _dp(_f64(ABC)), g,
                                st.ctypes.data_as(C.POINTER(C.c_longlong)), len(st), _dp(out))
    return out.reshape(-1, 3).T


def dipole_direct(ss, g, periodic=(0, 0, 0), ABC=(1, 0, 0, 0, 1, 0, 0, 0, 1)):
    abc = _f64(ABC)
    hx, hy, hz = np.zeros(ss.n), np.zeros(ss.n), np.zeros(ss.n)
    lib.orc_dipole_direct(ss.p, _dp(abc), g, *[int(p) for p in periodic], _dp(hx), _dp(hy), _dp(hz))
    return np.stack([hx, hy, hz])


def dipole_open_tensor(nx, ny, nz, ABC=(1, 0, 0, 0, 1, 0, 0, 0, 1)):
    """Gamma(r) of every offset of an open lattice (orc_dipole_open_tensor):
    six arrays XX..ZZ shaped (2nz-1, 2ny-1, 2nx-1), offset d at index d + n - 1."""
    abc = _f64(ABC)
    L = (2 * nx - 1) * (2 * ny - 1) * (2 * nz - 1)
    out = np.zeros(6 * L)
    lib.orc_dipole_open_tensor(nx, ny, nz, _dp(abc), _dp(out))
    return out.reshape(6, 2 * nz - 1, 2 * ny - 1, 2 * nx - 1)


class DipoleOpen:
    """The physical open-boundary dipole field h_t = g sum_s Gamma(r_t - r_s) s_s
    (the kernel of dipole_direct with no images) as a linear convolution by
    FP64 FFT (numpy.fft) on a grid padded to 2n per axis: the same sum as
    dipole_direct, in O(N log N), for trajectories of lattices too large for
    the direct sum."""

    def __init__(self, nx, ny, nz, ABC=(1, 0, 0, 0, 1, 0, 0, 0, 1)):
        self.dims = (nx, ny, nz)
        self.P = (2 * nz, 2 * ny, 2 * nx)
        T = dipole_open_tensor(nx, ny, nz, ABC)
        grid = np.zeros((6,) + self.P)
        # offset d lands at index d mod P (negative offsets wrap): circular = linear on the padded grid
        iz = np.arange(-(nz - 1), nz) % self.P[0]
        iy = np.arange(-(ny - 1), ny) % self.P[1]
        ix = np.arange(-(nx - 1), nx) % self.P[2]
        grid[:, iz[:, None, None], iy[None, :, None], ix[None, None, :]] = T
        self.TK = np.fft.rfftn(grid, axes=(1, 2, 3))

    def field(self, spins, g):
        nx, ny, nz = self.dims
        S = np.zeros((3,) + self.P)
        S[:, :nz, :ny, :nx] = np.asarray(spins, dtype=np.float64).reshape(3, nz, ny, nx)
        SK = np.fft.rfftn(S, axes=(1, 2, 3))
        t = self.TK
        HK = np.stack([t[0] * SK[0] + t[1] * SK[1] + t[2] * SK[2],
                       t[1] * SK[0] + t[3] * SK[1] + t[4] * SK[2],
                       t[2] * SK[0] + t[4] * SK[1] + t[5] * SK[2]])
        H = np.fft.irfftn(HK, s=self.P, axes=(1, 2, 3))[:, :nz, :ny, :nx]
        return g * H.reshape(3, -1)

    def apply(self, ss, g, slot="Dipole"):
        h = self.field(ss.spins(), g)
        v = ss.field_views(slot)
        for c in range(3):
            v[c][:] = h[c]
        ss.set_slot_used(slot, True)


# ---------------------------------------------------------------- LongRange2D / Dipole2D
def longrange2d_apply(spins, T, src_scale, dst_scale, gscale=1.0):
    """LongRange2D compile and apply (spinoperationlongrange2d.cpp:387-530).
    spins (3, nz, ny, nx); T (nz, nz, 9, ny, nx), T[i][j][ab] the array set
    for (dest i, src j).  compile: q = 2D transform of each array / (nx ny);
    apply: H_a[d] = sum_s src_scale[s] sum_b q[s][d][a b] M_b[s] (the
    tensors read [s][d]), unnormalised inverse transform, real part, times
    dst_scale[d] * gscale.  Returns (3, nz, ny, nx)."""
    spins = np.asarray(spins, dtype=np.float64)
    T = np.asarray(T, dtype=np.float64)
    _, nz, ny, nx = spins.shape
    q = np.fft.fft2(T, axes=(-2, -1)) / (nx * ny)
    S = np.fft.fft2(spins, axes=(-2, -1))
    H = np.zeros((3, nz, ny, nx), dtype=complex)
    for a in range(3):
        for d in range(nz):
            for s_ in range(nz):
                for b in range(3):
                    H[a, d] += src_scale[s_] * q[s_, d, 3 * a + b] * S[b, s_]
    h = np.fft.ifft2(H, axes=(-2, -1)).real * (nx * ny)
    return h * (np.asarray(dst_scale, dtype=np.float64) * gscale)[None, :, None, None]


def _d2_xx(X, Y, Z):
    r = math.sqrt(X * X + Y * Y + Z * Z)
    if r < 1e-80:
        return 0.0
    ir = 1.0 / r
    ir3 = ir * ir * ir
    ir5 = ir3 * ir * ir
    return -1.0 * (ir3 - 3.0 * X * X * ir5)


def _d2_xy(X, Y, Z):
    r = math.sqrt(X * X + Y * Y + Z * Z)
    if r < 1e-80:
        return 0.0
    ir = 1.0 / r
    ir3 = ir * ir * ir
    ir5 = ir3 * ir * ir
    return -1.0 * (-3.0 * X * Y * ir5)


def dipole2d_tensor(nx, ny, nz, abc, off, trunc):
    """Dipole2D makeData (dip2d_luafuncs.lua:516-660, elements demag.cpp:
    3-56), pure Python: abc (nz, 3, 3) unit cell A, B, C per layer, off
    (nz, 3), trunc (radial, x, y, z).  Returns T (nz, nz, 9, ny, nx)
    indexed [dest][src][ab]."""
    abc = np.asarray(abc, dtype=np.float64).reshape(nz, 3, 3)
    off = np.asarray(off, dtype=np.float64).reshape(nz, 3)
    T = np.zeros((nz, nz, 9, ny, nx))

    def idx2pos(i, j, layer):
        dz = [0.0, 0.0, 0.0]
        for Z in range(layer):
            c = abc[Z][2]
            dz = [dz[0] + float(c[0]), dz[1] + float(c[1]), dz[2] + float(c[2])]
        A, B = abc[0][0], abc[0][1]
        di = [i * float(A[0]), i * float(A[1]), i * float(A[2])]
        dj = [j * float(B[1]), j * float(B[1]), j * float(B[2])]
        o = off[layer]
        return [di[k] + dj[k] + dz[k] + float(o[k]) for k in range(3)]

    tX, tY, tZ = int(trunc[1]), int(trunc[2]), int(trunc[3])
    for d in range(nz):
        for s_ in range(nz):
            if abs(s_ - d) > tZ:
                continue
            for X in range(-tX, tX + 1):
                for Y in range(-tY, tY + 1):
                    pd, ps = idx2pos(X, Y, d), idx2pos(X, Y, s_)
                    rx, ry, rz = ps[0] - pd[0], ps[1] - pd[1], ps[2] - pd[2]
                    x = X + 100000 * nx if X < 0 else X
                    y = Y + 100000 * ny if Y < 0 else Y
                    x, y = x % nx, y % ny
                    v = (_d2_xx(rx, ry, rz), _d2_xy(rx, ry, rz), _d2_xy(rx, rz, ry),
                         _d2_xy(ry, rx, rz), _d2_xx(ry, rx, rz), _d2_xy(ry, rz, rx),
                         _d2_xy(rz, rx, ry), _d2_xy(rz, ry, rx), _d2_xx(rz, rx, ry))
                    for ab in range(9):
                        T[d, s_, ab, y, x] += v[ab]
    return T


def _ms_log(num, den):
    out = np.zeros(np.broadcast(num, den).shape)
    m = (num != 0) & (den != 0)
    with np.errstate(divide="ignore", invalid="ignore"):
        out[m] = np.log(num[m] / den[m])
    return out


def _ms_atan(num, den):
    out = np.zeros(np.broadcast(num, den).shape)
    m = ~((num == 0) & (den == 0))
    out[m] = np.arctan2(num[m], den[m])
    return out


def _ms_f(X, Y, Z):
    """Newell's f (Newell, Williams and Dunlop 1993) in logarithms."""
    x, y, z = np.abs(X), np.abs(Y), np.abs(Z)
    xx, yy, zz = x * x, y * y, z * z
    R = np.sqrt(xx + yy + zz)
    return ((2 * xx - yy - zz) * R / 6 - x * y * z * _ms_atan(y * z, x * R)
            + (y / 4) * (zz - xx) * _ms_log((y + R) * (y + R), xx + zz)
            + (z / 4) * (yy - xx) * _ms_log((z + R) * (z + R), xx + yy))


def _ms_g(X, Y, Z):
    """Newell's g in logarithms, odd in X and in Y."""
    x, y, z = np.abs(X), np.abs(Y), np.abs(Z)
    xx, yy, zz = x * x, y * y, z * z
    R = np.sqrt(xx + yy + zz)
    sg = np.where(X < 0, -1.0, 1.0) * np.where(Y < 0, -1.0, 1.0)
    return sg * (-x * y * R / 3
                 - (z / 2) * (xx * _ms_atan(y * z, x * R) + yy * _ms_atan(x * z, y * R)
                              + (zz / 3) * _ms_atan(x * y, z * R))
                 + (x * y * z / 2) * _ms_log((z + R) * (z + R), xx + yy)
                 + (y / 12) * (3 * zz - yy) * _ms_log((x + R) * (x + R), yy + zz)
                 + (x / 12) * (3 * zz - xx) * _ms_log((y + R) * (y + R), xx + zz))


def _ms_pair(fn, X, Y, Z, d1, d2):
    sg = (1.0, -1.0, 1.0, -1.0)
    ox = (0.0, d2[0], d2[0] - d1[0], -d1[0])
    oy = (0.0, d2[1], d2[1] - d1[1], -d1[1])
    oz = (0.0, d2[2], d2[2] - d1[2], -d1[2])
    acc = np.zeros(np.shape(X))
    for a in range(4):
        for b in range(4):
            for c in range(4):
                acc = acc + sg[a] * sg[b] * sg[c] * fn(X + ox[a], Y + oy[b], Z + oz[c])
    return acc / (4.0 * math.pi * d2[0] * d2[1] * d2[2])


def magnetostatics2d_elements(rx, ry, rz, d1, d2):
    """The nine prism-prism elements XX..ZZ (magnetostatics2d/demag.cpp:
    256-350) for source prism d1 and destination prism d2 at offset r."""
    def P(d, i, j, k):
        return (d[i], d[j], d[k])
    xx = _ms_pair(_ms_f, rx, ry, rz, d1, d2)
    xy = _ms_pair(_ms_g, rx, ry, rz, d1, d2)
    xz = _ms_pair(_ms_g, rx, rz, ry, P(d1, 0, 2, 1), P(d2, 0, 2, 1))
    yy = _ms_pair(_ms_f, ry, rx, rz, P(d1, 1, 0, 2), P(d2, 1, 0, 2))
    yz = _ms_pair(_ms_g, ry, rz, rx, P(d1, 1, 2, 0), P(d2, 1, 2, 0))
    zz = _ms_pair(_ms_f, rz, ry, rx, P(d1, 2, 1, 0), P(d2, 2, 1, 0))
    return [xx, xy, xz, xy, yy, yz, xz, yz, zz]


def magnetostatics2d_tensor(nx, ny, nz, abc, grain, trunc):
    """Magnetostatics2D makeData (mag2d_luafuncs.lua:598-744), vectorised
    over the in-plane images: abc (nz, 3, 3) unit cells, grain (nz, 3),
    trunc (radial, x, y, z).  Returns T (nz, nz, 9, ny, nx) indexed
    [source z1][destination z2][ab], each image adding -N."""
    abc = np.asarray(abc, dtype=np.float64).reshape(nz, 3, 3)
    grain = np.asarray(grain, dtype=np.float64).reshape(nz, 3)
    mx = int(trunc[0])
    Xs = [X for X in range(-mx, mx + 1) if abs(X) <= trunc[1]]
    Ys = [Y for Y in range(-mx, mx + 1) if abs(Y) <= trunc[2]]
    XX, YY = np.meshgrid(np.asarray(Xs, float), np.asarray(Ys, float), indexing="ij")
    xi = XX.astype(int) % nx
    yi = YY.astype(int) % ny
    A, B = abc[0][0], abc[0][1]
    T = np.zeros((nz, nz, 9, ny, nx))
    for z1 in range(nz):
        c1 = np.zeros(3)
        for j in range(z1):
            c1 = c1 + abc[j][2]
        for z2 in range(nz):
            if abs(z1 - z2) > trunc[3]:
                continue
            c2 = np.zeros(3)
            for j in range(z2):
                c2 = c2 + abc[j][2]
            c = c2 - c1
            rx = A[0] * XX + B[0] * YY + c[0]
            ry = A[1] * XX + B[1] * YY + c[1]
            rz = A[2] * XX + B[2] * YY + c[2]
            v = magnetostatics2d_elements(rx, ry, rz, grain[z1], grain[z2])
            for k in range(9):
                np.add.at(T[z1, z2, k], (yi, xi), -v[k])
    return T


# ---------------------------------------------------------------- DipoleEwald3D
def ewald_geometry(d, a):
    """Supercell vectors, reciprocal vectors and volume (ewald3d.cpp:76-104)."""
    u = [[d[i] * a[i][c] for c in range(3)] for i in range(3)]

    def cross(p, q):
        return [p[1] * q[2] - p[2] * q[1], p[2] * q[0] - p[0] * q[2], p[0] * q[1] - p[1] * q[0]]

    def dot(p, q):
        return p[0] * q[0] + p[1] * q[1] + p[2] * q[2]

    c23, c31, c12 = cross(u[1], u[2]), cross(u[2], u[0]), cross(u[0], u[1])
    vu = abs(dot(u[0], c23))
    b = [[2.0 * math.pi * c23[c] / vu for c in range(3)], [2.0 * math.pi * c31[c] / vu for c in range(3)],
         [2.0 * math.pi * c12[c] / vu for c in range(3)]]
    return u, b, vu


def _ew_term(g, alpha, beta, r, eta, n, m, k):
    u, b, vu = g
    eta2 = eta * eta
    delta = 1.0 if alpha == beta else 0.0
    Q = [n * b[0][i] + m * b[1][i] + k * b[2][i] for i in range(3)]
    r0 = (r[0] * r[0] + r[1] * r[1] + r[2] * r[2]) == 0
    if r0:
        R = [n * u[0][i] + m * u[1][i] + k * u[2][i] for i in range(3)]
    else:
        R = [n * u[0][i] + m * u[1][i] + k * u[2][i] + r[i] for i in range(3)]
    Q2 = Q[0] * Q[0] + Q[1] * Q[1] + Q[2] * Q[2]
    if math.sqrt(Q2) > 0:
        if r0:
            rec = -4.0 * math.pi * math.exp(-Q2 / (4.0 * eta2)) * (Q2 * delta - 3 * Q[alpha] * Q[beta]) / (3.0 * vu * Q2)
        else:
            rq = r[0] * Q[0] + r[1] * Q[1] + r[2] * Q[2]
            rec = 4.0 * math.pi * Q[alpha] * Q[beta] * math.cos(rq) * math.exp(-Q2 / (4.0 * eta2)) / (Q2 * vu)
    else:
        rec = 0.0
    Rab = R[alpha] * R[beta]
    R2 = R[0] * R[0] + R[1] * R[1] + R[2] * R[2]
    R1 = math.sqrt(R2)
    R4 = R2 * R2
    R5 = R4 * R1
    sp = 1.772453850905516027
    if R1 > 0:
        if r0:
            real = (R2 * delta - 3.0 * R[alpha] * R[beta]) * (
                2.0 * eta * math.exp(-R2 * eta2) * (3.0 + 2.0 * R2 * eta2) / (3.0 * R4 * sp) + math.erfc(R1 * eta) / R5)
        else:
            real = (2.0 * eta * math.exp(-eta2 * R2) * (R2 * delta - 3.0 * Rab - 2.0 * eta2 * Rab * R2) / (sp * R4)
                    + (R2 * delta - 3.0 * Rab) * math.erfc(eta * R1) / R5)
    else:
        real = 0.0
    return real, rec


def ewald_element(g, alpha, beta, r, eta, N):
    """G_ab(r) (ewald3d.cpp:330-358): real and reciprocal parts summed
    separately over n, m, k in [-N, N]."""
    tq = tr = 0.0
    for n in range(-N, N + 1):
        for m in range(-N, N + 1):
            for k in range(-N, N + 1):
                a, b = _ew_term(g, alpha, beta, r, eta, n, m, k)
                tr += a
                tq += b
    return tq + tr


def ewald_next_shell(g, alpha, beta, r, eta, N):
    """G(N + 1) - G(N) by its surface shell (ewald3d.cpp:361-422)."""
    tq = tr = 0.0
    M = N + 1
    faces = [[(n, m, M) for n in range(-M, M + 1) for m in range(-M, M + 1)],
             [(n, M, k) for n in range(-M, M + 1) for k in range(-N, N + 1)],
             [(M, m, k) for m in range(-N, N + 1) for k in range(-N, N + 1)]]
    for fi, face in enumerate(faces):
        for t in face:
            neg = list(t)
            neg[2 - fi] = -neg[2 - fi]
            a1, b1 = _ew_term(g, alpha, beta, r, eta, *t)
            a2, b2 = _ew_term(g, alpha, beta, r, eta, *neg)
            tr += a1
            tq += b1
            tr += a2
            tq += b2
    return tq + tr


def ewald_find_eta(g, r3, N, tol=1e-3):
    """Golden-section search for eta (ewald3d.cpp:109-218); None when the 100
    levels run out."""
    RGR, MINA = 0.3819660112501051518, 1e-10

    def F(x):
        return abs(ewald_next_shell(g, 0, 0, r3, x, N))

    def rec(depth, a, fa, b, fb, c, fc):
        if depth < 0:
            return None
        if a > MINA and fa < fb < fc:
            x = c + RGR * (c - b)
            return rec(depth - 1, b, fb, c, fc, x, F(x))
        if fa > fb > fc:
            x = a - RGR * (b - a)
            return rec(depth - 1, x, F(x), a, fa, b, fb)
        if (c - b) > (b - a):
            x = b + RGR * (c - b)
            if (c - a) < tol * (abs(b) + abs(x)):
                return (c + a) * 0.5
            fx = F(x)
            if fx < fb:
                return rec(depth - 1, b, fb, x, fx, c, fc)
            return rec(depth - 1, a, fa, b, fb, x, fx)
        x = b - RGR * (b - a)
        if (c - a) < tol * (abs(b) + abs(x)):
            return (c + a) * 0.5
        fx = F(x)
        if fx < fb:
            return rec(depth - 1, a, fa, x, fx, b, fb)
        return rec(depth - 1, x, fx, b, fb, c, fc)

    a, c = MINA, 1000.0
    b = a + RGR * (c - a)
    return rec(100, a, F(a), b, F(b), c, F(c))


# ------------------------------------------------------------ SpinSystem encode
# The LuaBaseObject byte stream (M/common/luabaseobject/luabaseobject.cpp:
# 142-205, 250-360): native-endian int32, double and char with no padding;
# an object is LUA_TUSERDATA (7), its type id, then its own encode, which
# opens with ENCODE_PREAMBLE: char 111 (new) and its index in the stream's
# object list, or char 222 (seen before) and that index.

LUA_TUSERDATA = 7
LUA_TNIL = 0
ENC_NEW = 111
ENC_OLD = 222


def type_hash32(name):
    """hash32 (M/common/luabaseobject/factory.cpp:123-131): MurmurHash3
    x86_32 of the type name with seed 1000 as the reference wrote it
    (MurmurHash3.cpp:101-155), whose tail block rotates by 16 where the
    published algorithm rotates by 15; returned as a signed int."""
    data = name.encode()
    c1, c2, M = 0xCC9E2D51, 0x1B873593, 0xFFFFFFFF
    rotl = lambda x, r: ((x << r) | (x >> (32 - r))) & M
    h = 1000
    nb = len(data) // 4
    for i in range(nb):
        k = int.from_bytes(data[4 * i:4 * i + 4], "little")
        k = rotl((k * c1) & M, 15)
        k = (k * c2) & M
        h = rotl(h ^ k, 13)
        h = (h * 5 + 0xE6546B64) & M
    tail = data[4 * nb:]
    k = 0
    if len(tail) >= 3:
        k ^= tail[2] << 16
    if len(tail) >= 2:
        k ^= tail[1] << 8
    if len(tail) >= 1:
        k ^= tail[0]
        k = rotl((k * c1) & M, 16)
        k = (k * c2) & M
        h ^= k
    h ^= len(data)
    h ^= h >> 16
    h = (h * 0x85EBCA6B) & M
    h ^= h >> 13
    h = (h * 0xC2B2AE35) & M
    h ^= h >> 16
    return h - (1 << 32) if h >= 1 << 31 else h


def _enc_darray(out, idx, a, dims):
    """encodeT<dArray> (luabaseobject.h:101-106) of Array<double>::encode
    (M/cpu/array/array_core_cpu.h:200-225): version 0, nx, ny, nz, then flag
    1 and one double when every value compares equal, else flag 0 and the
    values in site order."""
    import struct
    a = np.ascontiguousarray(a, dtype=np.float64).ravel()
    out += struct.pack("=iibib", LUA_TUSERDATA, type_hash32("Array.Double"), ENC_NEW, idx, 0)
    out += struct.pack("=iii", *dims)
    if a.size and np.all(a == a[0]):
        out += struct.pack("=id", 1, float(a[0]))
    else:
        out += struct.pack("=i", 0) + a.tobytes()


def encode_spinsystem(nx, ny, nz, alpha, dt, gamma, time, x, y, z, ms, site_alpha=None,
                      site_gamma=None, first_index=0):
    """SpinSystem::encode (M/cpu/core/spinsystem.cpp:669-757) as exported as a
    Lua value (luamigrate.cpp:75-76, 265-275): the system's header, version 0,
    nx, ny, nz, alpha, dt, gamma, time, the arrays x, y, z, ms, the flag and
    array of per-site alpha, then of per-site gamma, and the count of sites
    with extra data (0: none).  first_index: the system's index in the
    stream's object list (its arrays take the next ones)."""
    import struct
    out = bytearray()
    out += struct.pack("=iibib", LUA_TUSERDATA, type_hash32("SpinSystem"), ENC_NEW, first_index, 0)
    out += struct.pack("=iii", nx, ny, nz)
    out += struct.pack("=dddd", alpha, dt, gamma, time)
    dims = (nx, ny, nz)
    idx = first_index + 1
    for a in (x, y, z, ms):
        _enc_darray(out, idx, a, dims)
        idx += 1
    for a in (site_alpha, site_gamma):
        out += struct.pack("=i", 0 if a is None else 1)
        if a is not None:
            _enc_darray(out, idx, a, dims)
            idx += 1
    out += struct.pack("=i", 0)
    return bytes(out)


def _enc_op_head(out, type_name, idx, nx, ny, nz, gs):
    """encodeT header of an operator (type id, ENCODE_PREAMBLE) and
    SpinOperation::encode (M/cpu/core/spinoperation.cpp:67-75): version 0,
    nx, ny, nz, global scale."""
    import struct
    out += struct.pack("=iibib", LUA_TUSERDATA, type_hash32(type_name), ENC_NEW, idx, 0)
    out += struct.pack("=iiid", nx, ny, nz, gs)


def encode_exchange(nx, ny, nz, gs, normalize, pbc, frm, to, J, first_index=0):
    """Exchange::encode (M/cpu/exchange/spinoperationexchange.cpp:52-73):
    version 1, normalizeMoments, pbc[3], the pathway count and (from, to, J)
    per pathway, sites 0-based as stored."""
    import struct
    out = bytearray()
    _enc_op_head(out, "Exchange", first_index, nx, ny, nz, gs)
    out += struct.pack("=biiiii", 1, int(normalize), *[int(p) for p in pbc], len(frm))
    for f, t, j in zip(frm, to, J):
        out += struct.pack("=iid", int(f), int(t), float(j))
    return bytes(out)


def anisotropy_add_axis(a):
    """The axis Anisotropy's Lua add stores (l_add,
    spinoperationanisotropy.cpp:385-398): divided by its length."""
    import math
    a0, a1, a2 = (float(v) for v in a)
    lena = math.sqrt(a0 * a0 + a1 * a1 + a2 * a2)
    return (a0 / lena, a1 / lena, a2 / lena)


def encode_anisotropy(nx, ny, nz, gs, sites, axes, K, first_index=0):
    """Anisotropy::encode (M/cpu/anisotropy/spinoperationanisotropy.cpp:
    191-207): version 0, the count, (site, axis[3], K) per entry."""
    import struct
    out = bytearray()
    _enc_op_head(out, "Anisotropy", first_index, nx, ny, nz, gs)
    out += struct.pack("=bi", 0, len(sites))
    for st, ax, k in zip(sites, axes, K):
        out += struct.pack("=idddd", int(st), *[float(v) for v in ax], float(k))
    return bytes(out)


def encode_uniaxial(nx, ny, nz, gs, sites, axes, K1, K2, first_index=0):
    """AnisotropyUniaxial::encode (..._uniaxial.cpp:181-199): version 0, the
    count, (site, axis[3], K1, K2) per entry."""
    import struct
    out = bytearray()
    _enc_op_head(out, "Anisotropy.Uniaxial", first_index, nx, ny, nz, gs)
    out += struct.pack("=bi", 0, len(sites))
    for st, ax, k1, k2 in zip(sites, axes, K1, K2):
        out += struct.pack("=iddddd", int(st), *[float(v) for v in ax], float(k1), float(k2))
    return bytes(out)


def encode_cubic(nx, ny, nz, gs, sites, axes9, K3, first_index=0):
    """AnisotropyCubic::encode (..._cubic.cpp:239-258): version 0, the count,
    (site, the first two axes, K[3]) per entry (the third axis is computed
    on decode)."""
    import struct
    out = bytearray()
    _enc_op_head(out, "Anisotropy.Cubic", first_index, nx, ny, nz, gs)
    out += struct.pack("=bi", 0, len(sites))
    for st, ax, k in zip(sites, axes9, K3):
        out += struct.pack("=i", int(st)) + struct.pack("=6d", *[float(v) for v in ax[:6]])
        out += struct.pack("=3d", *[float(v) for v in k])
    return bytes(out)


def encode_thermal(nx, ny, nz, gs, T, scale=None, first_index=0):
    """Thermal::encode (M/cpu/thermal/spinoperationthermal.cpp:51-61):
    version 0, the temperature, then scale->encode: the array's own
    ENCODE_PREAMBLE (char 111, the next object index) and Array::encode
    without an encodeT type header (array_core_cpu.h:200-225)."""
    import struct
    out = bytearray()
    _enc_op_head(out, "Thermal", first_index, nx, ny, nz, gs)
    out += struct.pack("=bd", 0, float(T))
    out += struct.pack("=bibiii", ENC_NEW, first_index + 1, 0, nx, ny, nz)
    a = np.ones(nx * ny * nz) if scale is None else np.ascontiguousarray(scale, dtype=np.float64).ravel()
    if np.all(a == a[0]):
        out += struct.pack("=id", 1, float(a[0]))
    else:
        out += struct.pack("=i", 0) + a.tobytes()
    return bytes(out)


def encode_appliedfield(nx, ny, nz, gs, B, first_index=0):
    """AppliedField::encode (spinoperationappliedfield.cpp:33-42): version
    0, B[3]."""
    import struct
    out = bytearray()
    _enc_op_head(out, "AppliedField", first_index, nx, ny, nz, gs)
    out += struct.pack("=bddd", 0, *[float(v) for v in B])
    return bytes(out)


def encode_dipole(nx, ny, nz, gs, gmax, g, ABC, first_index=0):
    """Dipole::encode (M/cpu/dipole/spinoperationdipole.cpp:35-41): the
    preamble, LongRange::encode (spinoperationlongrange.cpp:55-68: the base,
    version 0, gmax[4], g, ABC[9]), then the Dipole's version 0."""
    import struct
    out = bytearray()
    _enc_op_head(out, "Dipole", first_index, nx, ny, nz, gs)
    out += struct.pack("=biiii", 0, *[int(v) for v in gmax])
    out += struct.pack("=d", float(g)) + struct.pack("=9d", *[float(v) for v in ABC])
    out += struct.pack("=b", 0)
    return bytes(out)


def encode_llg(kind, thermal_only_first_term=1, disable_renormalization=0, precess=1.0, damp=1.0,
               first_index=0):
    """LLG::encode (M/cpu/llg/llg.cpp:50-60) of an LLG.Cartesian or
    LLG.Quaternion: version 1, the two flags, the precession and damping
    scales."""
    import struct
    return struct.pack("=iibibiidd", LUA_TUSERDATA, type_hash32("LLG." + kind), ENC_NEW, first_index, 1,
                       int(thermal_only_first_term), int(disable_renormalization), float(precess), float(damp))


def decode_spinsystem(buf):
    """SpinSystem::decode (spinsystem.cpp:759-851) of a stream that
    encode_spinsystem writes, or that has sites' extra data all nil; returns
    a dict of the scalars and arrays (site_alpha / site_gamma None when
    absent)."""
    import struct
    pos = 0

    def take(fmt):
        nonlocal pos
        v = struct.unpack_from("=" + fmt, buf, pos)
        pos += struct.calcsize("=" + fmt)
        return v

    objs = {}
    t, ty, magic, idx = take("iibi")
    assert t == LUA_TUSERDATA and ty == type_hash32("SpinSystem") and magic == ENC_NEW
    (ver,) = take("b")
    assert ver == 0
    nx, ny, nz = take("iii")
    alpha, dt, gamma, time = take("dddd")
    n = nx * ny * nz

    def arr():
        nonlocal pos
        t, ty, magic, idx = take("iibi")
        assert t == LUA_TUSERDATA and ty == type_hash32("Array.Double")
        if magic == ENC_OLD:
            return objs[idx]
        (ver,) = take("b")
        assert ver == 0
        dims = take("iii")
        assert dims == (nx, ny, nz)
        (flag,) = take("i")
        if flag == 1:
            (v,) = take("d")
            a = np.full(n, v)
        else:
            a = np.frombuffer(buf, dtype=np.float64, count=n, offset=pos).copy()
            pos += 8 * n
        objs[idx] = a
        return a

    d = dict(nx=nx, ny=ny, nz=nz, alpha=alpha, dt=dt, gamma=gamma, time=time)
    for k in ("x", "y", "z", "ms"):
        d[k] = arr()
    for k in ("site_alpha", "site_gamma"):
        (e,) = take("i")
        d[k] = arr() if e else None
    (ne,) = take("i")
    if ne < 0:
        for _ in range(n):
            (lt,) = take("i")
            assert lt == LUA_TNIL
    else:
        assert ne == 0
    assert pos == len(buf)
    return d


def fft1d(data, sign):
    d = np.ascontiguousarray(np.asarray(data, dtype=np.complex128)).copy()
    lib.orc_fft1d(d.view(np.float64).ctypes.data_as(_D), len(d), 1, sign)
    return d


def fft3d(data, sign):
    """data shaped (nz, ny, nx) complex."""
    d = np.ascontiguousarray(np.asarray(data, dtype=np.complex128)).copy()
    nz, ny, nx = d.shape
    lib.orc_fft3d(d.view(np.float64).ctypes.data_as(_D), nx, ny, nz, sign)
    return d


def fft2d_layers(data, sign):
    d = np.ascontiguousarray(np.asarray(data, dtype=np.complex128)).copy()
    nz, ny, nx = d.shape
    lib.orc_fft2d_layers(d.view(np.float64).ctypes.data_as(_D), nx, ny, nz, sign)
    return d


def run_steps(ss, nsteps, *, paths=None, ex_normalize=True, ani=None, cubic=None,
              cubic_quirk=True, T=0.0, rng=None, B=None, lr=None, g=0.0,
              llg="Cartesian", llg_kw=None):
    """Canonical step loop in C (used for CPU timing)."""
    c = _StepCfg()
    keep = []
    if paths is not None:
        f, t, j = _i32(paths[0]), _i32(paths[1]), _f64(paths[2])
        keep += [f, t, j]
        c.npath, c.from_, c.to, c.J = len(f), _ip(f), _ip(t), _dp(j)
        c.ex_normalize = int(ex_normalize)
    if ani is not None:
        s, a, k = _i32(ani[0]), _f64(ani[1]).reshape(-1), _f64(ani[2])
        keep += [s, a, k]
        c.nani, c.ani_site, c.ani_axis, c.ani_K = len(s), _ip(s), _dp(a), _dp(k)
    if cubic is not None:
        s, a, k = _i32(cubic[0]), _f64(cubic[1]).reshape(-1), _f64(cubic[2]).reshape(-1)
        keep += [s, a, k]
        c.ncub, c.cub_site, c.cub_axes, c.cub_K = len(s), _ip(s), _dp(a), _dp(k)
        c.cub_quirk = int(cubic_quirk)
    if T and rng is not None:
        c.T = T
        c.rng = rng.ptr()
    if B is not None:
        c.zeeman = 1
        for i in range(3):
            c.B[i] = B[i]
    if lr is not None:
        c.dipole = 1
        c.lr = lr.c
        c.g = g
    c.llg_type = 0 if llg == "Cartesian" else 1
    lib.orc_llg_default(C.byref(c.llg))
    for k, v in (llg_kw or {}).items():
        setattr(c.llg, k, v)
    lib.orc_run_steps(ss.p, C.byref(c), nsteps)


def nn_paths(nx, ny, nz, J=1.0, pbc=(1, 1, 1), dirs=6):
    """Pathways the canonical Lua setup loop adds with ex:add({i,j,k},{i±1,..},J):
    from = neighbour, to = site, periodic wrap per pbc, open edges dropped
    (spinoperationexchange.cpp:368-420)."""
    frm, to, Js = [], [], []
    offs = [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)][:dirs]
    dims = (nx, ny, nz)
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                for o in offs:
                    a = [i, j, k]
                    b = [i + o[0], j + o[1], k + o[2]]
                    ok = True
                    for d in range(3):
                        if pbc[d]:
                            a[d] %= dims[d]
                            b[d] %= dims[d]
                        if not (0 <= b[d] < dims[d]):
                            ok = False
                    if ok:
                        frm.append(a[0] + nx * (a[1] + ny * a[2]))
                        to.append(b[0] + nx * (b[1] + ny * b[2]))
                        Js.append(J)
    return np.array(frm, np.int32), np.array(to, np.int32), np.array(Js)
