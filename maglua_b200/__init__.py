"""maglua_b200 -- B200-native MagLua spin-dynamics step.

Python mirror of MagLua's Lua classes over the C ABI in include/mlb200.h
(libmlb200.so, sm_100a).  Class and method names follow the reference's Lua
API so scripts translate line by line:

    ss  = SpinSystem.new(32, 32, 1)
    ex  = Exchange.new(ss)
    ani = Anisotropy.new(ss)
    llg = LLG.new("Quaternion")
    ...
    ss.resetFields(); ex.apply(ss); ani.apply(ss); ss.sumFields(); llg.apply(ss)

Sites are 1-based {x, y, z} tuples as in Lua.  Everything runs on the GPU;
there is no CPU path: importing without the built library, or using it
without a CUDA device, raises.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmlb200.so")

MLB_OK = 0
_ERRNAMES = {-1: "EINVAL", -2: "ENOMEM", -3: "ECUDA", -4: "ESTATE", -5: "ENOTFOUND", -6: "ERANGE",
             -7: "EUNSUP"}


class MagLuaError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{_ERRNAMES.get(code, code)}: {msg}")
        self.code = code


_P = C.c_void_p
_D = C.POINTER(C.c_double)
_F = C.POINTER(C.c_float)
_I = C.POINTER(C.c_int)

_SIGS = {
    "mlb_last_error": ([], C.c_char_p),
    "mlb_version": ([], C.c_int),
    "mlb_init": ([C.c_int], C.c_int),
    "mlb_profile_begin": ([], C.c_int),
    "mlb_profile_end": ([C.c_int, C.c_char_p, _D, _I, _I], C.c_int),
    "mlb_philox4x32_10": ([C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)], C.c_int),
    "mlb_system_create": ([C.c_int, C.c_int, C.c_int, C.POINTER(_P)], C.c_int),
    "mlb_system_create_ex": ([C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(_P)], C.c_int),
    "mlb_system_real_bytes": ([_P, C.POINTER(C.c_int)], C.c_int),
    "mlb_system_destroy": ([_P], C.c_int),
    "mlb_system_dims": ([_P, _I], C.c_int),
    "mlb_system_set_stream": ([_P, _P], C.c_int),
    "mlb_system_get_stream": ([_P, C.POINTER(_P)], C.c_int),
    "mlb_system_synchronize": ([_P], C.c_int),
    "mlb_system_set_spin": ([_P, C.c_int, C.c_double, C.c_double, C.c_double], C.c_int),
    "mlb_system_get_spin": ([_P, C.c_int, _D], C.c_int),
    "mlb_system_set_spins": ([_P, _D, _D, _D, _D], C.c_int),
    "mlb_system_get_spins": ([_P, _D, _D, _D, _D], C.c_int),
    "mlb_system_upload_f32": ([_P, _P, _P, _P, _P], C.c_int),
    "mlb_system_download_f32": ([_P, _P, _P, _P], C.c_int),
    "mlb_system_set_param": ([_P, C.c_int, C.c_double], C.c_int),
    "mlb_system_get_param": ([_P, C.c_int, _D], C.c_int),
    "mlb_system_set_site_alpha": ([_P, _D], C.c_int),
    "mlb_system_set_site_gamma": ([_P, _D], C.c_int),
    "mlb_system_reset_fields": ([_P], C.c_int),
    "mlb_system_sum_fields": ([_P], C.c_int),
    "mlb_system_sum_fields_custom": ([_P, C.c_char_p, C.c_int, C.POINTER(C.c_char_p), _D], C.c_int),
    "mlb_system_get_field": ([_P, C.c_char_p, _D, _D, _D], C.c_int),
    "mlb_system_set_field": ([_P, C.c_char_p, _D, _D, _D], C.c_int),
    "mlb_system_slot_used": ([_P, C.c_char_p, _I], C.c_int),
    "mlb_system_set_slot_used": ([_P, C.c_char_p, C.c_int], C.c_int),
    "mlb_system_ensure_slot": ([_P, C.c_char_p], C.c_int),
    "mlb_system_netmoment": ([_P, C.c_double, _D], C.c_int),
    "mlb_system_field_dot": ([_P, C.c_char_p, _D], C.c_int),
    "mlb_system_copy": ([_P, _P, C.c_int], C.c_int),
    "mlb_op_create": ([C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(_P)], C.c_int),
    "mlb_op_destroy": ([_P], C.c_int),
    "mlb_op_kind": ([_P, _I], C.c_int),
    "mlb_op_set_scale": ([_P, C.c_double], C.c_int),
    "mlb_op_get_scale": ([_P, _D], C.c_int),
    "mlb_op_set_slot_name": ([_P, C.c_char_p], C.c_int),
    "mlb_op_get_slot_name": ([_P, C.c_char_p, C.c_size_t], C.c_int),
    "mlb_op_set_quirks": ([_P, C.c_int], C.c_int),
    "mlb_op_apply": ([_P, _P], C.c_int),
    "mlb_op_apply_many": ([_P, C.POINTER(_P), C.c_int], C.c_int),
    "mlb_exchange_add_path": ([_P, C.c_int, C.c_int, C.c_double], C.c_int),
    "mlb_exchange_add_paths": ([_P, _I, _I, _D, C.c_int], C.c_int),
    "mlb_exchange_set_normalize": ([_P, C.c_int], C.c_int),
    "mlb_exchange_num_paths": ([_P, _I], C.c_int),
    "mlb_anisotropy_add": ([_P, C.c_int, _D, C.c_double], C.c_int),
    "mlb_uniaxial_add": ([_P, C.c_int, _D, C.c_double, C.c_double], C.c_int),
    "mlb_cubic_add": ([_P, C.c_int, _D, _D, _D], C.c_int),
    "mlb_anisotropy_add_many": ([_P, C.c_int, _I, _D, _D], C.c_int),
    "mlb_uniaxial_add_many": ([_P, C.c_int, _I, _D, _D, _D], C.c_int),
    "mlb_cubic_add_many": ([_P, C.c_int, _I, _D, _D, _D], C.c_int),
    "mlb_thermal_set_temperature": ([_P, C.c_double], C.c_int),
    "mlb_thermal_get_temperature": ([_P, _D], C.c_int),
    "mlb_thermal_scale_site": ([_P, C.c_int, C.c_double], C.c_int),
    "mlb_thermal_set_seed": ([_P, C.c_uint64], C.c_int),
    "mlb_thermal_set_counter": ([_P, C.c_uint64], C.c_int),
    "mlb_thermal_inject": ([_P, _D, _D, _D], C.c_int),
    "mlb_appliedfield_set": ([_P, C.c_double, C.c_double, C.c_double], C.c_int),
    "mlb_appliedfield_get": ([_P, _D], C.c_int),
    "mlb_appliedfield_set_sweep": ([_P, C.c_double, C.c_double, C.c_double], C.c_int),
    "mlb_longrange_set_strength": ([_P, C.c_double], C.c_int),
    "mlb_longrange_get_strength": ([_P, _D], C.c_int),
    "mlb_longrange_get_truncation": ([_P, _I], C.c_int),
    "mlb_magnetostatic_set_cell_dimensions": ([_P, _D], C.c_int),
    "mlb_magnetostatic_get_cell_dimensions": ([_P, _D], C.c_int),
    "mlb_magnetostatic_set_crossover_tolerance": ([_P, C.c_double], C.c_int),
    "mlb_magnetostatic_get_crossover_tolerance": ([_P, _D], C.c_int),
    "mlb_op_encode": ([_P, C.c_int, C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t), _I], C.c_int),
    "mlb_op_decode": ([C.c_char_p, C.c_size_t, C.POINTER(_P), C.POINTER(C.c_size_t), _I], C.c_int),
    "mlb_llg_encode": ([_P, C.c_int, C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t), _I], C.c_int),
    "mlb_llg_decode": ([C.c_char_p, C.c_size_t, C.POINTER(_P), C.POINTER(C.c_size_t), _I], C.c_int),
    "mlb_exchange_set_pbc": ([_P, C.c_int, C.c_int, C.c_int], C.c_int),
    "mlb_llg_kind": ([_P, _I], C.c_int),
    "mlb_exchange_get_pbc": ([_P, _I], C.c_int),
    "mlb_dipole_set_huge_rings": ([_P, C.c_int], C.c_int),
    "mlb_longrange_set_truncation": ([_P, _I], C.c_int),
    "mlb_longrange_set_unit_cell": ([_P, _D], C.c_int),
    "mlb_longrange_set_open": ([_P, C.c_int, C.c_int, C.c_int], C.c_int),
    "mlb_longrange_set_matrix": ([_P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double], C.c_int),
    "mlb_longrange_get_matrix": ([_P, C.c_int, C.c_int, C.c_int, C.c_int, _D], C.c_int),
    "mlb_longrange_get_tensor": ([_P, _D * 6], C.c_int),
    "mlb_longrange3d_set_tensor": ([_P, C.c_int, _D], C.c_int),
    "mlb_longrange2d_set_tensor": ([_P, C.c_int, C.c_int, C.c_int, _D], C.c_int),
    "mlb_longrange2d_get_tensor": ([_P, C.c_int, C.c_int, C.c_int, _D], C.c_int),
    "mlb_longrange2d_set_layer_scales": ([_P, C.c_int, C.c_double, C.c_double], C.c_int),
    "mlb_longrange2d_get_layer_scales": ([_P, C.c_int, _D, _D], C.c_int),
    "mlb_longrange2d_set_required": ([_P, C.c_int, C.c_int], C.c_int),
    "mlb_longrange2d_get_required": ([_P, _I, _I], C.c_int),
    "mlb_dipole2d_set_unit_cell": ([_P, C.c_int, _D], C.c_int),
    "mlb_dipole2d_get_unit_cell": ([_P, C.c_int, _D], C.c_int),
    "mlb_dipole2d_set_offset": ([_P, C.c_int, _D], C.c_int),
    "mlb_dipole2d_get_offset": ([_P, C.c_int, _D], C.c_int),
    "mlb_dipole2d_set_truncation": ([_P, _I], C.c_int),
    "mlb_dipole2d_get_truncation": ([_P, _I], C.c_int),
    "mlb_dipole2d_make_data": ([_P], C.c_int),
    "mlb_magnetostatics2d_set_grain_size": ([_P, C.c_int, _D], C.c_int),
    "mlb_magnetostatics2d_get_grain_size": ([_P, C.c_int, _D], C.c_int),
    "mlb_lr2d_write_data_file": ([_P, C.c_char_p], C.c_int),
    "mlb_system_netmoment_async": ([_P, C.c_double, C.c_int], C.c_int),
    "mlb_ewald3d_create": ([C.c_int, C.c_int, C.c_int, C.POINTER(_P)], C.c_int),
    "mlb_ewald3d_destroy": ([_P], C.c_int),
    "mlb_ewald3d_set_unit_cell": ([_P, _D, _D, _D], C.c_int),
    "mlb_ewald3d_get_unit_cell": ([_P, _D], C.c_int),
    "mlb_ewald3d_set_lattice_size": ([_P, C.c_int, C.c_int, C.c_int], C.c_int),
    "mlb_ewald3d_get_lattice_size": ([_P, _I], C.c_int),
    "mlb_ewald3d_set_tau": ([_P, C.c_double], C.c_int),
    "mlb_ewald3d_get_tau": ([_P, _D], C.c_int),
    "mlb_ewald3d_set_nsites": ([_P, C.c_int], C.c_int),
    "mlb_ewald3d_get_nsites": ([_P, _I], C.c_int),
    "mlb_ewald3d_get_eta": ([_P, _D], C.c_int),
    "mlb_ewald3d_get_volume": ([_P, _D], C.c_int),
    "mlb_ewald3d_element": ([_P, C.c_int, _I, _D], C.c_int),
    "mlb_ewald3d_element_real": ([_P, C.c_int, _D, _D], C.c_int),
    "mlb_ewald3d_tensor": ([_P, _D], C.c_int),
    "mlb_system_netmoment_wait": ([_P, C.c_int, _D], C.c_int),
    "mlb_lr2d_read_data_file": ([_P, C.c_char_p, _I], C.c_int),
    "mlb_llg_create": ([C.c_int, C.POINTER(_P)], C.c_int),
    "mlb_llg_destroy": ([_P], C.c_int),
    "mlb_llg_set_flags": ([_P, C.c_int, C.c_int, C.c_double, C.c_double], C.c_int),
    "mlb_llg_apply": ([_P, _P, C.c_double, _P, _P, C.c_int], C.c_int),
    "mlb_run": ([_P, C.POINTER(_P), C.c_int, _P, C.c_int], C.c_int),
    "mlb_dipole_field_noalloc": ([_P, _P, _P, _P, _P, _P, _P, _P], C.c_int),
    "mlb_surrogate_create": ([_P, C.c_int, C.c_int, C.c_int, C.POINTER(_P)], C.c_int),
    "mlb_surrogate_destroy": ([_P], C.c_int),
    "mlb_surrogate_sizes": ([_P, _I], C.c_int),
    "mlb_surrogate_get_params": ([_P, _F, _F], C.c_int),
    "mlb_surrogate_set_params": ([_P, _F, _F], C.c_int),
    "mlb_surrogate_set_schedule": ([_P, C.c_int, C.c_double, C.c_double], C.c_int),
    "mlb_surrogate_train": ([_P, _P, C.POINTER(_P), C.c_int, _P, C.c_int, C.c_int, C.c_double, _D], C.c_int),
    "mlb_surrogate_validate": ([_P, _P, C.POINTER(_P), C.c_int, _P, C.c_int, C.c_int, _D], C.c_int),
    "mlb_surrogate_run": ([_P, _P, C.POINTER(_P), C.c_int, _P, C.c_int], C.c_int),
    "mlb_surrogate_attach": ([_P, _P], C.c_int),
    "mlb_surrogate_detach": ([_P], C.c_int),
    "mlb_surrogate_stats": ([_P, C.POINTER(C.c_longlong), _D], C.c_int),
    "mlb_surrogate_forward": ([_P, C.POINTER(_F), C.POINTER(_F)], C.c_int),
    "mlb_surrogate_gradients": ([_P, C.POINTER(_F), C.POINTER(_F), _F, _F, C.POINTER(_F), _D], C.c_int),
    "mlb_rk_create": ([_P, C.c_char_p, C.POINTER(_P), C.c_int, _P, _P, C.POINTER(_P)], C.c_int),
    "mlb_rk_step": ([_P, C.c_int], C.c_int),
    "mlb_rk_set_graph": ([_P, C.c_int], C.c_int),
    "mlb_rk_graph_steps": ([_P, C.POINTER(C.c_longlong)], C.c_int),
    "mlb_rk_step_on": ([_P, _P, C.c_int], C.c_int),
    "mlb_adapt_create": ([_P, _P, C.c_double, _P, _P, C.POINTER(_P)], C.c_int),
    "mlb_adapt_step": ([_P, _I], C.c_int),
    "mlb_adapt_destroy": ([_P], C.c_int),
    "mlb_system_diff": ([_P, _P, _D], C.c_int),
    "mlb_system_encode": ([_P, C.c_int, _P, C.c_size_t, C.POINTER(C.c_size_t), _I], C.c_int),
    "mlb_system_decode": ([_P, C.c_size_t, C.c_int, C.POINTER(_P), C.POINTER(C.c_size_t), _I], C.c_int),
    "mlb_dipole_write_wab": ([_P, C.c_char_p], C.c_int),
    "mlb_dipole_read_wab": ([_P, C.c_char_p], C.c_int),
    "mlb_rk_destroy": ([_P], C.c_int),
    "mlb_plan_create": ([_P, C.POINTER(_P), C.c_int, _P, C.c_int, C.POINTER(_P)], C.c_int),
    "mlb_plan_launch": ([_P, C.c_int], C.c_int),
    "mlb_plan_kernel_times": ([_P, C.c_int, C.c_char_p, _D, _I], C.c_int),
    "mlb_plan_device_times": ([_P, _D, _D], C.c_int),
    "mlb_plan_destroy": ([_P], C.c_int),
    "mlb_ensemble_create": ([C.c_int, _I, C.POINTER(_P)], C.c_int),
    "mlb_ensemble_destroy": ([_P], C.c_int),
    "mlb_ensemble_configure": ([_P, _P], C.c_int),
    "mlb_ensemble_set_spins": ([_P, C.c_int, _D, _D, _D], C.c_int),
    "mlb_ensemble_get_spins": ([_P, C.c_int, _D, _D, _D], C.c_int),
    "mlb_ensemble_run": ([_P, C.c_int], C.c_int),
    "mlb_ensemble_netmoment": ([_P, _D], C.c_int),
    "mlb_ensemble_info": ([_P, C.POINTER(C.c_longlong), _I, _D], C.c_int),
    "mlb_ensemble_get_stream": ([_P, C.POINTER(_P)], C.c_int),
    "mlb_surrogate_set_wait_limit": ([_P, C.c_uint], C.c_int),
    "mlb_ensemble_status": ([_P, C.c_int, C.POINTER(C.c_uint)], C.c_int),
    "mlb_system_status": ([_P, C.c_int, C.POINTER(C.c_uint)], C.c_int),
    "mlb_ensemble_set_replica_params": ([_P, C.c_int, C.c_double, _D, _D], C.c_int),
    "mlb_ensemble_get_replica_field": ([_P, C.c_int, _D], C.c_int),
    "mlb_ensemble_tune_log": ([_P, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)], C.c_int),
    "mlb_ensemble_config_info": ([_P, _I, _I, _I], C.c_int),
}
EXPORTED = tuple(_SIGS)


class _Lib:
    """libmlb200.so, loaded on first use.  A missing library raises: there
    is no fallback implementation."""

    def __init__(self):
        self._cdll = None

    def load(self):
        if self._cdll is None:
            if not os.path.exists(LIB_PATH):
                raise ImportError(f"{LIB_PATH} is missing: build it with "
                                  "`python -m maglua_b200.build` (nvcc, sm_100a)")
            lib = C.CDLL(LIB_PATH)
            for name, (args, res) in _SIGS.items():
                f = getattr(lib, name)
                f.argtypes = args
                f.restype = res
            self._cdll = lib
        return self._cdll

    def __getattr__(self, name):
        return getattr(self.load(), name)


_lib = _Lib()


def philox4x32_10(ctr, key):
    """Host evaluation of the Thermal noise generator (for checks)."""
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    _lib.mlb_philox4x32_10(c, k, o)
    return tuple(o)


def _ck(rc):
    if rc != MLB_OK:
        raise MagLuaError(rc, _lib.mlb_last_error().decode())


_initialised = [False]


def init(device=None):
    """Select the CUDA device (MagLua's -gpu N).  Called on first use."""
    if device is None:
        device = int(os.environ.get("LOCAL_RANK", "0"))
    _ck(_lib.mlb_init(device))
    _initialised[0] = True


def _ensure_init():
    if not _initialised[0]:
        init()


def _f64(a, n=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if n is not None and a.size != n:
        raise ValueError(f"expected {n} values, got {a.size}")
    return a


def _dp(a):
    return a.ctypes.data_as(_D) if a is not None else None


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _site3(site):
    s = list(site) if hasattr(site, "__len__") else [site]
    while len(s) < 3:
        s.append(1)
    return int(s[0]), int(s[1]), int(s[2])


# ====================================================================== SpinSystem
class SpinSystem:
    """SpinSystem (M/cpu/core/spinsystem.h:33-140) with its state on the GPU."""

    ALPHA, GAMMA, DT, TIME = 0, 1, 2, 3

    def __init__(self, nx, ny=1, nz=1, precision="f32"):
        """precision "f32" (default) or "f64": the width of the spins, fields
        and LLG arithmetic on the device."""
        _ensure_init()
        if isinstance(nx, SpinSystem):
            nx, ny, nz = nx.nx(), nx.ny(), nx.nz()
        elif hasattr(nx, "__len__"):
            nx, ny, nz = _site3(nx)
        rb = {"f32": 4, "f64": 8}.get(precision)
        if rb is None:
            raise MagLuaError(-1, "precision must be 'f32' or 'f64'")
        h = _P()
        _ck(_lib.mlb_system_create_ex(int(nx), int(ny), int(nz), rb, C.byref(h)))
        self._h = h
        self._dims = (int(nx), int(ny), int(nz))
        self._precision = precision

    new = classmethod(lambda cls, *a, **k: cls(*a, **k))

    def precision(self):
        return self._precision

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.mlb_system_destroy(h)
            self._h = None

    def close(self):
        self.__del__()

    # geometry
    def nx(self):
        return self._dims[0]

    def ny(self):
        return self._dims[1]

    def nz(self):
        return self._dims[2]

    def nxyz(self):
        return self._dims[0] * self._dims[1] * self._dims[2]

    def _idx(self, site):
        x, y, z = _site3(site)
        nx, ny, nz = self._dims
        # SpinSystem::getidx wraps periodically (spinsystem.cpp:1125-1142)
        x, y, z = (x - 1) % nx, (y - 1) % ny, (z - 1) % nz
        return x + nx * (y + ny * z)

    # streams
    def setStream(self, stream):
        _ck(_lib.mlb_system_set_stream(self._h, C.c_void_p(stream or 0)))

    def stream(self):
        out = _P()
        _ck(_lib.mlb_system_get_stream(self._h, C.byref(out)))
        return out.value or 0

    def synchronize(self):
        _ck(_lib.mlb_system_synchronize(self._h))

    # spins
    def status(self, clear=False):
        """Status word of the steps queued so far (synchronises the system's
        stream): bit 0 (1) when an LLG step wrote a non-finite spin."""
        f = C.c_uint()
        _ck(_lib.mlb_system_status(self._h, int(bool(clear)), C.byref(f)))
        return f.value

    def setSpin(self, site, spin, m=None):
        """l_setspin (spinsystem.cpp:1312-1361): optional length m."""
        sx, sy, sz = (list(spin) + [0, 0, 0])[:3]
        if m is not None:
            ln = abs(m)
            rr = sx * sx + sy * sy + sz * sz
            if rr > 0:
                rr = ln / np.sqrt(rr)
                sx, sy, sz = sx * rr, sy * rr, sz * rr
            else:
                sx, sy, sz = 0.0, 0.0, ln
        _ck(_lib.mlb_system_set_spin(self._h, self._idx(site), sx, sy, sz))

    def spin(self, site):
        out = np.zeros(4)
        _ck(_lib.mlb_system_get_spin(self._h, self._idx(site), _dp(out)))
        return tuple(out)

    def setSpinArrays(self, x, y, z, ms=None):
        n = self.nxyz()
        x, y, z = _f64(x, n), _f64(y, n), _f64(z, n)
        m = None if ms is None else _f64(ms, n)
        _ck(_lib.mlb_system_set_spins(self._h, _dp(x), _dp(y), _dp(z), _dp(m)))

    def spinArrays(self):
        n = self.nxyz()
        x, y, z, m = (np.zeros(n) for _ in range(4))
        _ck(_lib.mlb_system_get_spins(self._h, _dp(x), _dp(y), _dp(z), _dp(m)))
        return x, y, z, m

    def spinArrayX(self):
        return self.spinArrays()[0]

    def spinArrayY(self):
        return self.spinArrays()[1]

    def spinArrayZ(self):
        return self.spinArrays()[2]

    def spinArrayM(self):
        return self.spinArrays()[3]

    def uploadF32(self, x, y, z, ms=None):
        """Bulk FP32 upload from host buffers (pinned memory recommended)."""
        _ck(_lib.mlb_system_upload_f32(self._h, x.ctypes.data, y.ctypes.data, z.ctypes.data,
                                       ms.ctypes.data if ms is not None else None))

    def downloadF32(self, x, y, z):
        _ck(_lib.mlb_system_download_f32(self._h, x.ctypes.data, y.ctypes.data, z.ctypes.data))

    # scalars
    def _set(self, which, v):
        _ck(_lib.mlb_system_set_param(self._h, which, float(v)))

    def _get(self, which):
        v = C.c_double()
        _ck(_lib.mlb_system_get_param(self._h, which, C.byref(v)))
        return v.value

    def setAlpha(self, a):
        self._set(0, a)

    def alpha(self):
        return self._get(0)

    def setGamma(self, g):
        self._set(1, g)

    def gamma(self):
        return self._get(1)

    def setTimeStep(self, dt):
        self._set(2, dt)

    def timeStep(self):
        return self._get(2)

    def setTime(self, t):
        self._set(3, t)

    def time(self):
        return self._get(3)

    def setSiteAlphaArray(self, a):
        _ck(_lib.mlb_system_set_site_alpha(self._h, _dp(None if a is None else _f64(a, self.nxyz()))))

    def setSiteGammaArray(self, g):
        _ck(_lib.mlb_system_set_site_gamma(self._h, _dp(None if g is None else _f64(g, self.nxyz()))))

    # fields
    def resetFields(self):
        _ck(_lib.mlb_system_reset_fields(self._h))

    zeroFields = resetFields

    def sumFields(self, dest=None, srcs=None):
        """sumFields() / sumFields({names}) / sumFields(dest, {{w, name}, ...})."""
        if dest is None and srcs is None:
            _ck(_lib.mlb_system_sum_fields(self._h))
            return
        if isinstance(dest, (list, tuple)) and srcs is None:
            dest, srcs = "Total", dest
        names, w = [], []
        for s in srcs:
            if isinstance(s, (list, tuple)):
                w.append(float(s[0]))
                names.append(_slotname(s[1]))
            else:
                w.append(1.0)
                names.append(_slotname(s))
        arr = (C.c_char_p * len(names))(*[n.encode() for n in names])
        ww = _f64(w)
        _ck(_lib.mlb_system_sum_fields_custom(self._h, _slotname(dest).encode(), len(names), arr, _dp(ww)))

    def fieldArrays(self, name):
        n = self.nxyz()
        hx, hy, hz = np.zeros(n), np.zeros(n), np.zeros(n)
        _ck(_lib.mlb_system_get_field(self._h, _slotname(name).encode(), _dp(hx), _dp(hy), _dp(hz)))
        return hx, hy, hz

    def fieldArrayX(self, name):
        return self.fieldArrays(name)[0]

    def fieldArrayY(self, name):
        return self.fieldArrays(name)[1]

    def fieldArrayZ(self, name):
        return self.fieldArrays(name)[2]

    def field(self, name, site=None):
        if site is None and not isinstance(name, str):
            name, site = "Total", name
        hx, hy, hz = self.fieldArrays(name)
        i = self._idx(site)
        v = (hx[i], hy[i], hz[i])
        return v + (float(np.sqrt(sum(a * a for a in v))),)

    def setFieldArrays(self, name, hx=None, hy=None, hz=None):
        n = self.nxyz()
        a = [None if v is None else _f64(v, n) for v in (hx, hy, hz)]
        _ck(_lib.mlb_system_set_field(self._h, _slotname(name).encode(), *[_dp(v) for v in a]))

    def setFieldArrayX(self, name, v):
        self.setFieldArrays(name, hx=v)

    def setFieldArrayY(self, name, v):
        self.setFieldArrays(name, hy=v)

    def setFieldArrayZ(self, name, v):
        self.setFieldArrays(name, hz=v)

    def slotUsed(self, name):
        u = C.c_int()
        _ck(_lib.mlb_system_slot_used(self._h, _slotname(name).encode(), C.byref(u)))
        return bool(u.value)

    def setSlotUsed(self, name, b=True):
        _ck(_lib.mlb_system_set_slot_used(self._h, _slotname(name).encode(), int(bool(b))))

    def ensureSlotExists(self, name):
        _ck(_lib.mlb_system_ensure_slot(self._h, _slotname(name).encode()))

    # reductions
    def netMoment(self, m=1.0):
        out = np.zeros(8)
        _ck(_lib.mlb_system_netmoment(self._h, float(m), _dp(out)))
        return tuple(out)

    def netMomentAsync(self, slot, m=1.0):
        """Enqueue netMoment of the current spins into pinned slot 0..3
        without waiting; netMomentWait(slot) returns it."""
        _ck(_lib.mlb_system_netmoment_async(self._h, float(m), int(slot)))

    def netMomentWait(self, slot):
        out = np.zeros(8)
        _ck(_lib.mlb_system_netmoment_wait(self._h, int(slot), _dp(out)))
        return tuple(out)

    def fieldDot(self, name):
        out = C.c_double()
        _ck(_lib.mlb_system_field_dot(self._h, _slotname(name).encode(), C.byref(out)))
        return out.value

    # copies
    def copyTo(self, dst):
        _ck(_lib.mlb_system_copy(dst._h, self._h, 1))

    def copySpinsTo(self, dst):
        _ck(_lib.mlb_system_copy(dst._h, self._h, 0))

    def diff(self, other):
        """(dx, dy, dz, |d|) with d_c = sum_i |self_c,i - other_c,i| (l_getdiff)."""
        out = np.zeros(4)
        _ck(_lib.mlb_system_diff(self._h, other._h, _dp(out)))
        return tuple(out)

    def copy(self):
        c = SpinSystem(*self._dims, precision=self._precision)
        self.copyTo(c)
        return c

    def encode(self, first_index=0):
        """The bytes SpinSystem::encode writes (spinsystem.cpp:669-757) for
        this state, with the object header of an exported Lua value
        (luamigrate.cpp:265-275): what a checkpoint of the reference holds.
        first_index: the system's object index in the enclosing stream."""
        n = C.c_size_t()
        _ck(_lib.mlb_system_encode(self._h, int(first_index), None, 0, C.byref(n), None))
        buf = C.create_string_buffer(n.value)
        nobj = C.c_int()
        _ck(_lib.mlb_system_encode(self._h, int(first_index), buf, n.value, C.byref(n), C.byref(nobj)))
        self._stream_objects = nobj.value
        return buf.raw[:n.value]

    @classmethod
    def decode(cls, data, precision="f32", partial=False):
        """A new system from a stream written by encode or by the reference's
        SpinSystem::encode (decode, spinsystem.cpp:759-851).  partial=True:
        the stream may continue after the system; returns (system, bytes
        read, objects read)."""
        _ensure_init()
        rb = {"f32": 4, "f64": 8}.get(precision)
        if rb is None:
            raise MagLuaError(-1, "precision must be 'f32' or 'f64'")
        data = bytes(data)
        h = _P()
        used = C.c_size_t()
        nobj = C.c_int()
        _ck(_lib.mlb_system_decode(data, len(data), rb, C.byref(h), C.byref(used) if partial else None,
                                   C.byref(nobj)))
        obj = cls.__new__(cls)
        obj._h = h
        d = (C.c_int * 3)()
        _ck(_lib.mlb_system_dims(h, d))
        obj._dims = (d[0], d[1], d[2])
        obj._precision = precision
        return (obj, used.value, nobj.value) if partial else obj


def _slotname(x):
    if isinstance(x, str):
        return x
    if hasattr(x, "slotName"):
        return x.slotName()
    raise TypeError("expected a slot name or an operator")


# ====================================================================== operators
class SpinOperation:
    KIND = 0

    def __init__(self, *args):
        _ensure_init()
        if args and isinstance(args[0], SpinSystem):
            dims = args[0]._dims
            rest = args[1:]
        elif args and hasattr(args[0], "__len__"):
            dims = _site3(args[0])
            rest = args[1:]
        else:
            nums = [a for a in args if isinstance(a, (int, np.integer))][:3]
            dims = _site3(nums or [1])
            rest = args[len(nums):]
        self._dims = tuple(int(d) for d in dims)
        h = _P()
        _ck(_lib.mlb_op_create(self.KIND, *self._dims, C.byref(h)))
        self._h = h
        self._init_extra(rest)

    def _init_extra(self, rest):
        pass

    @classmethod
    def new(cls, *a):
        return cls(*a)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.mlb_op_destroy(h)
            self._h = None

    def nx(self):
        return self._dims[0]

    def ny(self):
        return self._dims[1]

    def nz(self):
        return self._dims[2]

    def _idx(self, site):
        x, y, z = _site3(site)
        return (x - 1) + self._dims[0] * ((y - 1) + self._dims[1] * (z - 1))

    def member(self, site):
        x, y, z = _site3(site)
        return 1 <= x <= self._dims[0] and 1 <= y <= self._dims[1] and 1 <= z <= self._dims[2]

    def apply(self, ss):
        if isinstance(ss, (list, tuple)):
            arr = (_P * len(ss))(*[s._h for s in ss])
            _ck(_lib.mlb_op_apply_many(self._h, arr, len(ss)))
        else:
            _ck(_lib.mlb_op_apply(self._h, ss._h))

    def setScale(self, s):
        _ck(_lib.mlb_op_set_scale(self._h, float(s)))

    def scale(self):
        v = C.c_double()
        _ck(_lib.mlb_op_get_scale(self._h, C.byref(v)))
        return v.value

    def setSlotName(self, name):
        _ck(_lib.mlb_op_set_slot_name(self._h, name.encode()))

    def slotName(self):
        buf = C.create_string_buffer(256)
        _ck(_lib.mlb_op_get_slot_name(self._h, buf, 256))
        return buf.value.decode()

    def setQuirks(self, on=True):
        """Reproduce (True, default) or fix the reference's arithmetic quirks."""
        _ck(_lib.mlb_op_set_quirks(self._h, int(bool(on))))

    def encode(self, first_index=0):
        """The bytes the reference's encode writes for this operator inside a
        checkpoint (mlb_op_encode)."""
        return _encode_stream(_lib.mlb_op_encode, self._h, first_index, self)


class Exchange(SpinOperation):
    """Exchange (M/cpu/exchange): pathways from -> to with strength J."""
    KIND = 1
    defaultMomentNormalization = None

    def _init_extra(self, rest):
        self._pbc = [1, 1, 1]
        if Exchange.defaultMomentNormalization is not None:
            self.normalizeMoments(bool(Exchange.defaultMomentNormalization))

    def setPeriodicXYZ(self, px=True, py=True, pz=True):
        self._pbc = [int(bool(px)), int(bool(py)), int(bool(pz))]
        _ck(_lib.mlb_exchange_set_pbc(self._h, *self._pbc))

    def periodicXYZ(self):
        return tuple(bool(p) for p in self._pbc)

    def add(self, a, b, J=1.0):
        """l_addpath (spinoperationexchange.cpp:368-420): wrap by pbc, drop outside."""
        a, b = list(_site3(a)), list(_site3(b))
        for i in range(3):
            a[i] -= 1
            b[i] -= 1
            n = self._dims[i]
            if self._pbc[i]:
                a[i] %= n
                b[i] %= n
            if not (0 <= a[i] < n and 0 <= b[i] < n):
                return
        nx, ny = self._dims[0], self._dims[1]
        s1 = a[0] + nx * (a[1] + ny * a[2])
        s2 = b[0] + nx * (b[1] + ny * b[2])
        _ck(_lib.mlb_exchange_add_path(self._h, s1, s2, float(J)))

    addPath = add

    def addPaths(self, frm, to, J):
        """Bulk add of 0-based site indices (already wrapped)."""
        f, t, j = _i32(frm), _i32(to), _f64(J)
        _ck(_lib.mlb_exchange_add_paths(self._h, f.ctypes.data_as(_I), t.ctypes.data_as(_I), _dp(j), len(f)))

    def normalizeMoments(self, b=None):
        if isinstance(b, bool):
            _ck(_lib.mlb_exchange_set_normalize(self._h, int(b)))
            self._norm = b
        return getattr(self, "_norm", True)

    def numberOfPaths(self):
        n = C.c_int()
        _ck(_lib.mlb_exchange_num_paths(self._h, C.byref(n)))
        return n.value


class Anisotropy(SpinOperation):
    """Anisotropy (M/cpu/anisotropy/spinoperationanisotropy.cpp)."""
    KIND = 2

    def add(self, site, axis, K):
        if not self.member(site):
            raise MagLuaError(-1, f"site {site} is not part of operator {self._dims}")
        _ck(_lib.mlb_anisotropy_add(self._h, self._idx(site), _dp(_f64(axis, 3)), float(K)))

    def addMany(self, sites, axes, K):
        s, a, k = _i32(sites), _f64(axes).reshape(-1), _f64(K)
        _ck(_lib.mlb_anisotropy_add_many(self._h, len(s), s.ctypes.data_as(_I), _dp(a), _dp(k)))


class AnisotropyUniaxial(SpinOperation):
    KIND = 3

    def add(self, site, axis, K1, K2=0.0):
        if not self.member(site):
            raise MagLuaError(-1, f"site {site} is not part of operator {self._dims}")
        _ck(_lib.mlb_uniaxial_add(self._h, self._idx(site), _dp(_f64(axis, 3)), float(K1), float(K2)))

    def addMany(self, sites, axes, K1, K2):
        s, a = _i32(sites), _f64(axes).reshape(-1)
        k1, k2 = _f64(K1), _f64(K2)
        _ck(_lib.mlb_uniaxial_add_many(self._h, len(s), s.ctypes.data_as(_I), _dp(a), _dp(k1), _dp(k2)))


class AnisotropyCubic(SpinOperation):
    KIND = 4

    def add(self, site, a1, a2, K1, K2=0.0, K3=0.0):
        if not self.member(site):
            raise MagLuaError(-1, f"site {site} is not part of operator {self._dims}")
        K = _f64([K1, K2, K3])
        _ck(_lib.mlb_cubic_add(self._h, self._idx(site), _dp(_f64(a1, 3)), _dp(_f64(a2, 3)), _dp(K)))

    def addMany(self, sites, a1, a2, K):
        s = _i32(sites)
        A1, A2, KK = _f64(a1).reshape(-1), _f64(a2).reshape(-1), _f64(K).reshape(-1)
        _ck(_lib.mlb_cubic_add_many(self._h, len(s), s.ctypes.data_as(_I), _dp(A1), _dp(A2), _dp(KK)))


Anisotropy.Uniaxial = AnisotropyUniaxial
Anisotropy.Cubic = AnisotropyCubic


class Random:
    """Random.* stand-ins.  Philox is the device generator the Thermal
    operator uses: a seed plus a counter, one draw of three normals per site
    and apply."""

    class Philox:
        def __init__(self, seed=0):
            self.seed = int(seed) & 0xFFFFFFFFFFFFFFFF

        @classmethod
        def new(cls, seed=0):
            return cls(seed)

        def setSeed(self, seed):
            self.seed = int(seed) & 0xFFFFFFFFFFFFFFFF


class Thermal(SpinOperation):
    """Thermal (M/cpu/thermal): Langevin field with counter-based noise."""
    KIND = 5

    def _init_extra(self, rest):
        self._rng = None
        for r in rest:
            if isinstance(r, Random.Philox):
                self._use_rng(r)

    def _use_rng(self, rng):
        self._rng = rng
        _ck(_lib.mlb_thermal_set_seed(self._h, rng.seed))

    def setTemperature(self, T):
        if T is None:
            raise MagLuaError(-1, "set temp cannot be nil")
        _ck(_lib.mlb_thermal_set_temperature(self._h, float(T)))

    set = setTemperature

    def temperature(self):
        v = C.c_double()
        _ck(_lib.mlb_thermal_get_temperature(self._h, C.byref(v)))
        return v.value

    get = temperature

    def scaleSite(self, site, v):
        x, y, z = _site3(site)
        if self.member((x, y, z)):
            _ck(_lib.mlb_thermal_scale_site(self._h, self._idx(site), float(v)))

    def setSeed(self, seed):
        _ck(_lib.mlb_thermal_set_seed(self._h, int(seed) & 0xFFFFFFFFFFFFFFFF))
        _ck(_lib.mlb_thermal_set_counter(self._h, 0))

    def setCounter(self, c):
        _ck(_lib.mlb_thermal_set_counter(self._h, int(c)))

    def inject(self, nx, ny, nz):
        """Use these normals (one per site and component) on the next apply."""
        n = self._dims[0] * self._dims[1] * self._dims[2]
        a = [_f64(v, n) for v in (nx, ny, nz)]
        _ck(_lib.mlb_thermal_inject(self._h, *[_dp(v) for v in a]))

    def apply(self, ss, rng=None):
        """Thermal:apply(ss[, rng]).  As in the reference (l_apply,
        spinoperationthermal.cpp:205-217) a given RNG is applied first and
        the operator's own RNG second, so the stored RNG decides the field;
        without a stored RNG that second apply fails with "Missing RNG"."""
        if rng is not None:
            _ck(_lib.mlb_thermal_set_seed(self._h, rng.seed))
            SpinOperation.apply(self, ss)
            if self._rng is None:
                raise MagLuaError(-4, "Missing RNG")
            _ck(_lib.mlb_thermal_set_seed(self._h, self._rng.seed))
        SpinOperation.apply(self, ss)


class AppliedField(SpinOperation):
    """AppliedField (M/cpu/appliedfield): uniform field in slot "Zeeman"."""
    KIND = 6

    def set(self, x=0.0, y=0.0, z=0.0):
        if isinstance(x, (list, tuple)):
            v = list(x) + [0, 0, 0]
            x, y, z = v[0], v[1], v[2]
        _ck(_lib.mlb_appliedfield_set(self._h, float(x or 0), float(y or 0), float(z or 0)))

    def get(self):
        out = np.zeros(3)
        _ck(_lib.mlb_appliedfield_get(self._h, _dp(out)))
        return tuple(out)

    def add(self, x=0.0, y=0.0, z=0.0):
        if isinstance(x, (list, tuple)):
            v = list(x) + [0, 0, 0]
            x, y, z = v[0], v[1], v[2]
        b = self.get()
        self.set(b[0] + x, b[1] + y, b[2] + z)

    def toTable(self):
        return list(self.get())

    def x(self):
        return self.get()[0]

    def y(self):
        return self.get()[1]

    def z(self):
        return self.get()[2]

    def setX(self, v):
        b = self.get()
        self.set(v, b[1], b[2])

    def setY(self, v):
        b = self.get()
        self.set(b[0], v, b[2])

    def setZ(self, v):
        b = self.get()
        self.set(b[0], b[1], v)

    def setSweep(self, dx=0.0, dy=0.0, dz=0.0):
        """Per-step field increment used by run()."""
        _ck(_lib.mlb_appliedfield_set_sweep(self._h, float(dx), float(dy), float(dz)))


_AB6 = {"XX": 0, "XY": 1, "XZ": 2, "YY": 3, "YZ": 4, "ZZ": 5}
_AB9 = {"XX": 0, "XY": 1, "XZ": 2, "YX": 3, "YY": 4, "YZ": 5, "ZX": 6, "ZY": 7, "ZZ": 8}


class LongRange(SpinOperation):
    """LongRange (M/cpu/longrange): user tensor, 2D FFT in-plane + layer sum."""
    KIND = 8

    def setStrength(self, g):
        _ck(_lib.mlb_longrange_set_strength(self._h, float(g)))

    def strength(self):
        v = C.c_double()
        _ck(_lib.mlb_longrange_get_strength(self._h, C.byref(v)))
        return v.value

    def setTruncation(self, r, x=None, y=None, z=None):
        if x is None:
            g = [-1] * 4 if r == float("inf") else [int(r)] * 4
        else:
            xs = [max(1, int(v)) for v in (x, y, z)]
            g = [max(xs)] + xs
        arr = (C.c_int * 4)(*g)
        _ck(_lib.mlb_longrange_set_truncation(self._h, arr))

    def truncation(self):
        """getTruncation: four values, math.huge (inf) for an infinite radius."""
        g = (C.c_int * 4)()
        _ck(_lib.mlb_longrange_get_truncation(self._h, g))
        return tuple(float("inf") if v == -1 else v for v in g)

    def setUnitCell(self, A, B, C_):
        abc = _f64(list(A) + list(B) + list(C_), 9)
        _ck(_lib.mlb_longrange_set_unit_cell(self._h, _dp(abc)))

    def setMatrix(self, ab, offset, value):
        ox, oy, oz = (list(offset) + [0, 0, 0])[:3]
        _ck(_lib.mlb_longrange_set_matrix(self._h, _AB6[ab.upper()], int(ox), int(oy), int(oz), float(value)))

    def getMatrix(self, ab, offset):
        ox, oy, oz = (list(offset) + [0, 0, 0])[:3]
        v = C.c_double()
        _ck(_lib.mlb_longrange_get_matrix(self._h, _AB6[ab.upper()], int(ox), int(oy), int(oz), C.byref(v)))
        return v.value

    def tensorArrays(self):
        """XX, XY, XZ, YY, YZ, ZZ shaped (2nz-1, ny, nx)."""
        nx, ny, nz = self._dims
        arrs = [np.zeros(nx * ny * (2 * nz - 1)) for _ in range(6)]
        ptrs = (_D * 6)(*[_dp(a) for a in arrs])
        _ck(_lib.mlb_longrange_get_tensor(self._h, ptrs))
        return [a.reshape(2 * nz - 1, ny, nx) for a in arrs]


def _wab_methods(cls):
    def writeWAB(self, filename):
        """Write the tensor as the reference's WAB_<nx>x<ny>.<v>.lua cache file."""
        _ck(_lib.mlb_dipole_write_wab(self._h, str(filename).encode()))

    def readWAB(self, filename):
        """Take the tensor from a WAB file whose parameters match this operator."""
        _ck(_lib.mlb_dipole_read_wab(self._h, str(filename).encode()))

    cls.writeWAB, cls.readWAB = writeWAB, readWAB
    return cls


LongRange = _wab_methods(LongRange)


class Dipole(LongRange):
    """Dipole (M/cpu/dipole): periodic-in-plane lattice-sum tensor."""
    KIND = 7

    def setHugeRings(self, rings):
        """Rings of 5 lattices summed for truncation math.huge (default 1000,
        the reference's count); a B200 extension for checks."""
        _ck(_lib.mlb_dipole_set_huge_rings(self._h, int(rings)))

    def setOpen(self, ox=True, oy=True, oz=True):
        """Open (zero-padded) boundaries in x and y instead of periodic images."""
        _ck(_lib.mlb_longrange_set_open(self._h, int(bool(ox)), int(bool(oy)), int(bool(oz))))


class Magnetostatic(LongRange):
    """Magnetostatic (M/cpu/magnetostatics): LongRange with the volume-averaged
    interaction of rectangular prisms (deprecated in the reference in favour
    of Magnetostatics2D; kept for its scripts)."""
    KIND = 13

    def setCellDimensions(self, dx, dy=None, dz=None):
        d = list(dx) if hasattr(dx, "__len__") else [dx, dy, dz]
        _ck(_lib.mlb_magnetostatic_set_cell_dimensions(self._h, _dp(_f64(d, 3))))

    def cellDimensions(self):
        d = np.zeros(3)
        _ck(_lib.mlb_magnetostatic_get_cell_dimensions(self._h, _dp(d)))
        return tuple(d)

    def setCrossoverTolerance(self, tol):
        _ck(_lib.mlb_magnetostatic_set_crossover_tolerance(self._h, float(tol)))

    def crossoverTolerance(self):
        v = C.c_double()
        _ck(_lib.mlb_magnetostatic_get_crossover_tolerance(self._h, C.byref(v)))
        return v.value


class LongRange3D(SpinOperation):
    """LongRange3D (M/cpu/longrange3d): 9-component cyclic 3D convolution."""
    KIND = 9

    def setStrength(self, g):
        _ck(_lib.mlb_longrange_set_strength(self._h, float(g)))

    def strength(self):
        v = C.c_double()
        _ck(_lib.mlb_longrange_get_strength(self._h, C.byref(v)))
        return v.value

    def setTensorArray(self, ab, arr):
        n = self._dims[0] * self._dims[1] * self._dims[2]
        a = _f64(arr, n)
        _ck(_lib.mlb_longrange3d_set_tensor(self._h, _AB9[ab.upper()], _dp(a)))


class LongRange2D(SpinOperation):
    """LongRange2D (M/cpu/longrange2d): in-plane periodic convolution with a
    9-component tensor array per (destination, source) layer pair, a
    source-moment scale per source layer and a destination-field scale per
    destination layer (spinoperationlongrange2d.cpp:430-530).  Layers are
    1-based, as in the Lua API.  New data is required at first: apply then
    calls the function given to setMakeDataFunction (fails without one);
    after setTensorArray, call setCompileRequired() so that apply
    re-transforms the arrays, as in the reference."""
    KIND = 10

    def _init_extra(self, rest):
        self._make = None

    def _layer(self, layer):
        layer = int(layer)
        if layer < 1 or layer > self._dims[2]:
            raise MagLuaError(-1, "Invalid Layer")
        return layer - 1

    def setTensorArray(self, dest, src, ab, arr):
        a = _f64(arr, self._dims[0] * self._dims[1])
        _ck(_lib.mlb_longrange2d_set_tensor(self._h, self._layer(dest), self._layer(src), _AB9[ab.upper()[:2]],
                                            _dp(a)))

    def tensorArray(self, dest, src, ab):
        """Copy of the (dest, src) array of component ab, shape (ny, nx)."""
        out = np.zeros(self._dims[0] * self._dims[1])
        _ck(_lib.mlb_longrange2d_get_tensor(self._h, self._layer(dest), self._layer(src), _AB9[ab.upper()[:2]],
                                            _dp(out)))
        return out.reshape(self._dims[1], self._dims[0])

    def getMatrix(self, dest, src, x, y, ab):
        """Element (x, y) (1-based) of the (dest, src) array of component ab
        (longrange2d_luafuncs.lua:6-9)."""
        return float(self.tensorArray(dest, src, ab)[int(y) - 1, int(x) - 1])

    def _scales(self, layer):
        a, b = C.c_double(), C.c_double()
        _ck(_lib.mlb_longrange2d_get_layer_scales(self._h, self._layer(layer), C.byref(a), C.byref(b)))
        return a.value, b.value

    def setSourceMomentScale(self, layer, v):
        _, d = self._scales(layer)
        _ck(_lib.mlb_longrange2d_set_layer_scales(self._h, self._layer(layer), float(v), d))

    def sourceMomentScale(self, layer):
        return self._scales(layer)[0]

    def setDestinationFieldScale(self, layer, v):
        sm, _ = self._scales(layer)
        _ck(_lib.mlb_longrange2d_set_layer_scales(self._h, self._layer(layer), sm, float(v)))

    def destinationFieldScale(self, layer):
        return self._scales(layer)[1]

    def setStrength(self, *a):
        raise MagLuaError(-1, "setStrength is depreciated. Please use setSourceMomentScale and setDestinationFieldScale.")

    def strength(self, *a):
        raise MagLuaError(-1, "strength is depreciated. Please use sourceMomentScale and sestinationFieldScale.")

    def setNewDataRequired(self, on=True):
        _ck(_lib.mlb_longrange2d_set_required(self._h, int(bool(on)), -1))

    def setCompileRequired(self, on=True):
        _ck(_lib.mlb_longrange2d_set_required(self._h, -1, int(bool(on))))

    def _required(self):
        a, b = C.c_int(), C.c_int()
        _ck(_lib.mlb_longrange2d_get_required(self._h, C.byref(a), C.byref(b)))
        return bool(a.value), bool(b.value)

    def newDataRequired(self):
        return self._required()[0]

    def compileRequired(self):
        return self._required()[1]

    def setMakeDataFunction(self, fn):
        """fn(op) fills the tensor arrays when new data is required
        (spinoperationlongrange2d.cpp:366-385)."""
        if not callable(fn):
            raise MagLuaError(-1, "function required as argument")
        self._make = fn

    def makeData(self):
        if self.newDataRequired():
            self._make_now()

    def _make_now(self):
        if self._make is None:
            raise MagLuaError(-4, "make data function not set")
        self.setNewDataRequired(False)
        self._make(self)
        self.setCompileRequired(True)

    def apply(self, ss):
        if self._make is not None and self.newDataRequired():
            self._make_now()
        super().apply(ss)


class Dipole2D(LongRange2D):
    """Dipole2D (M/cpu/dipole2d): LongRange2D whose arrays come from the
    point-dipole builder of dip2d_luafuncs.lua:540-660 (unit cell and offset
    per layer, truncation), run natively on the first apply."""
    KIND = 11

    def setUnitCell(self, layer, A, B=None, Cv=None):
        if B is None:
            A, B, Cv = A[0], A[1], A[2]
        abc = np.asarray([*A, *B, *Cv], dtype=np.float64)
        _ck(_lib.mlb_dipole2d_set_unit_cell(self._h, self._layer(layer), _dp(abc)))

    def unitCell(self, layer):
        out = np.zeros(9)
        _ck(_lib.mlb_dipole2d_get_unit_cell(self._h, self._layer(layer), _dp(out)))
        return list(out[0:3]), list(out[3:6]), list(out[6:9])

    def setOffset(self, layer, v):
        a = np.asarray(v, dtype=np.float64)
        _ck(_lib.mlb_dipole2d_set_offset(self._h, self._layer(layer), _dp(a)))

    def offset(self, layer=None):
        if layer is None:
            return [self.offset(z + 1) for z in range(self._dims[2])]
        out = np.zeros(3)
        _ck(_lib.mlb_dipole2d_get_offset(self._h, self._layer(layer), _dp(out)))
        return list(out)

    def truncation(self):
        t = (C.c_int * 4)()
        _ck(_lib.mlb_dipole2d_get_truncation(self._h, t))
        return tuple(t)

    def setTruncation(self, trunc=None, tx=None, ty=None, tz=None):
        cur = list(self.truncation())
        for i, v in enumerate((trunc, tx, ty, tz)):
            if v is not None:
                cur[i] = int(v)
        _ck(_lib.mlb_dipole2d_set_truncation(self._h, (C.c_int * 4)(*cur)))

    def _make_now(self):
        if self._make is not None:
            return super()._make_now()
        _ck(_lib.mlb_dipole2d_make_data(self._h))

    def writeDataFile(self, filename):
        """Write the reference's tensor data file (GAB_... for Dipole2D,
        MAB_... for Magnetostatics2D; dip2d_luafuncs.lua:278-500)."""
        _ck(_lib.mlb_lr2d_write_data_file(self._h, os.fsencode(filename)))

    def readDataFile(self, filename):
        """Load the arrays of a tensor data file when its size and builder
        state match this operator's; returns whether it did."""
        ok = C.c_int()
        _ck(_lib.mlb_lr2d_read_data_file(self._h, os.fsencode(filename), C.byref(ok)))
        return bool(ok.value)

    def makeData(self):
        if self.newDataRequired():
            self._make_now()

    def apply(self, ss):
        if self.newDataRequired():
            self._make_now()
        SpinOperation.apply(self, ss)


class Magnetostatics2D(Dipole2D):
    """Magnetostatics2D (M/cpu/magnetostatics2d): LongRange2D whose arrays
    are minus the demagnetising tensors of prism-shaped grains (Newell's f
    and g), summed over the in-plane images within the truncations
    (mag2d_luafuncs.lua:598-744), built natively on the first apply.  The
    user applies the 1/V source scale and 4 pi destination scale."""
    KIND = 12

    def setOffset(self, layer, v):
        raise MagLuaError(-1, "Magnetostatics2D has no per-layer offset")

    def setGrainSize(self, layer, X, Y=None, Z=None):
        if Y is None:
            X, Y, Z = X
        g = np.asarray([X, Y, Z], dtype=np.float64)
        _ck(_lib.mlb_magnetostatics2d_set_grain_size(self._h, self._layer(layer), _dp(g)))

    def grainSize(self, layer):
        """x, y, z and the volume (mag2d_luafuncs.lua:109-122)."""
        g = np.zeros(3)
        _ck(_lib.mlb_magnetostatics2d_get_grain_size(self._h, self._layer(layer), _dp(g)))
        return float(g[0]), float(g[1]), float(g[2]), float(g[0] * g[1] * g[2])

    def getMatrix(self, dest, src, ab, x, y):
        """Element at 0-based offsets (x, y) of the (dest, src) array of
        component ab, data made first if needed (mag2d_luafuncs.lua:32-45)."""
        self.makeData()
        return float(self.tensorArray(dest, src, ab)[int(y), int(x)])

    def setMatrix(self, dest, src, ab, x, y, v):
        """mag2d_luafuncs.lua:47-62: set one element, compile required."""
        self.makeData()
        a = self.tensorArray(dest, src, ab)
        a[int(y), int(x)] = float(v)
        self.setTensorArray(dest, src, ab, a.reshape(-1))
        self.setCompileRequired(True)


class DipoleEwald3D:
    """DipoleEwald3D (M/cpu/ewald3d): the dipolar tensor G_ab(r) of a
    periodic nx x ny x nz lattice by Ewald summation in FP64, element by
    element on the host or every element of the lattice on the GPU
    (tensorArrays).  make_tensor.lua stores -G into LongRange3D."""

    def __init__(self, *args):
        dims = self._dims_of(args)
        h = _P()
        _ck(_lib.mlb_ewald3d_create(int(dims[0]), int(dims[1]), int(dims[2]), C.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.mlb_ewald3d_destroy(h)
            self._h = None

    @classmethod
    def new(cls, *a):
        return cls(*a)

    @staticmethod
    def _dims_of(args):
        if args and isinstance(args[0], SpinSystem):
            return (args[0].nx(), args[0].ny(), args[0].nz())
        if args and hasattr(args[0], "__len__"):
            return (tuple(int(v) for v in args[0]) + (1, 1, 1))[:3]
        return (tuple(int(a) for a in args) + (1, 1, 1))[:3]

    def setUnitCell(self, a, b, c):
        va, vb, vc = (np.asarray(v, dtype=np.float64) for v in (a, b, c))
        _ck(_lib.mlb_ewald3d_set_unit_cell(self._h, _dp(va), _dp(vb), _dp(vc)))

    def unitCell(self):
        out = np.zeros(9)
        _ck(_lib.mlb_ewald3d_get_unit_cell(self._h, _dp(out)))
        return list(out[0:3]), list(out[3:6]), list(out[6:9])

    def latticeSize(self):
        n = (C.c_int * 3)()
        _ck(_lib.mlb_ewald3d_get_lattice_size(self._h, n))
        return tuple(n)

    def setLatticeSize(self, *args):
        dims = self._dims_of(args)
        _ck(_lib.mlb_ewald3d_set_lattice_size(self._h, int(dims[0]), int(dims[1]), int(dims[2])))

    def volume(self):
        v = C.c_double()
        _ck(_lib.mlb_ewald3d_get_volume(self._h, C.byref(v)))
        return v.value

    def tau(self):
        v = C.c_double()
        _ck(_lib.mlb_ewald3d_get_tau(self._h, C.byref(v)))
        return v.value

    def setTau(self, t):
        _ck(_lib.mlb_ewald3d_set_tau(self._h, float(t)))

    def NSites(self):
        v = C.c_int()
        _ck(_lib.mlb_ewald3d_get_nsites(self._h, C.byref(v)))
        return v.value

    def setNSites(self, n):
        _ck(_lib.mlb_ewald3d_set_nsites(self._h, int(n)))

    def eta(self):
        v = C.c_double()
        _ck(_lib.mlb_ewald3d_get_eta(self._h, C.byref(v)))
        return v.value

    @staticmethod
    def _ab(AB):
        ab = str(AB).upper()[:2]
        if len(ab) < 2 or ab not in _AB9:
            raise MagLuaError(-1, "first argument of calculateTensorElement must be AB pair: `XX', `XY', ... `ZZ'")
        return _AB9[ab]

    def calculateTensorElement(self, AB, xyz):
        r = (C.c_int * 3)(*[int(v) for v in xyz])
        out = C.c_double()
        _ck(_lib.mlb_ewald3d_element(self._h, self._ab(AB), r, C.byref(out)))
        return out.value

    def calculateTensorElementRealR(self, AB, r):
        rr = np.asarray(r, dtype=np.float64)
        out = C.c_double()
        _ck(_lib.mlb_ewald3d_element_real(self._h, self._ab(AB), _dp(rr), C.byref(out)))
        return out.value

    def tensorArrays(self):
        """Every element of the lattice computed on the GPU: {AB: array
        (nz, ny, nx)} with the values calculateTensorElement returns."""
        nx, ny, nz = self.latticeSize()
        out = np.zeros(9 * nx * ny * nz)
        _ck(_lib.mlb_ewald3d_tensor(self._h, _dp(out)))
        out = out.reshape(9, nz, ny, nx)
        return {ab: out[k] for ab, k in _AB9.items()}


# ====================================================================== LLG
class _LLGBase:
    KIND = 0
    thermalOnlyFirstTerm = None

    def __init__(self):
        _ensure_init()
        h = _P()
        _ck(_lib.mlb_llg_create(self.KIND, C.byref(h)))
        self._h = h
        self._flags = [1, 0, 1.0, 1.0]
        if LLG.thermalOnlyFirstTerm is not None:
            self.setThermalOnlyFirstTerm(bool(LLG.thermalOnlyFirstTerm))

    @classmethod
    def new(cls):
        return cls()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.mlb_llg_destroy(h)
            self._h = None

    def _push(self):
        f = self._flags
        _ck(_lib.mlb_llg_set_flags(self._h, int(f[0]), int(f[1]), float(f[2]), float(f[3])))

    def setThermalOnlyFirstTerm(self, b):
        self._flags[0] = int(bool(b))
        self._push()

    def thermalOnlyFirstTerm(self):
        return bool(self._flags[0])

    def setDisableRenormalization(self, b):
        self._flags[1] = int(bool(b))
        self._push()

    def disableRenormalization(self):
        return bool(self._flags[1])

    def setUnphysicalPrecessionScale(self, v):
        self._flags[2] = float(v)
        self._push()

    def setUnphysicalDampingScale(self, v):
        self._flags[3] = float(v)
        self._push()

    def apply(self, *args):
        """apply(A[, x], B, C[, advance]) as l_apply (llg.cpp:91-171)."""
        args = list(args)
        advance = True
        if args and isinstance(args[-1], bool):
            advance = args.pop()
        frm = args[0]
        scale = 1.0
        rest = args[1:]
        if rest and isinstance(rest[0], (int, float)) and not isinstance(rest[0], bool):
            scale = float(rest[0])
            rest = rest[1:]
        dmdt = rest[0] if len(rest) > 0 and rest[0] is not None else frm
        to = rest[1] if len(rest) > 1 and rest[1] is not None else frm
        if isinstance(frm, (list, tuple)):
            d = dmdt if isinstance(dmdt, (list, tuple)) else [dmdt] * len(frm)
            t = to if isinstance(to, (list, tuple)) else [to] * len(frm)
            if not (len(frm) == len(d) == len(t)):
                raise MagLuaError(-1, "Size mismatch in number of SpinSystems given in each table")
            for a, b, c in zip(frm, d, t):
                _ck(_lib.mlb_llg_apply(self._h, a._h, scale, b._h, c._h, int(advance)))
            return
        _ck(_lib.mlb_llg_apply(self._h, frm._h, scale, dmdt._h, to._h, int(advance)))


def _encode_stream(fn, h, first_index, owner):
    n = C.c_size_t()
    _ck(fn(h, int(first_index), None, 0, C.byref(n), None))
    buf = C.create_string_buffer(n.value)
    nobj = C.c_int()
    _ck(fn(h, int(first_index), buf, n.value, C.byref(n), C.byref(nobj)))
    owner._stream_objects = nobj.value
    return buf.raw[:n.value]


def _encode_llg(self, first_index=0):
    """The bytes LLG::encode writes inside a checkpoint (mlb_llg_encode)."""
    return _encode_stream(_lib.mlb_llg_encode, self._h, first_index, self)


_LLGBase.encode = _encode_llg


def decode(data, partial=False):
    """An operator or LLG object from a stream written by encode or by the
    reference (Exchange, Anisotropy, Anisotropy.Uniaxial, Anisotropy.Cubic,
    Thermal, AppliedField, Dipole, LLG.Cartesian, LLG.Quaternion).
    partial=True: the stream may continue; returns (object, bytes read,
    objects read)."""
    _ensure_init()
    data = bytes(data)
    h = _P()
    used = C.c_size_t()
    nobj = C.c_int()
    kinds = {1: Exchange, 2: Anisotropy, 3: AnisotropyUniaxial, 4: AnisotropyCubic, 5: Thermal, 6: AppliedField,
             7: Dipole}
    rc = _lib.mlb_op_decode(data, len(data), C.byref(h), C.byref(used) if partial else None, C.byref(nobj))
    if rc == MLB_OK:
        k = C.c_int()
        _ck(_lib.mlb_op_kind(h, C.byref(k)))
        cls = kinds[k.value]
        obj = cls.__new__(cls)
        obj._h = h
        obj._dims = _op_dims_from_stream(data)
        if cls is Exchange:
            p = (C.c_int * 3)()
            _ck(_lib.mlb_exchange_get_pbc(h, p))
            obj._pbc = list(p)
        if cls is Thermal:
            obj._rng = None
    else:
        rc2 = _lib.mlb_llg_decode(data, len(data), C.byref(h), C.byref(used) if partial else None, C.byref(nobj))
        if rc2 != MLB_OK:
            _ck(rc)
        k = C.c_int()
        _ck(_lib.mlb_llg_kind(h, C.byref(k)))
        cls = LLGQuaternion if k.value == 1 else LLGCartesian
        obj = cls.__new__(cls)
        obj._h = h
        obj._flags = _llg_flags_from_stream(data)
    return (obj, used.value, nobj.value) if partial else obj


def _op_dims_from_stream(data):
    # LUA_TUSERDATA, type, char 111, index, char version, nx, ny, nz
    o = 4 + 4 + 1 + 4 + 1
    return tuple(int.from_bytes(data[o + 4 * i:o + 4 * i + 4], "little", signed=True) for i in range(3))


def _llg_flags_from_stream(data):
    import struct
    o = 4 + 4 + 1 + 4
    v = data[o]
    tof, dis = struct.unpack_from("<ii", data, o + 1)
    pre, dmp = struct.unpack_from("<dd", data, o + 9) if v == 1 else (1.0, 1.0)
    return [tof, dis, pre, dmp]


class LLGCartesian(_LLGBase):
    KIND = 0


class LLGQuaternion(_LLGBase):
    KIND = 1


class LLG:
    """LLG.new("Cartesian"|"Quaternion") (llg_wrapper.lua)."""
    Cartesian = LLGCartesian
    Quaternion = LLGQuaternion
    thermalOnlyFirstTerm = None

    @staticmethod
    def new(kind):
        if kind not in ("Cartesian", "Quaternion"):
            raise MagLuaError(-1, f"Failed to find LLG implementation of type `{kind}'")
        return getattr(LLG, kind)()


class profile:
    """with profile() as prof: ... -> prof.kernels = {name: (total_ms, launches)}"""

    def __enter__(self):
        _ck(_lib.mlb_profile_begin())
        self.kernels = {}
        return self

    def __exit__(self, *exc):
        cap = 64
        names = C.create_string_buffer(48 * cap)
        ms = np.zeros(cap)
        nl = np.zeros(cap, dtype=np.int32)
        cnt = C.c_int()
        _ck(_lib.mlb_profile_end(cap, names, _dp(ms), nl.ctypes.data_as(_I), C.byref(cnt)))
        raw = names.raw
        for k in range(cnt.value):
            nm = raw[48 * k:48 * (k + 1)].split(b"\0", 1)[0].decode()
            self.kernels[nm] = (float(ms[k]), int(nl[k]))
        return False


class Plan:
    """The canonical step of ss (resetFields; op.apply for op in ops;
    sumFields; llg.apply) captured as CUDA graphs; launch(n) runs n steps with
    one graph launch each.  timing=True (or 1) adds event nodes around every
    kernel (kernelTimes() -> {name: ms} of the last launched step); timing=2
    keeps the step's dependent launches and records a device timeline of the
    fused (y,z) and x passes (deviceTimes())."""

    def __init__(self, ss, ops, llg, timing=False):
        self._keep = (ss, list(ops), llg)
        arr = (_P * len(ops))(*[o._h for o in ops])
        h = _P()
        mode = 2 if timing == 2 else int(bool(timing))
        _ck(_lib.mlb_plan_create(ss._h, arr, len(ops), llg._h, mode, C.byref(h)))
        self._h = h

    def launch(self, nsteps=1):
        _ck(_lib.mlb_plan_launch(self._h, int(nsteps)))

    def kernelTimes(self):
        cap = 32
        names = C.create_string_buffer(48 * cap)
        ms = np.zeros(cap)
        cnt = C.c_int()
        _ck(_lib.mlb_plan_kernel_times(self._h, cap, names, _dp(ms), C.byref(cnt)))
        out = {}
        raw = names.raw
        for k in range(cnt.value):
            nm = raw[48 * k:48 * (k + 1)].split(b"\0", 1)[0].decode()
            out[nm] = out.get(nm, 0.0) + float(ms[k])
        return out

    def deviceTimes(self):
        """{"k_conv_yz": us, "k_xstep": us} over the steps launched since the
        last call (timing=2 plans): each pass from its first CTA released from
        the dependency wait to its last CTA's end; passes that did not run are
        left out."""
        a, b = C.c_double(), C.c_double()
        _ck(_lib.mlb_plan_device_times(self._h, C.byref(a), C.byref(b)))
        out = {}
        if a.value >= 0:
            out["k_conv_yz"] = a.value
        if b.value >= 0:
            out["k_xstep"] = b.value
        return out

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.mlb_plan_destroy(h)
            self._h = None

    close = __del__


class _EnsCfg(C.Structure):
    _fields_ = [("alpha", C.c_double), ("gamma", C.c_double), ("dt", C.c_double), ("J", C.c_double),
                ("pbc", C.c_int * 3), ("K", C.c_double), ("axis", C.c_double * 3), ("T", C.c_double),
                ("seed", C.c_uint64), ("B", C.c_double * 3), ("dB", C.c_double * 3), ("g", C.c_double),
                ("open_xy", C.c_int), ("llg", C.c_int)]


class Ensemble:
    """Replicas of uneven sizes stepped together: packed by size class, one
    launch per phase, graph-captured (the batched op:apply({ss1, ...}) form
    for systems that share one operator set)."""

    def __init__(self, dims):
        _ensure_init()
        d = np.ascontiguousarray(np.asarray(dims, dtype=np.int32).reshape(-1, 3))
        self.dims = [tuple(int(v) for v in row) for row in d]
        h = _P()
        _ck(_lib.mlb_ensemble_create(len(d), d.ctypes.data_as(_I), C.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.mlb_ensemble_destroy(h)
            self._h = None

    def configure(self, alpha=0.1, dt=0.01, gamma=1.0, J=1.0, pbc=(0, 0, 0), K=0.0, axis=(0, 0, 1), T=0.0,
                  seed=0, B=(0, 0, 0), dB=(0, 0, 0), g=0.0, open_xy=True, llg="Cartesian"):
        c = _EnsCfg()
        c.alpha, c.gamma, c.dt, c.J, c.K, c.T, c.g = alpha, gamma, dt, J, K, T, g
        for i in range(3):
            c.pbc[i] = int(bool(pbc[i]))
            c.axis[i] = axis[i]
            c.B[i] = B[i]
            c.dB[i] = dB[i]
        c.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
        c.open_xy = int(bool(open_xy))
        c.llg = 0 if llg == "Cartesian" else 1
        _ck(_lib.mlb_ensemble_configure(self._h, C.byref(c)))

    def setSpins(self, rep, x, y, z):
        n = int(np.prod(self.dims[rep]))
        x, y, z = _f64(x, n), _f64(y, n), _f64(z, n)
        _ck(_lib.mlb_ensemble_set_spins(self._h, int(rep), _dp(x), _dp(y), _dp(z)))

    def spins(self, rep):
        n = int(np.prod(self.dims[rep]))
        x, y, z = np.zeros(n), np.zeros(n), np.zeros(n)
        _ck(_lib.mlb_ensemble_get_spins(self._h, int(rep), _dp(x), _dp(y), _dp(z)))
        return x, y, z

    def run(self, nsteps):
        _ck(_lib.mlb_ensemble_run(self._h, int(nsteps)))

    def netMoment(self):
        out = np.zeros((len(self.dims), 8))
        _ck(_lib.mlb_ensemble_netmoment(self._h, _dp(out)))
        return out

    def info(self):
        n, bs, t = C.c_longlong(), C.c_int(), C.c_double()
        _ck(_lib.mlb_ensemble_info(self._h, C.byref(n), C.byref(bs), C.byref(t)))
        return {"sites": n.value, "block_size": bs.value, "time": t.value}

    def stream(self):
        out = _P()
        _ck(_lib.mlb_ensemble_get_stream(self._h, C.byref(out)))
        return out.value or 0

    def status(self, clear=False):
        """Status word of the steps run so far (bit 0: a non-finite spin)."""
        f = C.c_uint()
        _ck(_lib.mlb_ensemble_status(self._h, int(bool(clear)), C.byref(f)))
        return f.value

    def setReplicaParams(self, rep, T, B=(0, 0, 0), dB=(0, 0, 0)):
        """Temperature and applied field (start, per-step sweep) of one replica."""
        _ck(_lib.mlb_ensemble_set_replica_params(self._h, int(rep), float(T), _dp(_f64(B, 3)), _dp(_f64(dB, 3))))

    def replicaField(self, rep):
        out = np.zeros(3)
        _ck(_lib.mlb_ensemble_get_replica_field(self._h, int(rep), _dp(out)))
        return tuple(out)

    def tuneLog(self):
        n = C.c_size_t()
        _ck(_lib.mlb_ensemble_tune_log(self._h, None, 0, C.byref(n)))
        buf = C.create_string_buffer(n.value)
        _ck(_lib.mlb_ensemble_tune_log(self._h, buf, n.value, C.byref(n)))
        return buf.value.decode()

    def configInfo(self):
        g, nc, gc = C.c_int(), C.c_int(), C.c_int()
        _ck(_lib.mlb_ensemble_config_info(self._h, C.byref(g), C.byref(nc), C.byref(gc)))
        return {"grid": g.value, "classes": nc.value, "generic_classes": gc.value}


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _fptrs(arrs):
    return (_F * 3)(*[a.ctypes.data_as(_F) for a in arrs])


class Surrogate:
    """Learned dipolar surrogate bound to a Dipole or LongRange operator (a
    B200 extension without a reference counterpart): a linear spectral-conv
    network predicting the field change from the spin change since the last
    exact evaluation, BF16 on the tensor cores."""

    def __init__(self, op, modes=(16, 16), radius=2):
        _ensure_init()
        h = _P()
        _ck(_lib.mlb_surrogate_create(op._h, int(modes[0]), int(modes[1]), int(radius), C.byref(h)))
        self._h = h
        self._op = op
        self.dims = tuple(op._dims)
        out = (C.c_int * 7)()
        _ck(_lib.mlb_surrogate_sizes(h, out))
        self.C, self.CP, self.mx, self.my, self.radius, self.nw, self.nr = list(out)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.mlb_surrogate_destroy(h)
            self._h = None

    def params(self):
        w = np.zeros(self.nw, np.float32)
        r = np.zeros(self.nr, np.float32)
        _ck(_lib.mlb_surrogate_get_params(self._h, w.ctypes.data_as(_F), r.ctypes.data_as(_F)))
        dia = 2 * self.radius + 1
        W = w.reshape(dia * dia, self.C, self.C).astype(np.float64)
        R = r.reshape(self.mx, self.my, self.C, self.C, 2).astype(np.float64)
        return W, R[..., 0] + 1j * R[..., 1]

    def setParams(self, W, R):
        w = _f32(np.asarray(W).reshape(-1))
        Rc = np.asarray(R)
        r = _f32(np.stack([Rc.real, Rc.imag], axis=-1).reshape(-1))
        _ck(_lib.mlb_surrogate_set_params(self._h, w.ctypes.data_as(_F), r.ctypes.data_as(_F)))

    def setSchedule(self, k, tol=1e-3, eps=0.0):
        _ck(_lib.mlb_surrogate_set_schedule(self._h, int(k), float(tol), float(eps)))

    def setWaitLimit(self, polls):
        """Polls of each tensor-core completion wait before it gives up and
        sets the error flag (default 2**24; 0 exercises the failure path)."""
        _ck(_lib.mlb_surrogate_set_wait_limit(self._h, int(polls)))

    def forward(self, x):
        xs = [_f32(x[c]) for c in range(3)]
        out = [np.zeros_like(xs[0]) for _ in range(3)]
        _ck(_lib.mlb_surrogate_forward(self._h, _fptrs(xs), _fptrs(out)))
        return np.stack(out)

    def gradients(self, x, t):
        xs = [_f32(x[c]) for c in range(3)]
        ts = [_f32(t[c]) for c in range(3)]
        p = [np.zeros_like(xs[0]) for _ in range(3)]
        dw = np.zeros(self.nw, np.float32)
        dr = np.zeros(self.nr, np.float32)
        loss = C.c_double()
        _ck(_lib.mlb_surrogate_gradients(self._h, _fptrs(xs), _fptrs(ts), dw.ctypes.data_as(_F),
                                         dr.ctypes.data_as(_F), _fptrs(p), C.byref(loss)))
        dia = 2 * self.radius + 1
        dR = dr.reshape(self.mx, self.my, self.C, self.C, 2).astype(np.float64)
        return (dw.reshape(dia * dia, self.C, self.C).astype(np.float64), dR[..., 0] + 1j * dR[..., 1],
                np.stack(p), loss.value)

    @staticmethod
    def _ops(ops):
        return (_P * len(ops))(*[o._h for o in ops])

    def train(self, ss, ops, llg, nsteps, window=10, lr=1e-3):
        loss = C.c_double()
        _ck(_lib.mlb_surrogate_train(self._h, ss._h, self._ops(ops), len(ops), llg._h, int(nsteps), int(window),
                                     float(lr), C.byref(loss)))
        return loss.value

    def validate(self, ss, ops, llg, nsteps, window=10):
        out = np.zeros(6)
        _ck(_lib.mlb_surrogate_validate(self._h, ss._h, self._ops(ops), len(ops), llg._h, int(nsteps), int(window),
                                        _dp(out)))
        keys = ["dh_mean", "dh_max", "field_mean", "field_max", "field_without_mean", "field_without_max"]
        return dict(zip(keys, out.tolist()))

    def run(self, ss, ops, llg, nsteps):
        _ck(_lib.mlb_surrogate_run(self._h, ss._h, self._ops(ops), len(ops), llg._h, int(nsteps)))

    def attach(self, ss):
        _ck(_lib.mlb_surrogate_attach(self._h, ss._h))

    def detach(self, ss):
        _ck(_lib.mlb_surrogate_detach(ss._h))

    def stats(self):
        out = (C.c_longlong * 3)()
        b = C.c_double()
        _ck(_lib.mlb_surrogate_stats(self._h, out, C.byref(b)))
        return {"exact": out[0], "surrogate": out[1], "failed": out[2], "last_bound": b.value}


class RungeKutta:
    """make_rk_step_function(ss, type, {ops}, llg, temp) of the reference's
    RungeKutta.lua, run natively: step(n) advances ss by n steps of the
    Butcher scheme `kind` (RK1, RK2, K3, RK4, RK3, RK4_38, RK6, BS3) with the
    field of ops and the optional Thermal operator temp applied after the
    stages.  Steps whose parameters did not change since the previous step
    run as CUDA graphs of the same kernels (setGraph(False): all eager)."""

    def __init__(self, ss, kind, ops, llg, temp=None):
        arr = (_P * len(ops))(*[o._h for o in ops])
        h = _P()
        _ck(_lib.mlb_rk_create(ss._h, kind.encode(), arr, len(ops), llg._h, temp._h if temp is not None else None,
                               C.byref(h)))
        self._h = h
        self._keep = (ss, list(ops), llg, temp)

    def step(self, n=1):
        _ck(_lib.mlb_rk_step(self._h, int(n)))

    def setGraph(self, on=True):
        _ck(_lib.mlb_rk_set_graph(self._h, int(bool(on))))

    def graphSteps(self):
        n = C.c_longlong()
        _ck(_lib.mlb_rk_graph_steps(self._h, C.byref(n)))
        return n.value

    def __call__(self, ss=None, skip_temperature=False):
        """The script's step(ss_input, skip_temperature)."""
        if ss is None:
            self.step(1)
        else:
            _ck(_lib.mlb_rk_step_on(self._h, ss._h, int(bool(skip_temperature))))
        return True

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.mlb_rk_destroy(h)
            self._h = None


class AdaptiveTimeStep:
    """make_adapt_step_function(ss, step, tolerance, llg, temp) of the
    reference's AdaptiveTimeStep.lua over a RungeKutta scheme: step() makes
    one adaptive step of ss and returns whether it was accepted."""

    def __init__(self, ss, rk, tolerance, llg=None, temp=None):
        h = _P()
        _ck(_lib.mlb_adapt_create(ss._h, rk._h, float(tolerance), llg._h if llg is not None else None,
                                  temp._h if temp is not None else None, C.byref(h)))
        self._h = h
        self._keep = (ss, rk, llg, temp)

    def step(self):
        ok = C.c_int()
        _ck(_lib.mlb_adapt_step(self._h, C.byref(ok)))
        return bool(ok.value)

    __call__ = step

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.mlb_adapt_destroy(h)
            self._h = None


def run(ss, ops, llg, nsteps):
    """nsteps of: ss.resetFields(); op.apply(ss) for op in ops; ss.sumFields();
    llg.apply(ss) -- fused and captured in a CUDA graph."""
    arr = (_P * len(ops))(*[o._h for o in ops])
    _ck(_lib.mlb_run(ss._h, arr, len(ops), llg._h, int(nsteps)))
