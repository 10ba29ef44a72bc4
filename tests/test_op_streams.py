"""Operator and LLG checkpoint streams (mlb_op_encode / mlb_llg_encode and
their decoders) byte for byte against the oracle's restatement of the
reference's encode functions, and decode -> encode round trips, including
streams the oracle writes.  Host code only: runs without a GPU through the C
ABI (the operators are created, filled and encoded on the host).  References
(M/ = src/modules/): Exchange M/cpu/exchange/spinoperationexchange.cpp:52-112,
Anisotropy M/cpu/anisotropy/spinoperationanisotropy.cpp:191-236 (Uniaxial,
Cubic: ..._uniaxial.cpp:181-230, ..._cubic.cpp:239-290), Thermal
M/cpu/thermal/spinoperationthermal.cpp:51-77, AppliedField
M/cpu/appliedfield/spinoperationappliedfield.cpp:33-58, Dipole
M/cpu/dipole/spinoperationdipole.cpp:35-59 with LongRange's
M/cpu/longrange/spinoperationlongrange.cpp:55-95, LLG M/cpu/llg/llg.cpp:50-88."""
import ctypes as C

import numpy as np
import pytest

import oracle as O

DIMS = (5, 4, 3)
N = 60


@pytest.fixture(scope="module")
def L():
    import maglua_b200 as M
    return M._lib


def _new(L, kind):
    h = C.c_void_p()
    assert L.mlb_op_create(kind, *DIMS, C.byref(h)) == 0
    return h


def _enc(L, fn, h, idx=0):
    n = C.c_size_t()
    assert fn(h, idx, None, 0, C.byref(n), None) == 0
    buf = C.create_string_buffer(n.value)
    nobj = C.c_int()
    assert fn(h, idx, buf, n.value, C.byref(n), C.byref(nobj)) == 0, L.mlb_last_error().decode()
    return buf.raw[:n.value], nobj.value


def _roundtrip(L, data):
    h = C.c_void_p()
    used = C.c_size_t()
    assert L.mlb_op_decode(data, len(data), C.byref(h), C.byref(used), None) == 0, L.mlb_last_error().decode()
    assert used.value == len(data)
    out, _ = _enc(L, L.mlb_op_encode, h)
    L.mlb_op_destroy(h)
    return out


def _dp(a):
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(C.POINTER(C.c_double))


def test_exchange_stream(L):
    r = np.random.default_rng(1)
    f, t, j = O.nn_paths(*DIMS, pbc=(1, 0, 1))
    j = j * r.uniform(0.5, 1.5, len(j))
    h = _new(L, 1)
    fi, ti, jd = np.ascontiguousarray(f, np.int32), np.ascontiguousarray(t, np.int32), np.ascontiguousarray(j)
    I = C.POINTER(C.c_int)
    assert L.mlb_exchange_add_paths(h, fi.ctypes.data_as(I), ti.ctypes.data_as(I), _dp(jd), len(f)) == 0
    assert L.mlb_exchange_set_normalize(h, 0) == 0
    assert L.mlb_exchange_set_pbc(h, 1, 0, 1) == 0
    assert L.mlb_op_set_scale(h, 0.75) == 0
    got, nobj = _enc(L, L.mlb_op_encode, h, 3)
    want = O.encode_exchange(*DIMS, 0.75, False, (1, 0, 1), f, t, j, first_index=3)
    assert got == want and nobj == 1
    assert _roundtrip(L, want) == O.encode_exchange(*DIMS, 0.75, False, (1, 0, 1), f, t, j)
    L.mlb_op_destroy(h)


def test_anisotropy_streams(L):
    r = np.random.default_rng(2)
    sites = r.permutation(N)[:25].astype(np.int32)
    axes = r.normal(size=(25, 3))            # the Lua add normalises them
    K = r.normal(size=25)
    I = C.POINTER(C.c_int)
    h = _new(L, 2)
    assert L.mlb_anisotropy_add_many(h, 25, sites.ctypes.data_as(I), _dp(axes.ravel()), _dp(K)) == 0
    got, _ = _enc(L, L.mlb_op_encode, h)
    want = O.encode_anisotropy(*DIMS, 1.0, sites, [O.anisotropy_add_axis(a) for a in axes], K)
    assert got == want and _roundtrip(L, want) == want
    L.mlb_op_destroy(h)
    # Uniaxial (its addAnisotropy scales by 1/dot(a, a) on add and on decode:
    # signed coordinate axes, which it keeps exactly)
    axes = np.eye(3)[r.integers(0, 3, 25)] * r.choice([-1.0, 1.0], (25, 1))
    K2 = r.normal(size=25)
    h = _new(L, 3)
    assert L.mlb_uniaxial_add_many(h, 25, sites.ctypes.data_as(I), _dp(axes.ravel()), _dp(K), _dp(K2)) == 0
    got, _ = _enc(L, L.mlb_op_encode, h)
    want = O.encode_uniaxial(*DIMS, 1.0, sites, axes, K, K2)
    assert got == want and _roundtrip(L, want) == want
    L.mlb_op_destroy(h)
    # Cubic: the stored (orthonormalised) axes; the first two are written
    h = _new(L, 4)
    a1 = np.tile([1.0, 0, 0], (25, 1))
    a2 = np.tile([0, 1.0, 0], (25, 1))
    K3 = r.normal(size=(25, 3))
    assert L.mlb_cubic_add_many(h, 25, sites.ctypes.data_as(I), _dp(a1.ravel()), _dp(a2.ravel()),
                                _dp(K3.ravel())) == 0
    got, _ = _enc(L, L.mlb_op_encode, h)
    ax9 = np.tile([1.0, 0, 0, 0, 1.0, 0, 0, 0, 1.0], (25, 1))
    want = O.encode_cubic(*DIMS, 1.0, sites, ax9, K3)
    assert got == want and _roundtrip(L, want) == want
    L.mlb_op_destroy(h)


@pytest.mark.parametrize("per_site", [False, True])
def test_thermal_stream(L, per_site):
    h = _new(L, 5)
    assert L.mlb_thermal_set_temperature(h, 0.35) == 0
    scale = np.ones(N)
    if per_site:
        scale = np.random.default_rng(3).uniform(0.5, 2.0, N)
        for i in range(N):
            assert L.mlb_thermal_scale_site(h, i, float(scale[i])) == 0
    got, nobj = _enc(L, L.mlb_op_encode, h, 2)
    want = O.encode_thermal(*DIMS, 1.0, 0.35, scale if per_site else None, first_index=2)
    assert got == want and nobj == 2
    assert _roundtrip(L, O.encode_thermal(*DIMS, 1.0, 0.35, scale if per_site else None)) == \
        O.encode_thermal(*DIMS, 1.0, 0.35, scale if per_site else None)
    L.mlb_op_destroy(h)


def test_appliedfield_and_dipole_streams(L):
    h = _new(L, 6)
    assert L.mlb_appliedfield_set(h, 0.1, -0.2, 0.3) == 0
    got, _ = _enc(L, L.mlb_op_encode, h)
    want = O.encode_appliedfield(*DIMS, 1.0, (0.1, -0.2, 0.3))
    assert got == want and _roundtrip(L, want) == want
    L.mlb_op_destroy(h)
    h = _new(L, 7)
    gm = (C.c_int * 4)(12, 12, 8, 6)
    assert L.mlb_longrange_set_truncation(h, gm) == 0
    assert L.mlb_longrange_set_strength(h, 0.05) == 0
    abc = [1.0, 0, 0, 0.5, 1.0, 0, 0, 0, 2.0]
    assert L.mlb_longrange_set_unit_cell(h, _dp(abc)) == 0
    got, _ = _enc(L, L.mlb_op_encode, h)
    want = O.encode_dipole(*DIMS, 1.0, (12, 12, 8, 6), 0.05, abc)
    assert got == want and _roundtrip(L, want) == want
    # truncation math.huge is stored and written as -1
    assert L.mlb_longrange_set_truncation(h, (C.c_int * 4)(-1, 0, 0, 0)) == 0
    got, _ = _enc(L, L.mlb_op_encode, h)
    assert got == O.encode_dipole(*DIMS, 1.0, (-1, -1, -1, -1), 0.05, abc)
    L.mlb_op_destroy(h)
    # a plain LongRange has no readable stream in the reference
    h = _new(L, 8)
    n = C.c_size_t()
    assert L.mlb_op_encode(h, 0, None, 0, C.byref(n), None) == -7
    L.mlb_op_destroy(h)


@pytest.mark.parametrize("kind,k", [("Cartesian", 0), ("Quaternion", 1)])
def test_llg_stream(L, kind, k):
    h = C.c_void_p()
    assert L.mlb_llg_create(k, C.byref(h)) == 0
    assert L.mlb_llg_set_flags(h, 0, 1, 0.5, 2.0) == 0
    got, _ = _enc(L, L.mlb_llg_encode, h, 4)
    want = O.encode_llg(kind, 0, 1, 0.5, 2.0, first_index=4)
    assert got == want
    d = C.c_void_p()
    assert L.mlb_llg_decode(want, len(want), C.byref(d), None, None) == 0
    kk = C.c_int()
    assert L.mlb_llg_kind(d, C.byref(kk)) == 0 and kk.value == k
    again, _ = _enc(L, L.mlb_llg_encode, d, 4)
    assert again == want
    L.mlb_llg_destroy(h)
    L.mlb_llg_destroy(d)


def test_truncated_and_foreign_streams_are_rejected(L):
    want = O.encode_appliedfield(*DIMS, 1.0, (0.1, 0.2, 0.3))
    h = C.c_void_p()
    assert L.mlb_op_decode(want[:-3], len(want) - 3, C.byref(h), None, None) == -1
    ss = O.encode_spinsystem(1, 1, 1, 0.1, 0.01, 1.0, 0.0, [1.0], [0.0], [0.0], [1.0])
    assert L.mlb_op_decode(ss, len(ss), C.byref(h), None, None) == -7


# ---------------------------------------------------------------- Magnetostatic tensor (host builder)
@pytest.mark.parametrize("dims,gmax,prism,ABC", [
    ((4, 4, 2), 6, (1.0, 1.0, 1.0), (1, 0, 0, 0, 1, 0, 0, 0, 1)),
    ((5, 3, 3), 5, (1.0, 0.5, 2.0), (1, 0, 0, 0, 0.5, 0, 0, 0, 2.0)),
])
def test_magnetostatic_tensor_matches_oracle(L, dims, gmax, prism, ABC):
    """The Magnetostatic tensor (M/cpu/magnetostatics/magnetostaticssupport.cpp:
    81-187, 799-866 with gamma_ab_v.cpp) built on the host by the library,
    against the oracle's restatement: equal up to the order of images at equal
    distance (the reference sorts with std::sort, the oracle with qsort)."""
    h = C.c_void_p()
    assert L.mlb_op_create(13, *dims, C.byref(h)) == 0
    assert L.mlb_longrange_set_truncation(h, (C.c_int * 4)(gmax, gmax, gmax, gmax)) == 0
    assert L.mlb_longrange_set_unit_cell(h, _dp(ABC)) == 0
    assert L.mlb_magnetostatic_set_cell_dimensions(h, _dp(prism)) == 0
    n = dims[0] * dims[1] * (2 * dims[2] - 1)
    arrs = [np.zeros(n) for _ in range(6)]
    ptrs = (C.POINTER(C.c_double) * 6)(*[a.ctypes.data_as(C.POINTER(C.c_double)) for a in arrs])
    assert L.mlb_longrange_get_tensor(h, ptrs) == 0, L.mlb_last_error().decode()
    ref = O.magnetostatic_tensor(*dims, gmax=(gmax,) * 4, ABC=ABC, prism=prism, tol=1e-5)
    scale = max(np.abs(r).max() for r in ref)
    for a, r in zip(arrs, ref):
        assert np.abs(a.reshape(r.shape) - r).max() <= 1e-9 * scale
    # the crossover is on: the far images use the point dipole, which differs
    # from the prism tensor within the tolerance only
    ref0 = O.magnetostatic_tensor(*dims, gmax=(gmax,) * 4, ABC=ABC, prism=prism, tol=0.0)
    d = max(np.abs(r - r0).max() for r, r0 in zip(ref, ref0))
    assert 0 < d < 1e-3 * scale
    # math.huge is refused (the reference's ring sum for it is not a lattice sum)
    assert L.mlb_longrange_set_truncation(h, (C.c_int * 4)(-1, 0, 0, 0)) == 0
    assert L.mlb_longrange_get_tensor(h, ptrs) == -7
    L.mlb_op_destroy(h)
