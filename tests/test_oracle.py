"""CPU checks of the FP64 oracle: published known answers, numpy, closed
forms, a direct dipole sum, the reference's LongRange3D-vs-Exchange script,
and the committed golden fixtures."""
import json
import os

import numpy as np
import pytest

import oracle as O
from helpers import random_spins, rel_err

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


# ---------------------------------------------------------------- MT19937
def test_mt19937_published_outputs():
    # mt19937ar.c test vectors (Matsumoto & Nishimura): init_genrand(5489)
    # first output, and the first outputs after init_by_array({0x123,...}).
    assert O.MT(5489).randint() == 3499211612
    m = O.MT(key=[0x123, 0x234, 0x345, 0x456])
    assert [m.randint() for _ in range(5)] == [1067595299, 955945823, 477289528, 4107218783, 4228976476]


def test_mt_rand_and_polar_normal():
    m1, m2 = O.MT(7), O.MT(7)
    u = [m1.rand() for _ in range(4)]
    ints = [m2.randint() for _ in range(4)]
    assert u == [i * (1.0 / 4294967295.0) for i in ints]
    # MTRand::randNorm: polar method keeping only x*s (mersennetwister.h:340-352)
    m3, m4 = O.MT(11), O.MT(11)
    z = m3.normal()
    while True:
        x = 2.0 * m4.rand() - 1.0
        y = 2.0 * m4.rand() - 1.0
        r = x * x + y * y
        if not (r >= 1.0 or r == 0.0):
            break
    assert z == x * np.sqrt(-2.0 * np.log(r) / r)


def test_mt_normal_statistics():
    m = O.MT(3)
    v = np.array([m.normal() for _ in range(20000)])
    assert abs(v.mean()) < 0.03 and abs(v.std() - 1) < 0.03


# ---------------------------------------------------------------- FFT
@pytest.mark.parametrize("n", [1, 2, 3, 5, 7, 8, 12, 15, 16, 17, 48, 96, 100, 128, 256])
def test_fft_matches_numpy(n):
    r = np.random.default_rng(n)
    a = r.normal(size=n) + 1j * r.normal(size=n)
    np.testing.assert_allclose(O.fft1d(a, -1), np.fft.fft(a), atol=1e-12 * n)
    np.testing.assert_allclose(O.fft1d(a, +1), np.fft.ifft(a) * n, atol=1e-12 * n)


def test_fft3d_and_layers_match_numpy():
    r = np.random.default_rng(1)
    d = r.normal(size=(3, 6, 5)) + 1j * r.normal(size=(3, 6, 5))
    np.testing.assert_allclose(O.fft3d(d, -1), np.fft.fftn(d), atol=1e-12)
    np.testing.assert_allclose(O.fft2d_layers(d, -1), np.fft.fft2(d), atol=1e-12)


# ---------------------------------------------------------------- dipole tensor
def _gamma(r):
    n = np.linalg.norm(r)
    if n < 1e-40:
        return np.zeros((3, 3))
    return (3 * np.outer(r, r) - np.eye(3) * n * n) / n ** 5


def test_dipole_tensor_against_explicit_image_sum():
    nx, ny, nz, G = 4, 3, 2, 7
    T = O.dipole_tensor(nx, ny, nz, gmax=(G, G, G, G))
    for (i, j, k) in [(0, 0, 0), (1, 2, 0), (3, 1, 1), (2, 0, -1)]:
        acc = np.zeros((3, 3))
        for X in range(-(G - 1), G):
            for Y in range(-(G - 1), G):
                xx, yy = X * nx + i, Y * ny + j
                if abs(xx) <= G and abs(yy) <= G and xx * xx + yy * yy + k * k <= G * G:
                    acc += _gamma(np.array([xx, yy, k], float))
        got = [T[q][k + nz - 1, j, i] for q in range(6)]
        want = [acc[0, 0], acc[0, 1], acc[0, 2], acc[1, 1], acc[1, 2], acc[2, 2]]
        np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-14)


def test_dipole_tensor_even_and_trace_free():
    T = O.dipole_tensor(8, 8, 3, gmax=(30, 30, 30, 30))
    XX, XY, XZ, YY, YZ, ZZ = T
    # inversion symmetry of the lattice sum: W(-i,-j,-k) = W(i,j,k)
    inv = lambda a: np.roll(a[::-1, ::-1, ::-1], shift=(0, 1, 1), axis=(0, 1, 2))
    for a in T:
        np.testing.assert_allclose(inv(a), a, atol=1e-12)
    # Gamma is trace free term by term
    np.testing.assert_allclose(XX + YY + ZZ, 0, atol=1e-12)


# ---------------------------------------------------------------- LongRange
def test_longrange_matches_real_space_convolution():
    nx, ny, nz = 5, 4, 3
    n = nx * ny * nz
    s = random_spins(n, 2, lengths=True)
    ss = O.SpinSystem(nx, ny, nz)
    ss.set_spins(*s)
    T6 = O.dipole_tensor(nx, ny, nz, gmax=(20, 20, 20, 20))
    lr = O.LongRange(nx, ny, nz, T6)
    lr.apply(ss, g=0.3)
    h = ss.field("Dipole")
    # h_t = g sum_s W(r_t - r_s in plane, z offset s - t) s_s
    XX, XY, XZ, YY, YZ, ZZ = T6
    S = s.reshape(3, nz, ny, nx)
    want = np.zeros((3, nz, ny, nx))
    for tz in range(nz):
        for ty in range(ny):
            for tx in range(nx):
                acc = np.zeros(3)
                for sz in range(nz):
                    k = sz - tz + nz - 1
                    for sy in range(ny):
                        for sx in range(nx):
                            i, j = (tx - sx) % nx, (ty - sy) % ny
                            W = np.array([[XX[k, j, i], XY[k, j, i], XZ[k, j, i]],
                                          [XY[k, j, i], YY[k, j, i], YZ[k, j, i]],
                                          [XZ[k, j, i], YZ[k, j, i], ZZ[k, j, i]]])
                            acc += W @ S[:, sz, sy, sx]
                want[:, tz, ty, tx] = 0.3 * acc
    np.testing.assert_allclose(h, want.reshape(3, -1), atol=1e-12)


@pytest.mark.parametrize("dims", [(5, 4, 3), (8, 6, 1), (7, 7, 2)])
def test_open_dipole_fft_equals_direct_sum(dims):
    # the FFT form of the open-boundary dipole field (O.DipoleOpen, used for
    # ensemble trajectories) is the physical direct sum with no images
    n = int(np.prod(dims))
    s = random_spins(n, 6, lengths=True)
    ss = O.SpinSystem(*dims)
    ss.set_spins(*s)
    want = O.dipole_direct(ss, 0.3)
    got = O.DipoleOpen(*dims).field(s, 0.3)
    assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()


def test_longrange_single_layer_equals_direct_periodic_sum():
    # nz = 1: the periodic lattice sum with a radius cut-off equals a direct
    # sum over all images inside the same cut-off.
    nx, ny, G = 6, 5, 12
    n = nx * ny
    s = random_spins(n, 4)
    ss = O.SpinSystem(nx, ny, 1)
    ss.set_spins(*s)
    lr = O.LongRange(nx, ny, 1, O.dipole_tensor(nx, ny, 1, gmax=(G, G, G, G)))
    lr.apply(ss, g=1.0)
    h = ss.field("Dipole")
    pos = np.array([(i % nx, i // nx) for i in range(n)])
    want = np.zeros((3, n))
    for t in range(n):
        for sidx in range(n):
            for X in range(-3, 4):
                for Y in range(-3, 4):
                    d = pos[t] - pos[sidx] + np.array([X * nx, Y * ny])
                    if abs(d[0]) <= G and abs(d[1]) <= G and d @ d <= G * G:
                        want[:, t] += _gamma(np.array([d[0], d[1], 0.0])) @ s[:, sidx]
    np.testing.assert_allclose(h, want, atol=1e-12)


def test_longrange3d_nearest_neighbour_tensor_equals_exchange():
    # M/cpu/longrange3d/test.lua: LongRange3D with a nearest-neighbour
    # tensor reproduces Exchange; here with a tolerance.
    nx, ny, nz = 4, 5, 3
    n = nx * ny * nz
    s = random_spins(n, 5)
    a = O.SpinSystem(nx, ny, nz)
    a.set_spins(*s)
    b = O.SpinSystem(nx, ny, nz)
    b.set_spins(*s)
    f, t, j = O.nn_paths(nx, ny, nz, J=1.0)
    O.exchange_apply(a, f, t, j, normalize=False)
    T9 = [np.zeros((nz, ny, nx)) for _ in range(9)]
    for d in [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]:
        for q in (0, 4, 8):
            T9[q][d[2] % nz, d[1] % ny, d[0] % nx] += 1.0
    O.longrange3d_apply(b, T9, g=1.0)
    np.testing.assert_allclose(b.field("LongRange3D"), a.field("Exchange"), atol=1e-12)


# ---------------------------------------------------------------- operators / LLG
def test_uniaxial_quirk_zero_field_along_z():
    ss = O.SpinSystem(3, 1, 1)
    ss.set_spins(*random_spins(3, 1))
    O.anisotropy_uniaxial_apply(ss, [0, 1, 2], np.tile([0, 0, 1.0], (3, 1)), [1.0] * 3, [0.5] * 3, quirk=True)
    np.testing.assert_array_equal(ss.field("UniaxialAnisotropy"), 0)
    O.anisotropy_uniaxial_apply(ss, [0, 1, 2], np.tile([0, 0, 1.0], (3, 1)), [1.0] * 3, [0.5] * 3, quirk=False)
    u = ss.z / ss.ms
    np.testing.assert_allclose(ss.field("UniaxialAnisotropy")[2], 2 * u + 2 * u ** 3, rtol=1e-14)


def test_llg_preserves_length_and_zero_field_is_identity():
    n = 50
    s = random_spins(n, 8, lengths=True)
    for kind in ("Cartesian", "Quaternion"):
        ss = O.SpinSystem(n, 1, 1)
        ss.set_spins(*s)
        ss.dt = 0.05
        hx, hy, hz = ss.field_views("Total")
        hx[:], hy[:], hz[:] = random_spins(n, 9)
        O.LLG(kind).apply(ss)
        np.testing.assert_allclose(np.sqrt(ss.x ** 2 + ss.y ** 2 + ss.z ** 2), ss.ms, rtol=1e-14)
        assert ss.time == pytest.approx(0.05)
        ss2 = O.SpinSystem(n, 1, 1)
        ss2.set_spins(*s)
        O.LLG(kind).apply(ss2)
        np.testing.assert_allclose(ss2.spins(), s, atol=1e-15)


def test_quaternion_step_is_exact_rotation_for_precession():
    # alpha = 0: rotation by gamma |H| dt about H
    ss = O.SpinSystem(1, 1, 1)
    ss.set_spins([1.0], [0.0], [0.0])
    ss.alpha, ss.dt = 0.0, 0.3
    hx, hy, hz = ss.field_views("Total")
    hz[0] = 2.0
    O.LLG("Quaternion").apply(ss)
    ang = 2.0 * 0.3
    np.testing.assert_allclose([ss.x[0], ss.y[0]], [np.cos(ang), np.sin(ang)], atol=1e-14)


def test_thermal_sigma_and_stream_order():
    n = 20
    ss = O.SpinSystem(n, 1, 1)
    ss.set_spins(*random_spins(n, 3))
    ss.alpha, ss.dt, ss.gamma = 0.1, 0.01, 1.0
    m1 = O.MT(99)
    O.thermal_apply(ss, 0.5, m1)
    h = ss.field("Thermal")
    m2 = O.MT(99)
    nz = np.array([[m2.normal() for _ in range(3)] for _ in range(n)]).T
    sig = np.sqrt(2 * 0.1 * 0.5 / (1.0 * 0.01 * 1.0))
    np.testing.assert_allclose(h, sig * nz, rtol=1e-14)


# ---------------------------------------------------------------- golden fixtures
def _golden():
    with open(os.path.join(GOLDEN, "golden.json")) as f:
        return json.load(f)


def test_golden_fixtures_reproduce():
    """The oracle still produces the committed fixtures (tests/golden/make_golden.py)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    gold = _golden()
    fresh = mg.compute(quick=True)
    for key, val in fresh.items():
        ref = gold[key]
        np.testing.assert_allclose(np.asarray(val), np.asarray(ref), rtol=1e-12, atol=1e-13, err_msg=key)


def test_longrange2d_oracle_is_the_circular_convolution():
    """The transform-based LongRange2D oracle against the real-space sum it
    stands for: H_a[d](r) = dst[d] g sum_s src[s] sum_b sum_r' T[s][d][ab](r - r')
    M_b[s](r'), periodic in x and y."""
    nx, ny, nz = 5, 4, 2
    r = np.random.default_rng(88)
    T = r.normal(size=(nz, nz, 9, ny, nx))
    S = r.normal(size=(3, nz, ny, nx))
    src, dst = np.array([0.7, 1.3]), np.array([1.1, 0.4])
    h = O.longrange2d_apply(S, T, src, dst, 0.5)
    ref = np.zeros_like(h)
    for a in range(3):
        for d in range(nz):
            for y in range(ny):
                for x in range(nx):
                    acc = 0.0
                    for s_ in range(nz):
                        for b in range(3):
                            for yp in range(ny):
                                for xp in range(nx):
                                    acc += src[s_] * T[s_, d, 3 * a + b, (y - yp) % ny, (x - xp) % nx] * S[b, s_, yp, xp]
                    ref[a, d, y, x] = dst[d] * 0.5 * acc
    np.testing.assert_allclose(h, ref, rtol=1e-12, atol=1e-12)


def _mag2d_fixture():
    with open(os.path.join(GOLDEN, "mag2d_save_test.json")) as f:
        return json.load(f)


NAMES9 = ["XX", "XY", "XZ", "YX", "YY", "YZ", "ZX", "ZY", "ZZ"]


def _fixture_arrays(fx):
    out = {}
    for key, comps in fx["arrays"].items():
        d, s_ = (int(v) - 1 for v in key.split(","))
        for ab, rows in comps.items():
            out[(d, s_, NAMES9.index(ab))] = np.asarray(rows) * fx["sign_of_file"]
    return out


def test_magnetostatics2d_oracle_matches_reference_data_file():
    """The Magnetostatics2D builder restated in the oracle against the
    reference's tensor data file (dipole2d/save_test.lua, 16 x 16 x 2, 1e-6
    cells and grains, truncation 20, values printed to 7 significant
    digits).  The file holds +N; the current makeData adds -N."""
    fx = _mag2d_fixture()
    a, g = fx["unit_cell"], fx["grain"]
    abc = np.tile(np.eye(3) * a, (2, 1, 1))
    T = O.magnetostatics2d_tensor(16, 16, 2, abc, np.full((2, 3), g), fx["truncation"])
    for (d, s_, ab), ref in _fixture_arrays(fx).items():
        got = -T[d, s_, ab]
        np.testing.assert_allclose(got, ref, rtol=1e-6, atol=2e-7 * np.abs(ref).max() + 1e-12)


def test_magnetostatics2d_builder_in_the_library(tmp_path):
    """The library's native builder (host code, no GPU needed) against the
    oracle and the reference's data file."""
    import ctypes as C
    import maglua_b200
    lib = maglua_b200._lib.load()
    fx = _mag2d_fixture()
    a, g = fx["unit_cell"], fx["grain"]
    op = C.c_void_p()
    assert lib.mlb_op_create(12, 16, 16, 2, C.byref(op)) == 0
    try:
        for z in range(2):
            abc = (C.c_double * 9)(a, 0, 0, 0, a, 0, 0, 0, a)
            assert lib.mlb_dipole2d_set_unit_cell(op, z, abc) == 0
            assert lib.mlb_magnetostatics2d_set_grain_size(op, z, (C.c_double * 3)(g, g, g)) == 0
        assert lib.mlb_dipole2d_set_truncation(op, (C.c_int * 4)(*fx["truncation"])) == 0
        assert lib.mlb_dipole2d_make_data(op) == 0
        T = O.magnetostatics2d_tensor(16, 16, 2, np.tile(np.eye(3) * a, (2, 1, 1)), np.full((2, 3), g),
                                      fx["truncation"])
        ref = _fixture_arrays(fx)
        buf = np.zeros(256)
        for d in range(2):
            for s_ in range(2):
                for ab in range(9):
                    assert lib.mlb_longrange2d_get_tensor(op, d, s_, ab, buf.ctypes.data_as(C.POINTER(C.c_double))) == 0
                    got = buf.reshape(16, 16)
                    np.testing.assert_allclose(got, T[d, s_, ab], rtol=1e-11, atol=1e-11 * np.abs(T).max())
                    if (d, s_, ab) in ref:
                        r = ref[(d, s_, ab)]
                        np.testing.assert_allclose(-got, r, rtol=1e-6, atol=2e-7 * np.abs(r).max() + 1e-12)
    finally:
        lib.mlb_op_destroy(op)


def _mag2d_reference_layout_text(fx):
    """A Magnetostatics2D data file in the layout of the reference's writer
    (mag2d_luafuncs.lua:278-330: header, builder state, then the blocks), with
    the fixture's arrays as [1][1], [1][2] and their layer mirrors."""
    a, g = fx["unit_cell"], fx["grain"]
    lines = ["-- Magnetostatics2D Data File", "--", "MagLua_Version = 400", "", "-- system size",
             "local nx, ny, nz = 16, 16, 2", "\t", "-- internal state", "local internal = {}",
             "internal.ABC = {}", "internal.grainSize = {}"]
    for z in (1, 2):
        lines.append(f"internal.ABC[{z}] = {{{{{a:g}, 0, 0}}, {{0, {a:g}, 0}}, {{0, 0, {a:g}}}}}")
    lines.append("")
    for z in (1, 2):
        lines.append(f"internal.grainSize[{z}] = {{{g:g}, {g:g}, {g:g}}}")
    for k, v in zip(["truncation ", "truncationX", "truncationY", "truncationZ"], fx["truncation"]):
        lines.append(f"internal.{k} = {v}")
    lines += ["", "-- interaction tensors. Format is AB[destination_layer][source_layer]"]
    for ab in NAMES9:
        lines.append(f"local {ab} = {{{{}}, {{}}}}")
    arrays = {}
    for key, comps in fx["arrays"].items():
        d, s_ = (int(v) for v in key.split(","))
        for ab, rows in comps.items():
            arrays[(ab, d, s_)] = rows
            arrays[(ab, 3 - d, 3 - s_)] = rows
    for ab in NAMES9:
        for d in (1, 2):
            for s_ in (1, 2):
                lines.append(f"{ab}[{d}][{s_}] = [[")
                for row in arrays[(ab, d, s_)]:
                    lines.append(", ".join("0" if v == 0 else f"{v:E}" for v in row))
                lines.append("]]")
    lines.append("return function() end")
    return "\n".join(lines) + "\n", arrays


def test_lr2d_data_files_in_the_library(tmp_path):
    """Tensor data files (dip2d_luafuncs.lua:278-500, mag2d_luafuncs.lua:
    278-480) through the library's host code: a file in the reference's
    layout loads only into a matching operator; a written file reads back."""
    import ctypes as C
    import maglua_b200
    lib = maglua_b200._lib.load()
    fx = _mag2d_fixture()
    a, g = fx["unit_cell"], fx["grain"]
    text, arrays = _mag2d_reference_layout_text(fx)
    ref_file = tmp_path / "MAB_16x16x2.0.lua"
    ref_file.write_text(text)
    dp = C.POINTER(C.c_double)

    def mag_op(grain=g, trunc=fx["truncation"]):
        op = C.c_void_p()
        assert lib.mlb_op_create(12, 16, 16, 2, C.byref(op)) == 0
        for z in range(2):
            assert lib.mlb_dipole2d_set_unit_cell(op, z, (C.c_double * 9)(a, 0, 0, 0, a, 0, 0, 0, a)) == 0
            assert lib.mlb_magnetostatics2d_set_grain_size(op, z, (C.c_double * 3)(grain, grain, grain)) == 0
        assert lib.mlb_dipole2d_set_truncation(op, (C.c_int * 4)(*trunc)) == 0
        return op

    def tensor(op, d, s_, ab):
        buf = np.zeros(256)
        assert lib.mlb_longrange2d_get_tensor(op, d, s_, ab, buf.ctypes.data_as(dp)) == 0
        return buf.reshape(16, 16)

    loaded = C.c_int()
    op = mag_op()
    try:
        assert lib.mlb_lr2d_read_data_file(op, str(ref_file).encode(), C.byref(loaded)) == 0 and loaded.value == 1
        nd, cr = C.c_int(), C.c_int()
        assert lib.mlb_longrange2d_get_required(op, C.byref(nd), C.byref(cr)) == 0
        assert (nd.value, cr.value) == (0, 1)
        for (ab, d, s_), rows in arrays.items():
            np.testing.assert_array_equal(tensor(op, d - 1, s_ - 1, NAMES9.index(ab)), np.asarray(rows))
        # written by the library, read into a fresh operator
        out = tmp_path / "MAB_16x16x2.1.lua"
        assert lib.mlb_lr2d_write_data_file(op, str(out).encode()) == 0
        txt = out.read_text()
        assert txt.startswith("-- Magnetostatics2D Data File") and "internal.grainSize[2] = {1e-06, 1e-06, 1e-06}" in txt
        op2 = mag_op()
        assert lib.mlb_lr2d_read_data_file(op2, str(out).encode(), C.byref(loaded)) == 0 and loaded.value == 1
        for d in range(2):
            for s_ in range(2):
                for ab in range(9):
                    np.testing.assert_allclose(tensor(op2, d, s_, ab), tensor(op, d, s_, ab), rtol=1e-15, atol=0)
        lib.mlb_op_destroy(op2)
        # other grain size or truncation: not loaded, arrays untouched
        for other in (mag_op(grain=2e-6), mag_op(trunc=(25, 25, 25, 25))):
            assert lib.mlb_lr2d_read_data_file(other, str(ref_file).encode(), C.byref(loaded)) == 0
            assert loaded.value == 0
            assert lib.mlb_longrange2d_get_required(other, C.byref(nd), C.byref(cr)) == 0 and nd.value == 1
            lib.mlb_op_destroy(other)
        # a Dipole2D operator does not take a Magnetostatics2D file
        dop = C.c_void_p()
        assert lib.mlb_op_create(11, 16, 16, 2, C.byref(dop)) == 0
        assert lib.mlb_lr2d_read_data_file(dop, str(ref_file).encode(), C.byref(loaded)) == 0 and loaded.value == 0
        # Dipole2D round trip
        assert lib.mlb_dipole2d_set_truncation(dop, (C.c_int * 4)(25, 3, 2, 1)) == 0
        gab = tmp_path / "GAB_16x16x2.0.lua"
        assert lib.mlb_lr2d_write_data_file(dop, str(gab).encode()) == 0
        dop2 = C.c_void_p()
        assert lib.mlb_op_create(11, 16, 16, 2, C.byref(dop2)) == 0
        assert lib.mlb_dipole2d_set_truncation(dop2, (C.c_int * 4)(25, 3, 2, 1)) == 0
        assert lib.mlb_lr2d_read_data_file(dop2, str(gab).encode(), C.byref(loaded)) == 0 and loaded.value == 1
        T = O.dipole2d_tensor(16, 16, 2, np.tile(np.eye(3), (2, 1, 1)), np.zeros((2, 3)), (25, 3, 2, 1))
        for d in range(2):
            for s_ in range(2):
                for ab in range(9):
                    np.testing.assert_allclose(tensor(dop2, d, s_, ab), T[d, s_, ab], rtol=1e-15, atol=0)
        lib.mlb_op_destroy(dop)
        lib.mlb_op_destroy(dop2)
    finally:
        lib.mlb_op_destroy(op)


SHEARED = [[1, 0, 0], [0.5, 0.8, 0], [0.1, 0.2, 0.9]]


def test_ewald_oracle_physics():
    """Properties of the Ewald sum that hold whatever its implementation:
    trace G(r) = -4 pi / V away from the lattice points, independence of the
    real/reciprocal split eta, and G_aa(0) = 0 on a cubic lattice."""
    g = O.ewald_geometry((4, 4, 4), SHEARED)
    eta = O.ewald_find_eta(g, SHEARED[0], 0)
    assert eta is not None and 0.5 < eta < 5
    for r in ([0.3, -1.1, 2.0], [2.0, 2.0, 2.0]):
        tr = sum(O.ewald_element(g, a, a, r, eta, 10) for a in range(3))
        assert tr == pytest.approx(-4 * np.pi / g[2], rel=1e-9)
    v = O.ewald_element(g, 0, 1, [0.3, -1.1, 2.0], eta, 10)
    for e2 in (0.8 * eta, 1.2 * eta):
        assert O.ewald_element(g, 0, 1, [0.3, -1.1, 2.0], e2, 10) == pytest.approx(v, rel=1e-8)
    gc = O.ewald_geometry((3, 3, 3), np.eye(3))
    ec = O.ewald_find_eta(gc, [1, 0, 0], 0)
    for a in range(3):
        assert abs(O.ewald_element(gc, a, a, [0, 0, 0], ec, 8)) < 1e-12


def test_ewald_library_host_path():
    """DipoleEwald3D through the library's host code (no GPU): the eta search
    and single elements against the oracle's restatement of ewald3d.cpp."""
    import ctypes as C
    import maglua_b200
    lib = maglua_b200._lib.load()
    e = C.c_void_p()
    assert lib.mlb_ewald3d_create(4, 4, 4, C.byref(e)) == 0
    try:
        d3 = lambda v: (C.c_double * 3)(*v)   # noqa: E731
        assert lib.mlb_ewald3d_set_unit_cell(e, d3(SHEARED[0]), d3(SHEARED[1]), d3(SHEARED[2])) == 0
        vol = C.c_double()
        lib.mlb_ewald3d_get_volume(e, C.byref(vol))
        g = O.ewald_geometry((4, 4, 4), SHEARED)
        assert vol.value == g[2]
        out = C.c_double()
        assert lib.mlb_ewald3d_element(e, 1, (C.c_int * 3)(1, 2, 0), C.byref(out)) == 0
        eta = C.c_double()
        lib.mlb_ewald3d_get_eta(e, C.byref(eta))
        eta_o = O.ewald_find_eta(g, SHEARED[0], 0)
        assert eta.value == pytest.approx(eta_o, rel=2e-3)
        for ab, r3 in [(1, (1, 2, 0)), (0, (0, 0, 0)), (4, (0, 0, 0)), (5, (3, 1, 2)), (7, (3, 1, 2)), (8, (2, 0, 1))]:
            assert lib.mlb_ewald3d_element(e, ab, (C.c_int * 3)(*r3), C.byref(out)) == 0
            r = [sum(r3[j] * SHEARED[j][i] for j in range(3)) for i in range(3)]
            ref = O.ewald_element(g, ab // 3, ab % 3, r, eta.value, 10)
            assert out.value == pytest.approx(ref, rel=1e-12, abs=1e-15)
        assert lib.mlb_ewald3d_element_real(e, 2, d3([0.3, -1.1, 2.0]), C.byref(out)) == 0
        assert out.value == pytest.approx(O.ewald_element(g, 0, 2, [0.3, -1.1, 2.0], eta.value, 10), rel=1e-12)
        # reference setters: tau <= 0 and NSites <= 1 are ignored
        lib.mlb_ewald3d_set_tau(e, C.c_double(-1.0))
        lib.mlb_ewald3d_set_nsites(e, 1)
        t, n = C.c_double(), C.c_int()
        lib.mlb_ewald3d_get_tau(e, C.byref(t))
        lib.mlb_ewald3d_get_nsites(e, C.byref(n))
        assert (t.value, n.value) == (1e-3, 10)
        assert lib.mlb_ewald3d_element(e, 9, (C.c_int * 3)(0, 0, 0), C.byref(out)) != 0
        assert b"AB pair" in lib.mlb_last_error()
    finally:
        lib.mlb_ewald3d_destroy(e)


def test_type_ids_against_the_reference_murmur():
    """The oracle's hash32 against the ids the reference's own MurmurHash3
    (compiled from its source) gave for these names: every tail length."""
    with open(os.path.join(GOLDEN, "type_hashes.json")) as f:
        fx = json.load(f)
    assert fx["seed"] == 1000
    for name, v in fx["hash32"].items():
        assert O.type_hash32(name) == v, name


def test_spinsystem_stream_round_trip_on_the_oracle():
    """encode_spinsystem / decode_spinsystem: the field order and sizes of
    SpinSystem::encode (spinsystem.cpp:669-757) and Array<double>::encode."""
    import struct
    n = 5 * 4 * 3
    s = random_spins(n, 61)
    ms = np.full(n, 2.0)
    sg = np.linspace(0.5, 1.5, n)
    data = O.encode_spinsystem(5, 4, 3, 0.2, 0.01, 1.3, 7.0, s[0], s[1], s[2], ms, None, sg)
    t, ty, magic, idx, ver = struct.unpack_from("=iibib", data, 0)
    assert (t, ty, magic, idx, ver) == (7, O.type_hash32("SpinSystem"), 111, 0, 0)
    assert struct.unpack_from("=iiidddd", data, 14) == (5, 4, 3, 0.2, 0.01, 1.3, 7.0)
    # the x array follows: its own header, index 1, then flag 0 and n doubles
    t, ty, magic, idx, ver, ax, ay, az, flag = struct.unpack_from("=iibibiiii", data, 58)
    assert (t, ty, magic, idx, ver, (ax, ay, az), flag) == (7, O.type_hash32("Array.Double"), 111, 1, 0,
                                                            (5, 4, 3), 0)
    d = O.decode_spinsystem(data)
    assert np.array_equal(d["x"], s[0]) and np.array_equal(d["ms"], ms)
    assert d["site_alpha"] is None and np.array_equal(d["site_gamma"], sg)
    # the uniform ms array is one value (flag 1)
    assert len(data) == 13 + 1 + 12 + 32 + 5 * 30 + 4 * 8 * n + 8 + 12


def test_type_ids_against_the_built_reference_murmur():
    """Where oracle/_ref holds the reference's MurmurHash3 built from its
    source, the oracle's hash32 equals it on random names of every length."""
    import ctypes
    so = os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref", "libmurmur.so")
    if not os.path.exists(so):
        pytest.skip("oracle/_ref/libmurmur.so not built (reference tree absent)")
    fn = ctypes.CDLL(so)._Z18MurmurHash3_x86_32PKvijPv
    r = np.random.default_rng(7)
    for length in range(0, 40):
        name = bytes(r.integers(32, 127, size=length).astype(np.uint8)).decode()
        res = ctypes.c_int()
        b = name.encode()
        fn(b, len(b), 1000, ctypes.byref(res))
        assert O.type_hash32(name) == res.value, name
