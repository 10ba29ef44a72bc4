"""LongRange2D and Dipole2D (M/cpu/longrange2d, M/cpu/dipole2d) against the
oracle's restatement: the layer-pair convolution of
spinoperationlongrange2d.cpp:387-530 (compile + apply, tensors read [s][d],
per-layer source-moment and destination-field scales) and the Dipole2D
builder of dip2d_luafuncs.lua:516-660.  FP32 fields within 1e-5 of the FP64
oracle (relative norm), FP64 within 1e-11; the builder's arrays bitwise."""
import numpy as np
import pytest

import oracle as O
from helpers import random_spins, rel_err, tilted_spins

pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-5
F64_FIELD_TOL = 1e-11
AB = ["XX", "XY", "XZ", "YX", "YY", "YZ", "ZX", "ZY", "ZZ"]


@pytest.fixture(scope="module")
def M():
    import maglua_b200 as M
    M.init(0)
    return M


def _system(M, dims, spins, precision="f32"):
    ss = M.SpinSystem(*dims, precision=precision)
    ss.setSpinArrays(*spins)
    return ss


def _set_all(op, T):
    nz = T.shape[0]
    for i in range(nz):
        for j in range(nz):
            for ab in range(9):
                op.setTensorArray(i + 1, j + 1, AB[ab], T[i, j, ab].reshape(-1))


def _field(ss, name):
    return np.stack(ss.fieldArrays(name))


@pytest.mark.parametrize("dims,precision", [((16, 12, 3), "f32"), ((12, 10, 2), "f32"), ((16, 8, 4), "f64"),
                                            ((32, 32, 1), "f32"), ((64, 32, 3), "f32"), ((32, 64, 5), "f32")])
def test_longrange2d_random_tensors(M, dims, precision):
    nx, ny, nz = dims
    r = np.random.default_rng(81)
    T = r.normal(size=(nz, nz, 9, ny, nx)) / (nx * ny)
    src = r.uniform(0.5, 1.5, nz)
    dst = r.uniform(0.5, 1.5, nz)
    s = random_spins(nx * ny * nz, 82, lengths=True)
    ss = _system(M, dims, s, precision)
    op = M.LongRange2D(ss)
    op.setNewDataRequired(False)
    _set_all(op, T)
    for z in range(nz):
        op.setSourceMomentScale(z + 1, src[z])
        op.setDestinationFieldScale(z + 1, dst[z])
    op.setScale(0.7)
    op.apply(ss)
    ref = O.longrange2d_apply(s.reshape(3, nz, ny, nx), T, src, dst, 0.7).reshape(3, -1)
    tol = FIELD_TOL if precision == "f32" else F64_FIELD_TOL
    assert rel_err(_field(ss, "LongRange2D"), ref) <= tol
    # the tensors are read [s][d]: swapping the two layer arguments changes the field
    if nz > 1:
        assert rel_err(ref, O.longrange2d_apply(s.reshape(3, nz, ny, nx), T.transpose(1, 0, 2, 3, 4), src, dst,
                                                0.7).reshape(3, -1)) > 1e-3


def test_longrange2d_data_and_compile_flags(M):
    """New data required at first (apply fails without a make-data function);
    a make-data function fills the arrays; setTensorArray alone is not
    compiled until setCompileRequired, as in the reference."""
    dims = (8, 8, 2)
    nx, ny, nz = dims
    s = random_spins(nx * ny * nz, 83)
    ss = _system(M, dims, s)
    op = M.LongRange2D(ss)
    with pytest.raises(M.MagLuaError, match="make data function not set"):
        op.apply(ss)
    r = np.random.default_rng(84)
    T = r.normal(size=(nz, nz, 9, ny, nx)) / 64
    calls = []

    def make(o):
        calls.append(1)
        _set_all(o, T)

    op.setMakeDataFunction(make)
    op.apply(ss)
    op.apply(ss)
    assert calls == [1] and not op.newDataRequired()
    ones = np.ones(nz)
    ref0 = O.longrange2d_apply(s.reshape(3, nz, ny, nx), T, ones, ones).reshape(3, -1)
    assert rel_err(_field(ss, "LongRange2D"), ref0) <= FIELD_TOL
    T2 = T.copy()
    T2[1, 0, 8] *= -3.0
    op.setTensorArray(2, 1, "ZZ", T2[1, 0, 8].reshape(-1))
    np.testing.assert_array_equal(op.tensorArray(2, 1, "zz"), T2[1, 0, 8])
    assert op.getMatrix(2, 1, 3, 2, "ZZ") == T2[1, 0, 8, 1, 2]
    op.apply(ss)
    assert rel_err(_field(ss, "LongRange2D"), ref0) <= FIELD_TOL       # not compiled yet
    op.setCompileRequired()
    op.apply(ss)
    ref1 = O.longrange2d_apply(s.reshape(3, nz, ny, nx), T2, ones, ones).reshape(3, -1)
    assert rel_err(_field(ss, "LongRange2D"), ref1) <= FIELD_TOL
    with pytest.raises(M.MagLuaError, match="depreciated"):
        op.setStrength(1.0)
    with pytest.raises(M.MagLuaError, match="Invalid Layer"):
        op.setSourceMomentScale(3, 1.0)


def test_dipole2d_builder_and_field(M):
    dims = (8, 6, 3)
    nx, ny, nz = dims
    abc = [np.eye(3), [[1.0, 0.2, 0], [0.1, 1.0, 0], [0.0, 0.3, 1.5]], [[1, 0, 0], [0, 1, 0], [0.2, -0.1, 0.7]]]
    off = [[0, 0, 0], [0.25, 0.5, 0.0], [0.0, -0.3, 0.1]]
    trunc = (25, 4, 3, 1)
    s = random_spins(nx * ny * nz, 85, lengths=True)
    ss = _system(M, dims, s)
    dip = M.Dipole2D(ss)
    assert dip.truncation() == (25, 25, 25, 25)
    for z in range(nz):
        dip.setUnitCell(z + 1, *[list(v) for v in np.asarray(abc[z], float)])
        dip.setOffset(z + 1, off[z])
    dip.setTruncation(*trunc)
    assert dip.truncation() == trunc
    np.testing.assert_array_equal(np.asarray(dip.unitCell(2)), np.asarray(abc[1], float))
    dip.setSourceMomentScale(2, 0.5)
    dip.setDestinationFieldScale(3, 2.0)
    dip.apply(ss)
    T = O.dipole2d_tensor(nx, ny, nz, abc, off, trunc)
    for i in range(nz):
        for j in range(nz):
            for ab in range(9):
                np.testing.assert_array_equal(dip.tensorArray(i + 1, j + 1, AB[ab]), T[i, j, ab])
    src = np.array([1.0, 0.5, 1.0])
    dst = np.array([1.0, 1.0, 2.0])
    ref = O.longrange2d_apply(s.reshape(3, nz, ny, nx), T, src, dst).reshape(3, -1)
    assert rel_err(_field(ss, "Dipole2D"), ref) <= FIELD_TOL


def test_longrange2d_in_steps(M):
    """The operator inside captured steps: the same spins as individual calls."""
    dims = (32, 32, 2)
    nx, ny, nz = dims
    n = nx * ny * nz
    s0 = tilted_spins(n, 86, deg=20.0)
    r = np.random.default_rng(87)
    T = r.normal(size=(nz, nz, 9, ny, nx)) * 1e-3
    out = []
    for mode in ("calls", "run"):
        ss = _system(M, dims, s0)
        ss.setAlpha(0.1)
        ss.setTimeStep(0.01)
        ex = M.Exchange(ss)
        ex.addPaths(*O.nn_paths(*dims, pbc=(1, 1, 0)))
        lr = M.LongRange2D(ss)
        lr.setNewDataRequired(False)
        _set_all(lr, T)
        llg = M.LLG.new("Quaternion")
        ops = [ex, lr]
        if mode == "calls":
            for _ in range(6):
                ss.resetFields()
                for op in ops:
                    op.apply(ss)
                ss.sumFields()
                llg.apply(ss)
        else:
            M.run(ss, ops, llg, 6)
        out.append(np.stack(ss.spinArrays()[:3]))
    np.testing.assert_array_equal(out[0], out[1])
    assert float(np.abs(out[0] - s0).max()) > 1e-6


def test_longrange2d_layer_limit(M):
    ss = M.SpinSystem(4, 4, 65)
    op = M.LongRange2D(ss)
    op.setNewDataRequired(False)
    with pytest.raises(M.MagLuaError, match="at most 64 layers"):
        op.apply(ss)


def test_magnetostatics2d_field(M):
    """Magnetostatics2D with uneven grains per layer and a sheared unit cell:
    the native builder's arrays and the field (1/V source and 4 pi
    destination scales, as a user sets them) against the oracle."""
    dims = (16, 8, 2)
    nx, ny, nz = dims
    abc = [[[1.0, 0, 0], [0.2, 1.0, 0], [0, 0, 1.2]], [[1.0, 0, 0], [0.2, 1.0, 0], [0.1, 0, 0.9]]]
    grain = [[0.9, 0.8, 1.0], [0.7, 0.9, 0.8]]
    trunc = (6, 6, 5, 1)
    s = random_spins(nx * ny * nz, 89, lengths=True)
    ss = _system(M, dims, s)
    mag = M.Magnetostatics2D(ss)
    for z in range(nz):
        mag.setUnitCell(z + 1, *abc[z])
        mag.setGrainSize(z + 1, *grain[z])
        vol = grain[z][0] * grain[z][1] * grain[z][2]
        mag.setSourceMomentScale(z + 1, 1.0 / vol)
        mag.setDestinationFieldScale(z + 1, 4 * np.pi)
    mag.setTruncation(*trunc)
    assert mag.grainSize(2)[3] == pytest.approx(0.7 * 0.9 * 0.8)
    mag.apply(ss)
    T = O.magnetostatics2d_tensor(nx, ny, nz, abc, grain, trunc)
    for i in range(nz):
        for j in range(nz):
            for ab in range(9):
                np.testing.assert_allclose(mag.tensorArray(i + 1, j + 1, AB[ab]), T[i, j, ab], rtol=1e-10,
                                           atol=1e-11 * np.abs(T).max())
    src = [1.0 / np.prod(g) for g in grain]
    ref = O.longrange2d_apply(s.reshape(3, nz, ny, nx), T, src, [4 * np.pi] * nz).reshape(3, -1)
    assert rel_err(_field(ss, "Magnetostatics2D"), ref) <= FIELD_TOL
    # setMatrix marks compile required (mag2d_luafuncs.lua:47-62)
    v = mag.getMatrix(1, 2, "XZ", 3, 1)
    assert v == T[0, 1, 2, 1, 3]
    mag.setMatrix(1, 2, "XZ", 3, 1, v + 0.5)
    assert mag.compileRequired()
    T[0, 1, 2, 1, 3] += 0.5
    mag.apply(ss)
    ref = O.longrange2d_apply(s.reshape(3, nz, ny, nx), T, src, [4 * np.pi] * nz).reshape(3, -1)
    assert rel_err(_field(ss, "Magnetostatics2D"), ref) <= FIELD_TOL
