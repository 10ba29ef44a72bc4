"""Dipole convolutions whose padded (y,z) plane is larger than one CTA's
shared memory (the 256^3 open cube pads to 512 x 512 planes): the split
y | z + tensor multiply | inverse y passes, in FP32 (fast x passes and the
fused x pass of a step) and FP64 (generic x passes).  Fields against the
oracle's direct dipole sum (open boundaries, M/cpu/dipole/dipolesupport.cpp:
34-70 element) and the reference-mode LongRange algorithm (2D periodic
lattice sum, M/cpu/longrange/spinoperationlongrange.cpp:354-440); the full
256^3 cube at sampled sites."""
import numpy as np
import pytest

import oracle as O
from helpers import random_spins, rel_err, tilted_spins

pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-5        # FP32 state, as the per-term parity tests
F64_FIELD_TOL = 1e-11   # FP64 state


@pytest.fixture(scope="module")
def M():
    import maglua_b200 as M
    M.init(0)
    return M


def _dipole_field(M, dims, spins, g, open_xy=True, precision="f32", trunc=None):
    ss = M.SpinSystem(*dims, precision=precision)
    ss.setSpinArrays(*spins)
    dip = M.Dipole(ss)
    dip.setStrength(g)
    if open_xy:
        dip.setOpen(True, True, True)
    if trunc is not None:
        dip.setTruncation(trunc)
    dip.apply(ss)
    return np.stack(ss.fieldArrays("Dipole"))


@pytest.mark.parametrize("dims", [(8, 64, 24), (16, 40, 30)])
def test_split_fp32_open_direct_sum(M, dims):
    n = int(np.prod(dims))
    s = random_spins(n, 61, lengths=True)
    h = _dipole_field(M, dims, s, 0.4)
    o = O.SpinSystem(*dims)
    o.set_spins(*s)
    assert rel_err(h, O.dipole_direct(o, 0.4)) <= FIELD_TOL


def test_split_fp32_sheared_cell(M):
    # a sheared unit cell: the tensor lacks the per-axis parities, so the
    # split z pass reads the full tensor (no quarter storage)
    dims = (8, 64, 24)
    n = int(np.prod(dims))
    s = random_spins(n, 68, lengths=True)
    abc = (1.0, 0.0, 0.0, 0.3, 1.0, 0.0, 0.1, 0.2, 1.1)
    ss = M.SpinSystem(*dims)
    ss.setSpinArrays(*s)
    dip = M.Dipole(ss)
    dip.setStrength(0.4)
    dip.setOpen(True, True, True)
    dip.setUnitCell(abc[0:3], abc[3:6], abc[6:9])
    dip.apply(ss)
    h = np.stack(ss.fieldArrays("Dipole"))
    o = O.SpinSystem(*dims)
    o.set_spins(*s)
    assert rel_err(h, O.dipole_direct(o, 0.4, ABC=abc)) <= FIELD_TOL


def test_split_fp32_reference_mode(M):
    # periodic in-plane lattice sum (truncated to keep the oracle's sum short),
    # open z padded to 160: plane 32 x 160
    dims = (8, 32, 80)
    n = int(np.prod(dims))
    s = random_spins(n, 62)
    h = _dipole_field(M, dims, s, 0.3, open_xy=False, trunc=24)
    lr = O.LongRange(*dims, O.dipole_tensor(*dims, gmax=(24, 24, 24, 24)))
    o = O.SpinSystem(*dims)
    o.set_spins(*s)
    lr.apply(o, 0.3)
    assert rel_err(h, o.field("Dipole")) <= FIELD_TOL


def test_split_fp32_non_power_of_two_plane(M):
    # periodic y of 40 rows (Py = 40), open z padded to 128: the generic FP32
    # split passes around the fast x passes
    dims = (16, 40, 64)
    n = int(np.prod(dims))
    s = random_spins(n, 67)
    h = _dipole_field(M, dims, s, 0.3, open_xy=False, trunc=8)
    lr = O.LongRange(*dims, O.dipole_tensor(*dims, gmax=(8, 8, 8, 8)))
    o = O.SpinSystem(*dims)
    o.set_spins(*s)
    lr.apply(o, 0.3)
    assert rel_err(h, o.field("Dipole")) <= FIELD_TOL


def test_split_fp64_open_direct_sum(M):
    dims = (8, 64, 12)   # plane 128 x 24 at 16 bytes per complex: split
    n = int(np.prod(dims))
    s = random_spins(n, 63, lengths=True)
    h = _dipole_field(M, dims, s, 0.4, precision="f64")
    o = O.SpinSystem(*dims)
    o.set_spins(*s)
    assert rel_err(h, O.dipole_direct(o, 0.4)) <= F64_FIELD_TOL


def test_split_steps_match_calls_and_oracle(M):
    """Captured steps over the split passes (32 x 64 x 48 film, periodic
    in-plane, z padded to 128: plane 64 x 128) with the fused x pass and the
    carried spectrum equal the individual calls bitwise and follow the FP64
    oracle."""
    dims = (32, 64, 48)
    n = int(np.prod(dims))
    s0 = tilted_spins(n, 64, deg=15.0)
    f, t, j = O.nn_paths(*dims, pbc=(1, 1, 0))
    res = []
    for mode in ("calls", "run"):
        ss = M.SpinSystem(*dims)
        ss.setSpinArrays(*s0)
        ss.setAlpha(0.1)
        ss.setTimeStep(0.01)
        ex = M.Exchange(ss)
        ex.addPaths(f, t, j)
        dip = M.Dipole(ss)
        dip.setStrength(0.05)
        dip.setTruncation(24)
        ops = [ex, dip]
        llg = M.LLG.new("Quaternion")
        if mode == "calls":
            for _ in range(4):
                ss.resetFields()
                for op in ops:
                    op.apply(ss)
                ss.sumFields()
                llg.apply(ss)
        else:
            M.run(ss, ops, llg, 4)
        res.append(np.stack(ss.spinArrays()[:3]))
    np.testing.assert_array_equal(res[0], res[1])
    o = O.SpinSystem(*dims)
    o.set_spins(*s0)
    o.alpha, o.dt = 0.1, 0.01
    lr = O.LongRange(*dims, O.dipole_tensor(*dims, gmax=(24, 24, 24, 24)))
    O.run_steps(o, 4, paths=(f, t, j), lr=lr, g=0.05, llg="Quaternion")
    assert float(np.abs(res[1] - o.spins()).max()) < 1e-6


def test_cube_256_open_sampled_sites(M):
    """The 256^3 simple-cubic cube with open boundaries (zero-padded 512^3
    transform): dipole field of random spins at sampled sites against the
    direct sum over all 16.7M sources."""
    dims = (256, 256, 256)
    n = int(np.prod(dims))
    s = random_spins(n, 65)
    h = _dipole_field(M, dims, s, 0.03)
    r = np.random.default_rng(66)
    corners = [0, n - 1, 255, 256 * 255, n // 2 + 128 * 256 + 128]
    sites = np.concatenate([corners, r.integers(0, n, 5)])
    ref = O.dipole_direct_sites(dims, s, 0.03, sites)
    assert rel_err(h[:, sites], ref) <= FIELD_TOL


def test_split_fp64_steps_match_calls_and_oracle(M):
    """FP64 state on a plane larger than shared memory (32 x 64 x 24,
    periodic in-plane, z padded to 64: 64 x 64 complex doubles): the
    register split passes in double; captured steps equal the individual
    calls bitwise and follow the FP64 oracle."""
    dims = (32, 64, 24)
    n = int(np.prod(dims))
    s0 = tilted_spins(n, 69, deg=15.0)
    f, t, j = O.nn_paths(*dims, pbc=(1, 1, 0))
    res = []
    for mode in ("calls", "run"):
        ss = M.SpinSystem(*dims, precision="f64")
        ss.setSpinArrays(*s0)
        ss.setAlpha(0.1)
        ss.setTimeStep(0.01)
        ex = M.Exchange(ss)
        ex.addPaths(f, t, j)
        dip = M.Dipole(ss)
        dip.setStrength(0.05)
        dip.setTruncation(12)
        ops = [ex, dip]
        llg = M.LLG.new("Quaternion")
        if mode == "calls":
            for _ in range(4):
                ss.resetFields()
                for op in ops:
                    op.apply(ss)
                ss.sumFields()
                llg.apply(ss)
        else:
            M.run(ss, ops, llg, 4)
        res.append(np.stack(ss.spinArrays()[:3]))
    np.testing.assert_array_equal(res[0], res[1])
    o = O.SpinSystem(*dims)
    o.set_spins(*s0)
    o.alpha, o.dt = 0.1, 0.01
    lr = O.LongRange(*dims, O.dipole_tensor(*dims, gmax=(12, 12, 12, 12)))
    O.run_steps(o, 4, paths=(f, t, j), lr=lr, g=0.05, llg="Quaternion")
    assert float(np.abs(res[1] - o.spins()).max()) < 1e-11
