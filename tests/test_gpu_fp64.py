"""FP64 state on the device (SpinSystem(..., precision="f64")) against the
FP64 oracle: every term, the LLG forms and the C1 1000-step trajectories.

The reference's CPU build computes in FP64, so an FP64 system on the device
follows its trajectories to rounding: fields within 1e-11 relative, and the
chaotic random-start C1 configuration within 1e-4 (the trajectory bar) after
1000 steps, where the FP32 state cannot (its rounding alone moves the
trajectory by 5e-5 to 7e-5).
"""
import json
import os

import numpy as np
import pytest

import oracle as O
from helpers import Pair, random_spins, rel_err, tilted_spins

pytestmark = pytest.mark.gpu

F64_FIELD_TOL = 1e-11
TRAJ_TOL = 1e-4
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "golden.json")


@pytest.fixture(scope="module")
def M():
    import maglua_b200 as M
    M.init(0)
    return M


def _fields(p, names):
    p.o.reset_fields()
    for f in p.oapply:
        f(p.o)
    p.o.sum_fields()
    p.g.resetFields()
    for op in p.ops:
        op.apply(p.g)
    p.g.sumFields()
    return {nm: rel_err(np.stack(p.g.fieldArrays(nm)), p.o.field(nm)) for nm in names}


def test_precision_reported_and_validated(M):
    ss = M.SpinSystem(4, 4, 1, precision="f64")
    assert ss.precision() == "f64"
    with pytest.raises(M.MagLuaError):
        M.SpinSystem(4, 4, 1, precision="f16")


def test_mixed_precision_llg_rejected(M):
    a = M.SpinSystem(4, 1, 1, precision="f64")
    b = M.SpinSystem(4, 1, 1)
    a.setSpinArrays(*random_spins(4, 1))
    b.setSpinArrays(*random_spins(4, 2))
    with pytest.raises(M.MagLuaError):
        M.LLG.new("Cartesian").apply(a, 1.0, a, b)


@pytest.mark.parametrize("dims,pbc", [((8, 7, 5), (1, 1, 1)), ((6, 5, 4), (1, 0, 0))])
def test_fp64_short_range_terms(M, dims, pbc):
    n = int(np.prod(dims))
    p = Pair(*dims, random_spins(n, 41, lengths=True), precision="f64")
    p.exchange(J=0.7, pbc=pbc)
    p.anisotropy(axis=(1, 2, 2), K=0.3)
    p.cubic(K=(0.05, 0.02, 0.01))
    p.zeeman((0.1, -0.2, 0.3))
    e = _fields(p, ["Exchange", "Anisotropy", "Zeeman", "Total"])
    assert max(e.values()) <= F64_FIELD_TOL, e


@pytest.mark.parametrize("dims", [(8, 8, 4), (16, 16, 1), (7, 5, 3)])
def test_fp64_dipole_reference_mode(M, dims):
    n = int(np.prod(dims))
    p = Pair(*dims, random_spins(n, 42, lengths=True), precision="f64")
    p.dipole(g=0.3)
    e = _fields(p, ["Dipole"])
    assert e["Dipole"] <= F64_FIELD_TOL, e


@pytest.mark.parametrize("dims", [(8, 8, 4), (7, 5, 3)])
def test_fp64_dipole_open_boundaries(M, dims):
    n = int(np.prod(dims))
    p = Pair(*dims, random_spins(n, 43, lengths=True), precision="f64")
    p.dipole(g=0.5, open_xy=True)
    e = _fields(p, ["Dipole"])
    assert e["Dipole"] <= F64_FIELD_TOL, e


def test_fp64_thermal_injected(M):
    dims = (6, 5, 2)
    s = random_spins(60, 44, lengths=True)
    p = Pair(*dims, s, alpha=0.2, dt=0.005, precision="f64")
    th = p.M.Thermal(*dims)
    th.setTemperature(0.5)
    noise = O.thermal_draw(p.o, 0.5, O.MT(99))
    th.inject(*noise)
    O.thermal_apply(p.o, 0.5, O.MT(99))
    th.apply(p.g)
    assert rel_err(np.stack(p.g.fieldArrays("Thermal")), p.o.field("Thermal")) <= F64_FIELD_TOL


@pytest.mark.parametrize("kind", ["Cartesian", "Quaternion"])
@pytest.mark.parametrize("tof", [True, False])
def test_fp64_llg_single_step(M, kind, tof):
    n = 200
    s = random_spins(n, 45, lengths=True)
    H = random_spins(n, 46) * 0.7
    Th = random_spins(n, 47) * 0.2
    o = O.SpinSystem(n, 1, 1)
    o.set_spins(*s)
    o.alpha, o.dt = 0.3, 0.02
    hv, tv = o.field_views("Total"), o.field_views("Thermal")
    for c in range(3):
        hv[c][:] = H[c]
        tv[c][:] = Th[c]
    O.LLG(kind, thermal_only_first_term=int(tof), precess_scale=0.9, damp_scale=1.1).apply(o, 1.5)
    g = M.SpinSystem(n, 1, 1, precision="f64")
    g.setSpinArrays(*s)
    g.setAlpha(0.3)
    g.setTimeStep(0.02)
    g.setFieldArrays("Total", *H)
    g.setFieldArrays("Thermal", *Th)
    l = M.LLG.new(kind)
    l.setThermalOnlyFirstTerm(tof)
    l.setUnphysicalPrecessionScale(0.9)
    l.setUnphysicalDampingScale(1.1)
    l.apply(g, 1.5, g, g)
    x, y, z, _ = g.spinArrays()
    assert np.abs(np.stack([x, y, z]) - o.spins()).max() <= 1e-13


def _c1(M, kind):
    from golden.make_golden import c1_spins, NX, NY, NZ, J, K, G, ALPHA, DT
    p = Pair(NX, NY, NZ, c1_spins(), alpha=ALPHA, dt=DT, precision="f64")
    p.exchange(J=J, paths=O.nn_paths(NX, NY, NZ, J=J, dirs=4))
    p.anisotropy(axis=(0, 0, 1), K=K)
    p.dipole(g=G)
    return p, M.LLG.new(kind)


def _golden():
    with open(GOLDEN) as f:
        return json.load(f)


def test_fp64_c1_fields_against_golden(M):
    gold = _golden()
    p, _ = _c1(M, "Cartesian")
    p.g.resetFields()
    for op in p.ops:
        op.apply(p.g)
    p.g.sumFields()
    for name in ("Exchange", "Anisotropy", "Dipole", "Total"):
        assert rel_err(np.stack(p.g.fieldArrays(name)), gold["c1_field_" + name]) <= F64_FIELD_TOL, name


@pytest.mark.parametrize("kind", ["Cartesian", "Quaternion"])
def test_fp64_c1_trajectory_1000_steps(M, kind):
    """The C1 configuration (32x32x1, exchange + anisotropy + dipole, random
    start) for 1000 steps, step by step for 100 and graph-captured for 900:
    max |dm| <= 1e-4 against the FP64 golden trajectory."""
    gold = _golden()
    p, l = _c1(M, kind)
    for _ in range(100):
        p.step_gpu(l)
    x, y, z, _ = p.g.spinArrays()
    err100 = np.abs(np.stack([x, y, z]) - np.array(gold[f"c1_{kind}_100"])).max()
    assert err100 <= 1e-9, err100
    M.run(p.g, p.ops, l, 900)
    x, y, z, _ = p.g.spinArrays()
    err = np.abs(np.stack([x, y, z]) - np.array(gold[f"c1_{kind}_1000"])).max()
    assert err <= TRAJ_TOL, err
    assert p.g.time() == pytest.approx(10.0, rel=1e-12)


@pytest.mark.parametrize("kind", ["Cartesian", "Quaternion"])
def test_fp64_smooth_trajectory_with_field(M, kind):
    dims = (12, 10, 3)
    n = int(np.prod(dims))
    p = Pair(*dims, tilted_spins(n, 48), alpha=0.05, dt=0.005, precision="f64")
    p.exchange(pbc=(1, 1, 0))
    p.anisotropy(K=0.05)
    p.zeeman((0.1, 0, 0))
    p.dipole(g=0.02)
    l = M.LLG.new(kind)
    lo = O.LLG(kind)
    M.run(p.g, p.ops, l, 300)
    for _ in range(300):
        p.step_oracle(lo)
    x, y, z, _ = p.g.spinArrays()
    assert np.abs(np.stack([x, y, z]) - p.o.spins()).max() <= 1e-10


def test_fp64_netmoment(M):
    n = 1000
    s = random_spins(n, 49, lengths=True)
    g = M.SpinSystem(n, 1, 1, precision="f64")
    g.setSpinArrays(*s)
    v = g.netMoment()
    assert v[0] == pytest.approx(s[0].sum(), rel=1e-13, abs=1e-12)
    assert v[2] == pytest.approx(s[2].sum(), rel=1e-13, abs=1e-12)
