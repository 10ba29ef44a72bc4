"""Runge-Kutta integrators (mlb_rk_*) against the reference script they
replace, M/common/scripts/RungeKutta.lua:57-215 (make_rk_step_function and
its step function), restated below in Python over the FP64 oracle's own
operators and LLG (llg:apply(src, factor, dmdt, dst) with the reference's
argument meaning).  Fields ≤ 1e-5, so a short FP32 trajectory stays within
1e-5 of the FP64 one; the time bookkeeping must agree exactly."""
import numpy as np
import pytest

import oracle as O
from helpers import Pair, tilted_spins

pytestmark = pytest.mark.gpu

# RungeKutta.lua:100-158 (the c column is not used by the script)
BUTCHER = {
    "RK1": [[1.0]],
    "RK2": [[0.5], [0.0, 1.0]],
    "K3": [[0.5], [-1.0, 2.0], [1 / 6, 2 / 3, 1 / 6]],
    "RK4": [[0.5], [0.0, 0.5], [0.0, 0.0, 1.0], [1 / 6, 1 / 3, 1 / 3, 1 / 6]],
    "RK3": [[1 / 3], [0.0, 2 / 3], [0.25, 0.0, 0.75]],
    "RK4_38": [[1 / 3], [-1 / 3, 1.0], [1.0, -1.0, 1.0], [1 / 8, 3 / 8, 3 / 8, 1 / 8]],
    "RK6": [[1 / 3], [0.0, 2 / 3], [1 / 12, 4 / 12, -1 / 12], [-1 / 16, 18 / 16, -3 / 16, -6 / 16],
            [0.0, 9 / 8, -3 / 8, -6 / 8, 4 / 8], [9 / 44, -36 / 44, 63 / 44, 72 / 44, 0.0, -64 / 44],
            [11 / 120, 0.0, 81 / 120, 81 / 120, -32 / 120, -32 / 120, 11 / 120]],
    "BS3": [[0.5], [0.0, 0.75], [2 / 9, 1 / 3, 4 / 9], [7 / 24, 0.25, 1 / 3, 1 / 8]],
}


@pytest.fixture(scope="module")
def M():
    import maglua_b200 as M
    M.init(0)
    return M


def oracle_copy(o):
    c = O.SpinSystem(o.nx, o.ny, o.nz)
    c.set_spins(*o.spins())
    c.alpha, c.gamma, c.dt, c.time = o.alpha, o.gamma, o.dt, o.time
    return c


def oracle_rk_steps(p, kind, llg, nsteps):
    """make_rk_step_function(ss, kind, field, llg) and nsteps calls of the
    step function, on the oracle system p.o."""
    bt = BUTCHER[kind]
    nstep = len(bt)
    ss = p.o
    k = [ss] + [oracle_copy(ss) for _ in range(nstep - 1)]

    def field(s):
        s.reset_fields()
        for f in p.oapply:
            f(s)
        s.sum_fields()

    def istep(src, factors, dst):
        llg.apply(src, factors[0], src, dst)
        for i in range(2, nstep + 1):
            if i <= len(factors) and factors[i - 1] != 0:
                llg.apply(dst, factors[i - 1], k[i - 1], dst)

    for _ in range(nsteps):
        field(ss)
        for i in range(1, nstep):
            k[i].dt = ss.dt
            istep(ss, bt[i - 1], k[i])
            field(k[i])
        istep(ss, bt[nstep - 1], ss)


@pytest.mark.parametrize("kind,llg", [("RK1", "Cartesian"), ("RK2", "Quaternion"), ("K3", "Cartesian"),
                                      ("RK3", "Quaternion"), ("RK4", "Quaternion"), ("RK4", "Cartesian"),
                                      ("RK4_38", "Cartesian"), ("RK6", "Quaternion"), ("BS3", "Quaternion")])
def test_rk_matches_oracle(M, kind, llg):
    dims = (16, 12, 2)
    n = int(np.prod(dims))
    s0 = tilted_spins(n, 70, deg=25.0)
    p = Pair(*dims, s0, alpha=0.1, dt=0.02)
    p.exchange(J=1.0, pbc=(1, 1, 0))
    p.anisotropy(axis=(0, 0, 1), K=0.1)
    p.zeeman((0.05, 0.0, 0.02))
    p.dipole(g=0.05)
    rk = M.RungeKutta(p.g, kind, p.ops, M.LLG.new(llg))
    rk.step(4)
    rk.step(6)
    oracle_rk_steps(p, kind, O.LLG(llg), 10)
    got = np.stack(p.g.spinArrays()[:3])
    err = float(np.abs(got - p.o.spins()).max())
    assert err < 1e-5, err
    assert p.g.time() == pytest.approx(p.o.time, rel=1e-12, abs=1e-12)


def test_rk_thermal_kick_keeps_unit_spins(M):
    """The optional thermal step (RungeKutta.lua:206-211): llg:apply(ss, false)
    after the stages leaves the time unadvanced by the kick and the spins
    normalised."""
    dims = (32, 16, 1)
    n = int(np.prod(dims))
    out = []
    for T in (0.2, None):
        ss = M.SpinSystem(*dims)
        ss.setSpinArrays(*tilted_spins(n, 71))
        ss.setAlpha(0.1)
        ss.setTimeStep(0.01)
        ex = M.Exchange(ss)
        ex.addPaths(*O.nn_paths(*dims, pbc=(1, 1, 1)))
        th = None
        if T is not None:
            th = M.Thermal(ss, M.Random.Philox(3))
            th.setTemperature(T)
        rk = M.RungeKutta(ss, "RK4", [ex], M.LLG.new("Quaternion"), temp=th)
        rk.step(20)
        x, y, z, _ = ss.spinArrays()
        assert np.allclose(np.sqrt(x * x + y * y + z * z), 1.0, atol=1e-5)
        assert ss.time() == pytest.approx(20 * 0.01, rel=1e-12)
        out.append(np.stack([x, y, z]))
    assert np.abs(out[0] - out[1]).max() > 1e-3   # the kicks moved the spins


def test_rk_rejects_unknown_scheme(M):
    ss = M.SpinSystem(4, 4, 1)
    with pytest.raises(M.MagLuaError, match="RK type must be one of"):
        M.RungeKutta(ss, "RK5", [], M.LLG.new("Cartesian"))


class OracleRK:
    """The script's step function sfunc(ss_input) on the oracle: stage copies
    made once from the base system (RungeKutta.lua:182-185)."""

    def __init__(self, p, kind, llg):
        self.p, self.bt, self.llg = p, BUTCHER[kind], llg
        self.k = [None] + [oracle_copy(p.o) for _ in range(len(self.bt) - 1)]

    def field(self, s):
        s.reset_fields()
        for f in self.p.oapply:
            f(s)
        s.sum_fields()

    def __call__(self, ss):
        bt, nstep, llg = self.bt, len(self.bt), self.llg
        k = [ss] + self.k[1:]

        def istep(src, factors, dst):
            llg.apply(src, factors[0], src, dst)
            for i in range(2, nstep + 1):
                if i <= len(factors) and factors[i - 1] != 0:
                    llg.apply(dst, factors[i - 1], k[i - 1], dst)

        self.field(ss)
        for i in range(1, nstep):
            k[i].dt = ss.dt
            istep(ss, bt[i - 1], k[i])
            self.field(k[i])
        istep(ss, bt[nstep - 1], ss)


def test_diff_and_copy_spins(M):
    dims = (12, 10, 3)
    n = int(np.prod(dims))
    from helpers import random_spins
    a, b = M.SpinSystem(*dims), M.SpinSystem(*dims)
    sa, sb = random_spins(n, 72), random_spins(n, 73)
    a.setSpinArrays(*sa)
    b.setSpinArrays(*sb)
    b.setAlpha(0.3)
    b.setTimeStep(0.07)
    b.setTime(1.5)
    ga = np.stack(a.spinArrays()[:3])
    gb = np.stack(b.spinArrays()[:3])
    d = np.abs(ga - gb).sum(axis=1)
    got = a.diff(b)
    np.testing.assert_allclose(got[:3], d, rtol=1e-12)
    assert got[3] == pytest.approx(np.sqrt((d ** 2).sum()), rel=1e-12)
    # copySpinsTo (copySpinsFrom, spinsystem.cpp:393-409): spins and magnitudes only
    a.copySpinsTo(b)
    np.testing.assert_array_equal(np.stack(b.spinArrays()), np.stack(a.spinArrays()))
    assert (b.alpha(), b.timeStep(), b.time()) == (0.3, 0.07, 1.5)
    assert a.diff(b)[3] == 0.0


@pytest.mark.parametrize("kind,tol", [("RK2", 2e-3), ("RK4", 1e-4)])
def test_adaptive_time_step_matches_oracle(M, kind, tol):
    """make_adapt_step_function (AdaptiveTimeStep.lua:9-110) natively against
    the script restated over the oracle: the accept/reject sequence, the time
    steps and the trajectory."""
    dims = (16, 12, 2)
    n = int(np.prod(dims))
    s0 = tilted_spins(n, 74, deg=30.0)
    p = Pair(*dims, s0, alpha=0.2, dt=0.08)
    p.exchange(J=1.0, pbc=(1, 1, 0))
    p.anisotropy(axis=(0, 0, 1), K=0.2)
    p.dipole(g=0.05)
    rk = M.RungeKutta(p.g, kind, p.ops, M.LLG.new("Quaternion"))
    ad = M.AdaptiveTimeStep(p.g, rk, tol)
    got = []
    for _ in range(12):
        got.append((ad.step(), p.g.timeStep(), p.g.time()))
    # oracle
    o = p.o
    step = OracleRK(p, kind, O.LLG("Quaternion"))
    s2, s3 = oracle_copy(o), oracle_copy(o)
    ref = []
    for _ in range(12):
        s2.time = s3.time = o.time
        s2.dt, s3.dt = o.dt, o.dt / 2
        s2.set_spins(*o.spins())
        s3.set_spins(*o.spins())
        step(s2)
        step(s3)
        step(s3)
        d = np.abs(s2.spins() - s3.spins()).sum(axis=1)
        dxyz = float(np.sqrt((d ** 2).sum()))
        same = dxyz < tol
        ee = (tol - dxyz) / tol
        if same:
            o.set_spins(*s3.spins())
            o.time = s3.time
            ee = min(max(ee * ee, 0.1), 0.5)
            o.dt = o.dt * (1 + ee - 0.1)
        else:
            o.dt = o.dt * 0.5
        ref.append((same, o.dt, o.time))
    assert [g[0] for g in got] == [r[0] for r in ref], (got, ref)
    assert any(not r[0] for r in ref) and any(r[0] for r in ref)   # both branches taken
    for g, r in zip(got, ref):
        assert g[1] == pytest.approx(r[1], rel=1e-4)
        assert g[2] == pytest.approx(r[2], rel=1e-4, abs=1e-9)
    err = float(np.abs(np.stack(p.g.spinArrays()[:3]) - o.spins()).max())
    assert err < 2e-5, err


@pytest.mark.parametrize("kind,llg", [("RK4", "Quaternion"), ("RK2", "Cartesian"), ("RK6", "Quaternion")])
def test_rk_graph_steps_equal_eager_steps(M, kind, llg):
    """Steps run as graphs (the same kernels and arguments recorded with their
    dependent-launch edges) leave the spins, the stage systems' effect and the
    time exactly as eager steps do, through a parameter change in between
    (which runs that step eagerly)."""
    dims = (64, 32, 4)
    n = int(np.prod(dims))
    s0 = tilted_spins(n, 72, deg=20.0)
    res = []
    for graph in (False, True):
        ss = M.SpinSystem(*dims)
        ss.setSpinArrays(*s0)
        ss.setAlpha(0.05)
        ss.setTimeStep(0.005)
        ex = M.Exchange(ss)
        ex.addPaths(*O.nn_paths(*dims, pbc=(1, 1, 0)))
        ani = M.Anisotropy(ss)
        ani.addMany(np.arange(n), np.tile([0, 0, 1.0], (n, 1)), np.full(n, 0.05))
        z = M.AppliedField(ss)
        z.set(0.1, 0.0, 0.02)
        dip = M.Dipole(ss)
        dip.setStrength(0.03)
        th = M.Thermal(ss, M.Random.Philox(5))
        th.setTemperature(0.3)
        rk = M.RungeKutta(ss, kind, [ex, ani, z, dip], M.LLG.new(llg), temp=th)
        rk.setGraph(graph)
        rk.step(5)
        th.setTemperature(0.2)
        rk.step(5)
        res.append((np.stack(ss.spinArrays()[:3]), ss.time(), rk.graphSteps()))
    np.testing.assert_array_equal(res[0][0], res[1][0])
    assert res[0][1] == res[1][1]
    assert res[0][2] == 0 and res[1][2] >= 6, (res[0][2], res[1][2])
