"""Runs checked against the oracle over many steps: thermal trajectories with
the reference's noise stream injected, the equilibrium magnetisation of
thermal runs with the device generator, and one replica of every size class
of the packed ensemble (16^3, 32x32x4, 48x48x2, 64x64x4; open boundaries,
dipole on, swept field) stepped against the oracle's open-boundary dipole.

References (M/ = src/modules/): Thermal::apply
M/cpu/thermal/spinoperationthermal.cpp:135-217 with the Mersenne Twister
stream of M/common/random/mersennetwister.h:182-300; the canonical step of
doc/manual/BasicMicromagneticSimulation.lua:84-94."""
import numpy as np
import pytest

import oracle as O
from helpers import rel_err, tilted_spins

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def M():
    import maglua_b200 as M
    M.init(0)
    return M


# ---------------------------------------------------------------- injected noise
# The 256x256x8 headline film's physics on a 16x16x2 film: periodic x/y,
# open z, J=1, K=0.05 along z, B=0.1 along x, g=0.02 (the reference's
# Dipole), T=0.5, alpha=0.05, dt=0.005, LLG.Quaternion.
FILM = (16, 16, 2)
T_FILM, ALPHA, DT, K_ANI, G_DIP, BX = 0.5, 0.05, 0.005, 0.05, 0.02, 0.1


def _film_product(M, dims, spins, precision, philox_seed=None):
    n = int(np.prod(dims))
    ss = M.SpinSystem(*dims, precision=precision)
    ss.setSpinArrays(*spins)
    ss.setAlpha(ALPHA)
    ss.setTimeStep(DT)
    ex = M.Exchange(ss)
    ex.addPaths(*O.nn_paths(*dims, pbc=(1, 1, 0)))
    ani = M.Anisotropy(ss)
    ani.addMany(np.arange(n), np.tile([0, 0, 1.0], (n, 1)), np.full(n, K_ANI))
    th = M.Thermal(ss, M.Random.Philox(philox_seed)) if philox_seed is not None else M.Thermal(ss)
    th.setTemperature(T_FILM)
    z = M.AppliedField(ss)
    z.set(BX, 0, 0)
    dip = M.Dipole(ss)
    dip.setStrength(G_DIP)
    return ss, [ex, ani, th, z, dip], M.LLG.new("Quaternion")


def _film_oracle(dims, spins):
    n = int(np.prod(dims))
    o = O.SpinSystem(*dims)
    o.set_spins(*spins)
    o.alpha, o.dt = ALPHA, DT
    cfg = dict(paths=O.nn_paths(*dims, pbc=(1, 1, 0)),
               ani=(np.arange(n, dtype=np.int32), np.tile([0, 0, 1.0], (n, 1)), np.full(n, K_ANI)),
               B=(BX, 0, 0), lr=O.LongRange(*dims, O.dipole_tensor(*dims)), g=G_DIP, llg="Quaternion")
    return o, cfg


@pytest.mark.parametrize("precision,steps,tol", [("f64", 200, 1e-9), ("f32", 200, 1e-4)])
def test_thermal_run_with_injected_reference_noise(M, precision, steps, tol):
    """Every step the product's Thermal takes the normals the reference's
    Mersenne Twister draws (the oracle draws them from the same seed in the
    same order); the trajectory follows the oracle's run_steps."""
    dims = FILM
    n = int(np.prod(dims))
    s0 = tilted_spins(n, 31, deg=25.0)
    o, cfg = _film_oracle(dims, s0)
    O.run_steps(o, steps, T=T_FILM, rng=O.MT(4242), **cfg)
    ss, ops, llg = _film_product(M, dims, s0, precision)
    th = ops[2]
    draw = O.SpinSystem(*dims)        # same moment lengths as the run: only the stream matters
    draw.set_spins(*s0)
    draw.alpha, draw.dt = ALPHA, DT
    rng = O.MT(4242)
    for _ in range(steps):
        th.inject(*O.thermal_draw(draw, T_FILM, rng))
        ss.resetFields()
        for op in ops:
            op.apply(ss)
        ss.sumFields()
        llg.apply(ss)
    got = np.stack(ss.spinArrays()[:3])
    err = float(np.abs(got - o.spins()).max())
    assert err <= tol, err
    assert abs(ss.time() - steps * DT) < 1e-9


# ---------------------------------------------------------------- equilibrium
EQ = (8, 8, 2)
EQ_REPLICAS = 16
EQ_BURN, EQ_EVERY, EQ_SAMPLES = 2000, 100, 40


def _stats(samples):
    """samples: (replicas, times, 3) of the net moment per site.  Per replica
    the time means of m_x, m_z and |m| and the time variance of m_z."""
    mx = samples[:, :, 0].mean(1)
    mz = samples[:, :, 2].mean(1)
    mm = np.linalg.norm(samples, axis=2).mean(1)
    vz = samples[:, :, 2].var(1)
    return {"m_x": mx, "m_z": mz, "|m|": mm, "var m_z": vz}


def test_thermal_equilibrium_matches_oracle(M):
    """Equilibrium of the headline film's physics at T = 0.5: the device's
    Philox noise against the oracle's Mersenne Twister runs.  Per quantity
    the replica means of both ensembles (16 independent seeded runs each,
    after a burn-in of 2000 steps, 40 samples 100 steps apart) agree within
    3 standard errors of their difference."""
    dims = EQ
    n = int(np.prod(dims))
    s0 = tilted_spins(n, 5, deg=5.0)
    orc, gpu = [], []
    for r in range(EQ_REPLICAS):
        o, cfg = _film_oracle(dims, s0)
        rng = O.MT(9000 + r)
        O.run_steps(o, EQ_BURN, T=T_FILM, rng=rng, **cfg)
        rows = []
        for _ in range(EQ_SAMPLES):
            O.run_steps(o, EQ_EVERY, T=T_FILM, rng=rng, **cfg)
            rows.append(o.netmoment()[:3] / n)
        orc.append(rows)
        ss, ops, llg = _film_product(M, dims, s0, "f32", philox_seed=7000 + r)
        M.run(ss, ops, llg, EQ_BURN)
        rows = []
        for _ in range(EQ_SAMPLES):
            M.run(ss, ops, llg, EQ_EVERY)
            rows.append(np.array(ss.netMoment()[:3]) / n)
        gpu.append(rows)
    a, b = _stats(np.array(orc)), _stats(np.array(gpu))
    for k in a:
        se = np.sqrt(a[k].var(ddof=1) / len(a[k]) + b[k].var(ddof=1) / len(b[k]))
        diff = abs(a[k].mean() - b[k].mean())
        assert diff <= 3 * se, (k, a[k].mean(), b[k].mean(), se)
    # the thermal state is neither saturated nor disordered at T = 0.5
    assert 0.3 < b["|m|"].mean() < 0.999


# ---------------------------------------------------------------- ensemble classes
CLASSES = [(16, 16, 16), (32, 32, 4), (48, 48, 2), (64, 64, 4)]
ENS = dict(alpha=0.1, dt=0.01, K=0.2, B=(0.0, 0.0, 0.0), dB=(0.0, 0.0, -0.5 / 20000), g=0.02)


def _ensemble_oracle(dims, s0, steps):
    n = int(np.prod(dims))
    o = O.SpinSystem(*dims)
    o.set_spins(*s0)
    o.alpha, o.dt = ENS["alpha"], ENS["dt"]
    paths = O.nn_paths(*dims, pbc=(0, 0, 0))
    sites = np.arange(n, dtype=np.int32)
    axes = np.tile([0, 0, 1.0], (n, 1))
    Ks = np.full(n, ENS["K"])
    D = O.DipoleOpen(*dims)
    llg = O.LLG("Cartesian")
    for k in range(steps):
        B = [ENS["B"][c] + k * ENS["dB"][c] for c in range(3)]
        o.reset_fields()
        O.exchange_apply(o, *paths)
        O.anisotropy_apply(o, sites, axes, Ks)
        O.zeeman_apply(o, B)
        D.apply(o, ENS["g"])
        o.sum_fields()
        llg.apply(o)
    return o.spins()


def test_ensemble_size_classes_match_oracle(M):
    """One replica of each size class in one packed ensemble (T = 0, open
    boundaries, dipole g = 0.02, B_z swept as in the benchmark, Cartesian
    LLG) against the oracle with the open-boundary dipole (O.DipoleOpen,
    itself equal to the direct sum): every replica within 1e-6 after one
    step and 1e-4 after 100."""
    starts = [tilted_spins(int(np.prod(d)), 60 + r, deg=20.0) for r, d in enumerate(CLASSES)]
    e = M.Ensemble(CLASSES)
    e.configure(alpha=ENS["alpha"], dt=ENS["dt"], J=1.0, pbc=(0, 0, 0), K=ENS["K"], axis=(0, 0, 1.0), T=0.0,
                B=ENS["B"], dB=ENS["dB"], g=ENS["g"], open_xy=True, llg="Cartesian")
    for r, s in enumerate(starts):
        e.setSpins(r, *s)
    e.run(1)
    for r, d in enumerate(CLASSES):
        err = float(np.abs(np.stack(e.spins(r)) - _ensemble_oracle(d, starts[r], 1)).max())
        assert err <= 1e-6, (d, err)
    e.run(99)
    for r, d in enumerate(CLASSES):
        err = float(np.abs(np.stack(e.spins(r)) - _ensemble_oracle(d, starts[r], 100)).max())
        assert err <= 1e-4, (d, err)


@pytest.mark.parametrize("dims", CLASSES)
def test_open_dipole_field_of_each_class_matches_oracle(M, dims):
    """The open-boundary Dipole field of each ensemble size class (the same
    passes the ensemble runs per class) within 1e-5 of the oracle's."""
    n = int(np.prod(dims))
    s = tilted_spins(n, 70, deg=40.0)
    ss = M.SpinSystem(*dims)
    ss.setSpinArrays(*s)
    dip = M.Dipole(ss)
    dip.setStrength(0.02)
    dip.setOpen(True, True, True)
    dip.apply(ss)
    got = np.stack(ss.fieldArrays("Dipole"))
    assert rel_err(got, O.DipoleOpen(*dims).field(s, 0.02)) <= 1e-5
