"""Edge cases of the step: vacancies (sites with zero moment, which the
reference's operators and LLG skip), a single-site lattice, an x length
beyond the convolution kernels, and a step with no operators."""
import numpy as np
import pytest

import oracle as O
from helpers import Pair, random_spins, tilted_spins

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def M():
    import maglua_b200 as M
    M.init(0)
    return M


@pytest.mark.parametrize("llg", ["Cartesian", "Quaternion"])
def test_vacancies_follow_the_oracle(M, llg):
    dims = (24, 20, 3)
    n = int(np.prod(dims))
    s = tilted_spins(n, 94, deg=30.0)
    r = np.random.default_rng(95)
    vac = r.random(n) < 0.1
    s[:, vac] = 0.0
    p = Pair(*dims, s, alpha=0.1, dt=0.01)
    p.exchange(J=1.0, pbc=(1, 1, 0))
    p.anisotropy(axis=(0, 0, 1), K=0.1)
    p.zeeman((0.05, 0.0, 0.02))
    p.dipole(g=0.05)
    M.run(p.g, p.ops, M.LLG.new(llg), 20)
    ol = O.LLG(llg)
    for _ in range(20):
        p.step_oracle(ol)
    got = np.stack(p.g.spinArrays()[:3])
    assert np.all(got[:, vac] == 0.0)
    assert float(np.abs(got - p.o.spins()).max()) < 1e-5


def test_single_site_lattice(M):
    s = random_spins(1, 96)
    p = Pair(1, 1, 1, s, alpha=0.2, dt=0.02)
    p.exchange(J=1.0, pbc=(1, 1, 1))
    p.anisotropy(axis=(1, 0, 0), K=0.3)
    p.zeeman((0.0, 0.1, 0.0))
    p.dipole(g=0.1)
    ol = O.LLG("Quaternion")
    for _ in range(5):
        p.step_gpu(M.LLG.new("Quaternion"))
        p.step_oracle(ol)
    assert float(np.abs(np.stack(p.g.spinArrays()[:3]) - p.o.spins()).max()) < 1e-6


def test_x_length_beyond_the_kernels(M):
    ss = M.SpinSystem(8192, 1, 1)
    ss.setSpinArrays(*random_spins(8192, 97))
    dip = M.Dipole(ss)
    with pytest.raises(M.MagLuaError, match="x length too large"):
        dip.apply(ss)


def test_step_without_operators(M):
    dims = (16, 8, 2)
    n = int(np.prod(dims))
    s = tilted_spins(n, 98)
    ss = M.SpinSystem(*dims)
    ss.setSpinArrays(*s)
    ss.setTimeStep(0.01)
    M.run(ss, [], M.LLG.new("Quaternion"), 3)
    np.testing.assert_allclose(np.stack(ss.spinArrays()[:3]), s, atol=1e-7)
    assert ss.time() == pytest.approx(0.03)


@pytest.mark.parametrize("path", ["fused", "generic_f64", "eager_llg"])
def test_nonfinite_spin_sets_the_status_word(M, path):
    """A non-finite spin written by an LLG step sets bit 0 of the system's
    status word (mlb_system_status), on the fused fast kernels, the generic
    kernels and the stand-alone LLG; clearing resets it; a finite run leaves
    it clear.  The bad input is made on the host (one site set to NaN)."""
    dims = (16, 8, 2)
    n = int(np.prod(dims))
    prec = "f64" if path == "generic_f64" else "f32"

    def build(s0):
        ss = M.SpinSystem(*dims, precision=prec)
        ss.setSpinArrays(*s0, np.ones(n))     # uniform moments: the fast kernels take the fused step
        ss.setAlpha(0.1)
        ss.setTimeStep(0.01)
        if path == "generic_f64":
            ss.setSiteAlphaArray(np.full(n, 0.1))      # per-site alpha: the generic kernels
        ex = M.Exchange(ss)
        ex.addPaths(*O.nn_paths(*dims, pbc=(1, 1, 0)))
        dip = M.Dipole(ss)
        dip.setStrength(0.05)
        return ss, [ex, dip]

    def step(ss, ops, k):
        llg = M.LLG.new("Quaternion")
        if path == "eager_llg":
            for _ in range(k):
                ss.resetFields()
                for op in ops:
                    op.apply(ss)
                ss.sumFields()
                other = M.SpinSystem(*dims, precision=prec)
                ss.copyTo(other)
                llg.apply(other, 1.0, ss, ss)        # from != dmdt: the stand-alone LLG kernel
        else:
            M.run(ss, ops, llg, k)

    s0 = tilted_spins(n, 96, deg=20.0)
    ss, ops = build(s0)
    step(ss, ops, 3)
    assert ss.status() == 0
    bad = s0.copy()
    bad[0, 37] = np.nan
    ss2, ops2 = build(bad)
    step(ss2, ops2, 2)
    assert ss2.status() & 1
    assert ss2.status(clear=True) & 1
    assert ss2.status() == 0
