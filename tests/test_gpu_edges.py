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
