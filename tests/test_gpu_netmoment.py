"""netMoment (the scaled sums of the spin components and of their squares)
read without waiting: the asynchronous slots return what the synchronous
call returns for the same spins (up to the order of the FP64 additions: a
slot's read runs on fewer blocks), also when the next step is already
queued, and the FP64 oracle's sums."""
import numpy as np
import pytest

import oracle as O
from helpers import tilted_spins

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def M():
    import maglua_b200 as M
    M.init(0)
    return M


def test_netmoment_async_slots(M):
    dims = (64, 32, 4)
    n = int(np.prod(dims))
    s0 = tilted_spins(n, 91, deg=30.0)
    ss = M.SpinSystem(*dims)
    ss.setSpinArrays(*s0)
    ss.setAlpha(0.1)
    ss.setTimeStep(0.01)
    ex = M.Exchange(ss)
    ex.addPaths(*O.nn_paths(*dims, pbc=(1, 1, 0)))
    llg = M.LLG.new("Quaternion")
    plan = M.Plan(ss, [ex], llg)
    sync = []
    asyn = []
    for k in range(6):
        plan.launch(1)
        sync.append(ss.netMoment(0.5))
        ss.netMomentAsync(k & 1, 0.5)
        if k:
            asyn.append(ss.netMomentWait((k - 1) & 1))
    asyn.append(ss.netMomentWait(1))
    np.testing.assert_allclose(np.asarray(asyn), np.asarray(sync), rtol=1e-13, atol=1e-12)
    x, y, z, _ = ss.spinArrays()
    o = O.SpinSystem(*dims)
    o.set_spins(x, y, z)
    np.testing.assert_allclose(np.asarray(sync[-1]), o.netmoment(0.5), rtol=1e-9, atol=1e-9)
    with pytest.raises(M.MagLuaError, match="no netMoment enqueued"):
        ss.netMomentWait(0)
    with pytest.raises(M.MagLuaError, match="slot must be 0..3"):
        ss.netMomentAsync(4)
