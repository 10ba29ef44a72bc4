"""DipoleEwald3D (M/cpu/ewald3d) on the GPU: every element of a sheared
6 x 5 x 4 lattice computed one thread per element in FP64 against the
library's host elements (the path checked against the oracle's restatement
of ewald3d.cpp on the CPU) and the trace identity of the Ewald sum; the
tensor fed into LongRange3D as make_tensor.lua does (-G) against the FP64
oracle's LongRange3D."""
import numpy as np
import pytest

import oracle as O
from helpers import random_spins, rel_err

pytestmark = pytest.mark.gpu

AB = ["XX", "XY", "XZ", "YX", "YY", "YZ", "ZX", "ZY", "ZZ"]
SHEARED = [[1, 0, 0], [0.5, 0.8, 0], [0.1, 0.2, 0.9]]


@pytest.fixture(scope="module")
def M():
    import maglua_b200 as M
    M.init(0)
    return M


def test_ewald_tensor_on_the_gpu(M):
    dims = (6, 5, 4)
    nx, ny, nz = dims
    ew = M.DipoleEwald3D(*dims)
    ew.setUnitCell(*SHEARED)
    ew.setNSites(6)
    T = ew.tensorArrays()
    scale = max(np.abs(T[ab]).max() for ab in AB)
    r = np.random.default_rng(92)
    sites = [(0, 0, 0), (nx - 1, ny - 1, nz - 1)] + [tuple(int(v) for v in r.integers(0, (nx, ny, nz))) for _ in range(6)]
    for (x, y, z) in sites:
        for ab in AB:
            host = ew.calculateTensorElement(ab, (x, y, z))
            assert abs(T[ab][z, y, x] - host) <= 1e-12 * scale, (ab, x, y, z)
    # trace = -4 pi / V away from the lattice point at the origin
    tr = T["XX"] + T["YY"] + T["ZZ"]
    off = np.ones_like(tr, dtype=bool)
    off[0, 0, 0] = False
    np.testing.assert_allclose(tr[off], -4 * np.pi / ew.volume(), rtol=1e-7)
    assert ew.eta() > 0


def test_ewald_tensor_through_longrange3d(M):
    dims = (6, 5, 4)
    nx, ny, nz = dims
    ew = M.DipoleEwald3D(*dims)
    ew.setUnitCell(*SHEARED)
    ew.setNSites(4)
    T = ew.tensorArrays()
    s = random_spins(nx * ny * nz, 93)
    ss = M.SpinSystem(*dims)
    ss.setSpinArrays(*s)
    lr = M.LongRange3D(ss)
    T9 = [-T[ab] for ab in AB]
    for q, ab in enumerate(AB):
        lr.setTensorArray(ab, T9[q])
    lr.setStrength(0.6)
    lr.apply(ss)
    o = O.SpinSystem(*dims)
    o.set_spins(*s)
    O.longrange3d_apply(o, T9, 0.6)
    assert rel_err(np.stack(ss.fieldArrays("LongRange3D")), o.field("LongRange3D")) <= 1e-5
