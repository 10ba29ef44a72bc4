"""SpinSystem encode / decode: the byte stream of the reference's CPU build
(spinsystem.cpp:669-851, luabaseobject.cpp:142-360), compared byte for byte
with the oracle's restatement, decoded back, and resumed from."""
import struct

import numpy as np
import pytest

import oracle as O
from helpers import random_spins

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def M():
    import maglua_b200 as M
    M.init(0)
    return M


def _state(M, dims, precision, seed, uniform_ms=False, site=False):
    n = int(np.prod(dims))
    s = random_spins(n, seed)
    r = np.random.default_rng(seed + 1)
    ms = np.full(n, 1.5) if uniform_ms else 0.5 + r.random(n)
    ss = M.SpinSystem(*dims, precision=precision)
    ss.setSpinArrays(s[0] * ms, s[1] * ms, s[2] * ms, ms)
    ss.setAlpha(0.125)
    ss.setTimeStep(0.01)
    ss.setGamma(1.75)
    ss.setTime(3.5)
    sa = sg = None
    if site:
        sa = 0.05 + 0.1 * r.random(n)
        sg = 1.0 + r.random(n)
        ss.setSiteAlphaArray(sa)
        ss.setSiteGammaArray(sg)
        if precision == "f32":
            sa, sg = sa.astype(np.float32).astype(np.float64), sg.astype(np.float32).astype(np.float64)
    return ss, sa, sg


def _oracle_stream(ss, sa=None, sg=None):
    x, y, z, ms = ss.spinArrays()
    nx, ny, nz = ss._dims
    return O.encode_spinsystem(nx, ny, nz, ss.alpha(), ss.timeStep(), ss.gamma(), ss.time(), x, y, z, ms, sa, sg)


@pytest.mark.parametrize("precision", ["f32", "f64"])
@pytest.mark.parametrize("uniform_ms,site", [(False, False), (True, False), (False, True)])
def test_encode_matches_the_oracle_bytes(M, precision, uniform_ms, site):
    ss, sa, sg = _state(M, (12, 10, 3), precision, 11, uniform_ms, site)
    got = ss.encode()
    assert got == _oracle_stream(ss, sa, sg)
    assert ss._stream_objects == (7 if site else 5)
    d = O.decode_spinsystem(got)
    assert (d["nx"], d["ny"], d["nz"]) == (12, 10, 3)
    assert (d["alpha"], d["dt"], d["gamma"], d["time"]) == (0.125, 0.01, 1.75, 3.5)
    # one value for a uniform array (flag 1), else every site
    n = 12 * 10 * 3
    arrays = 6 if site else 4
    full = arrays - (1 if uniform_ms else 0)
    header = 4 + 4 + 1 + 4
    arr_head = header + 1 + 12 + 4
    expect = header + 1 + 12 + 32 + arrays * arr_head + full * 8 * n + (arrays - full) * 8 + 4 + 4 + 4
    assert len(got) == expect


def test_decode_restores_the_state_exactly(M):
    n = 9 * 7 * 2
    s = random_spins(n, 21)
    r = np.random.default_rng(22)
    ms = 0.5 + r.random(n)
    sa = 0.02 + 0.1 * r.random(n)
    data = O.encode_spinsystem(9, 7, 2, 0.3, 0.005, 1.1, 12.25, s[0] * ms, s[1] * ms, s[2] * ms, ms, sa, None)
    ss = M.SpinSystem.decode(data, precision="f64")
    assert ss._dims == (9, 7, 2)
    assert (ss.alpha(), ss.timeStep(), ss.gamma(), ss.time()) == (0.3, 0.005, 1.1, 12.25)
    x, y, z, m = ss.spinArrays()
    assert np.array_equal(x, s[0] * ms) and np.array_equal(y, s[1] * ms) and np.array_equal(z, s[2] * ms)
    assert np.array_equal(m, ms)
    # decode then encode gives the same bytes back
    assert ss.encode() == data
    # into FP32 state: the values rounded to float
    s32 = M.SpinSystem.decode(data, precision="f32")
    assert np.array_equal(s32.spinArrays()[0], (s[0] * ms).astype(np.float32).astype(np.float64))


def test_decode_accepts_all_nil_extra_data_and_refuses_values(M):
    n = 4 * 4 * 1
    s = random_spins(n, 31)
    base = O.encode_spinsystem(4, 4, 1, 1.0, 0.01, 1.0, 0.0, s[0], s[1], s[2], np.ones(n))
    # "all sites" form (-1) with nil at every site
    nil_all = base[:-4] + struct.pack("=i", -1) + struct.pack("=%di" % n, *([O.LUA_TNIL] * n))
    ss = M.SpinSystem.decode(nil_all, precision="f64")
    assert np.array_equal(ss.spinArrays()[0], s[0])
    # a site with a Lua number: not held by this library
    one = base[:-4] + struct.pack("=ii", 1, 3) + struct.pack("=id", 3, 2.0)
    with pytest.raises(M.MagLuaError, match="extra data"):
        M.SpinSystem.decode(one)


def test_decode_rejects_malformed_streams(M):
    n = 3 * 3 * 1
    s = random_spins(n, 41)
    data = O.encode_spinsystem(3, 3, 1, 1.0, 0.01, 1.0, 0.0, s[0], s[1], s[2], np.ones(n))
    with pytest.raises(M.MagLuaError, match="ends early"):
        M.SpinSystem.decode(data[:-9])
    with pytest.raises(M.MagLuaError, match="trailing"):
        M.SpinSystem.decode(data + b"\0")
    bad = bytearray(data)
    bad[4:8] = struct.pack("=i", O.type_hash32("Array.Double"))
    with pytest.raises(M.MagLuaError, match="SpinSystem"):
        M.SpinSystem.decode(bytes(bad))


def test_resume_from_a_checkpoint_follows_the_same_trajectory(M):
    dims = (32, 32, 4)
    n = int(np.prod(dims))
    ss = M.SpinSystem(*dims, precision="f64")
    ss.setSpinArrays(*random_spins(n, 51))
    ss.setAlpha(0.1)
    ss.setTimeStep(0.01)

    f, t, j = O.nn_paths(*dims, J=1.0, pbc=(1, 1, 0))

    def ops():
        ex = M.Exchange(*dims)
        ex.addPaths(f, t, j)
        ani = M.Anisotropy(*dims)
        ani.addMany(np.arange(n, dtype=np.int32), np.tile([0.0, 0.0, 1.0], (n, 1)), np.full(n, 0.2))
        dip = M.Dipole(*dims)
        dip.setStrength(0.05)
        return [ex, ani, dip]

    llg = M.LLG.new("Quaternion")
    M.run(ss, ops(), llg, 10)
    data = ss.encode()
    resumed = M.SpinSystem.decode(data, precision="f64")
    assert resumed.time() == ss.time()
    M.run(ss, ops(), llg, 15)
    M.run(resumed, ops(), llg, 15)
    assert ss.diff(resumed)[3] == 0.0
    assert resumed.time() == ss.time()


def test_stream_inside_a_larger_checkpoint(M):
    """The system as the fourth object of a stream (object indices 3..7) and
    followed by more data: decode reads it and reports the bytes used."""
    ss, _, _ = _state(M, (6, 5, 2), "f64", 71)
    own = ss.encode()
    inner = ss.encode(first_index=3)
    assert len(inner) == len(own) and inner != own
    assert inner == _oracle_stream_at(ss, 3)
    tail = struct.pack("=id", 3, 42.0)
    got, used, nobj = M.SpinSystem.decode(inner + tail, precision="f64", partial=True)
    assert used == len(inner) and nobj == 5 and ss._stream_objects == 5
    assert got.encode(first_index=3) == inner
    with pytest.raises(M.MagLuaError, match="trailing"):
        M.SpinSystem.decode(inner + tail, precision="f64")


def _oracle_stream_at(ss, first):
    x, y, z, ms = ss.spinArrays()
    nx, ny, nz = ss._dims
    return O.encode_spinsystem(nx, ny, nz, ss.alpha(), ss.timeStep(), ss.gamma(), ss.time(), x, y, z, ms,
                               first_index=first)


def test_checkpoint_of_operators_and_llg_resumes_the_run(M):
    """A whole script state -- the SpinSystem, Exchange, Anisotropy,
    Anisotropy.Cubic, AppliedField, Dipole and the LLG -- encoded into one
    stream (object indices running on), decoded into new objects, and the run
    resumed from them: the same trajectory bit for bit as the run continued
    in place (M/cpu/exchange/spinoperationexchange.cpp:52-112,
    spinoperationanisotropy.cpp:191-236, ..._cubic.cpp:239-290,
    spinoperationappliedfield.cpp:33-58, spinoperationdipole.cpp:35-59,
    llg.cpp:50-88)."""
    dims = (16, 8, 2)
    n = int(np.prod(dims))
    ss = M.SpinSystem(*dims)
    ss.setSpinArrays(*random_spins(n, 91))
    ss.setAlpha(0.1)
    ss.setTimeStep(0.01)
    ex = M.Exchange(ss)
    ex.setPeriodicXYZ(True, True, False)
    ex.addPaths(*O.nn_paths(*dims, pbc=(1, 1, 0)))
    ani = M.Anisotropy(ss)
    r = np.random.default_rng(4)
    ani.addMany(np.arange(n), r.normal(size=(n, 3)), r.uniform(0.0, 0.2, n))
    cub = M.AnisotropyCubic(ss)
    cub.addMany(np.arange(n), np.tile([1.0, 0, 0], (n, 1)), np.tile([0, 1.0, 0], (n, 1)),
                np.tile([0.05, 0.01, 0.0], (n, 1)))
    z = M.AppliedField(ss)
    z.set(0.02, 0.0, -0.05)
    dip = M.Dipole(ss)
    dip.setStrength(0.04)
    llg = M.LLG.new("Quaternion")
    ops = [ex, ani, cub, z, dip]
    M.run(ss, ops, llg, 5)
    stream = bytearray()
    idx = 0
    objs = [ss] + ops + [llg]
    for o in objs:
        b = o.encode(idx)
        idx += o._stream_objects
        stream += b
    pos = 0
    back = []
    s2, used, k = M.SpinSystem.decode(bytes(stream), partial=True)
    pos += used
    for _ in range(len(ops) + 1):
        o, used, k = M.decode(bytes(stream[pos:]), partial=True)
        back.append(o)
        pos += used
    assert pos == len(stream)
    assert [type(o).__name__ for o in back] == ["Exchange", "Anisotropy", "AnisotropyCubic", "AppliedField",
                                                "Dipole", "LLGQuaternion"]
    assert back[0].periodicXYZ() == (True, True, False)
    M.run(ss, ops, llg, 20)
    M.run(s2, back[:-1], back[-1], 20)
    np.testing.assert_array_equal(np.stack(ss.spinArrays()[:3]), np.stack(s2.spinArrays()[:3]))
    assert ss.time() == s2.time()
