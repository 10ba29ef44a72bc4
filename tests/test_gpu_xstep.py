"""The fused x pass of a step (inverse x transform of the dipole spectrum,
field terms + LLG update, forward x transform of the new spins in one
kernel) against the same step issued as the reference's individual calls
(M/cpu/core/spinsystem_luafuncs.lua resetFields / op:apply / sumFields,
M/cpu/llg/llg.cpp apply), which run the separate inverse-x, fused-step and
forward-x kernels.  Both orders perform the same float operations, so the
spins, the Total field and the Dipole slot must agree bitwise; so must every
path that invalidates the spectrum carried from one step to the next
(spins set from the host, an individual call in between, two systems
sharing one Dipole operator)."""
import numpy as np
import pytest

import oracle as O
from helpers import random_spins, tilted_spins

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def M():
    import maglua_b200 as M
    M.init(0)
    return M


def build(M, dims, spins, llg="Quaternion", T=0.5, ani=True, open_xy=False, dip_op=None):
    n = int(np.prod(dims))
    ss = M.SpinSystem(*dims)
    ss.setSpinArrays(*spins)
    ss.setAlpha(0.05)
    ss.setTimeStep(0.005)
    ex = M.Exchange(ss)
    ex.addPaths(*O.nn_paths(*dims, pbc=(0, 0, 0) if open_xy else (1, 1, 0)))
    ops = [ex]
    if ani:
        a = M.Anisotropy(ss)
        a.addMany(np.arange(n), np.tile([0, 0, 1.0], (n, 1)), np.full(n, 0.05))
        ops.append(a)
    if T > 0:
        th = M.Thermal(ss, M.Random.Philox(11))
        th.setTemperature(T)
        ops.append(th)
    z = M.AppliedField(ss)
    z.set(0.1, 0, 0.02)
    ops.append(z)
    dip = dip_op
    if dip is None:
        dip = M.Dipole(ss)
        dip.setStrength(0.03)
        if open_xy:
            dip.setOpen(True, True, True)
    ops.append(dip)
    return ss, ops, M.LLG.new(llg)


def calls(ss, ops, l, k):
    for _ in range(k):
        ss.resetFields()
        for op in ops:
            op.apply(ss)
        ss.sumFields()
        l.apply(ss)


def state(ss):
    return (np.stack(ss.spinArrays()[:3]), np.stack(ss.fieldArrays("Total")), np.stack(ss.fieldArrays("Dipole")))


def assert_same(a, b):
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


CASES = [
    # dims, llg, T, anisotropy, open in-plane
    ((64, 20, 3), "Quaternion", 0.5, True, False),     # 20 rows: a partial row band
    ((32, 16, 2), "Cartesian", 0.0, False, True),      # open x/y: padded x = 64
    ((128, 16, 1), "Cartesian", 0.5, True, False),
    ((256, 24, 2), "Quaternion", 0.0, True, False),
    ((512, 8, 2), "Quaternion", 0.5, False, False),
    ((96, 8, 2), "Quaternion", 0.5, True, False),      # x length without the fused pass
]


@pytest.mark.parametrize("dims,llg,T,ani,open_xy", CASES)
def test_run_equals_calls_bitwise(M, dims, llg, T, ani, open_xy):
    n = int(np.prod(dims))
    s0 = random_spins(n, 41)
    out = []
    for mode in ("calls", "run", "plan"):
        ss, ops, l = build(M, dims, s0, llg, T, ani, open_xy)
        if mode == "calls":
            calls(ss, ops, l, 7)
        elif mode == "run":
            M.run(ss, ops, l, 2)      # eager steps (below the capture threshold)
            M.run(ss, ops, l, 5)      # captured steps
        else:
            p = M.Plan(ss, ops, l)
            p.launch(3)
            p.launch(4)
        out.append(state(ss))
    assert_same(out[0], out[1])
    assert_same(out[0], out[2])


def test_carried_spectrum_invalidated_by_host_writes(M):
    dims = (64, 16, 2)
    n = int(np.prod(dims))
    s0 = tilted_spins(n, 42)
    res = []
    for mode in ("calls", "run"):
        ss, ops, l = build(M, dims, s0)
        step = (lambda k: calls(ss, ops, l, k)) if mode == "calls" else (lambda k: M.run(ss, ops, l, k))
        step(4)
        ss.setSpin((3, 5, 2), (0.6, 0.0, 0.8))
        step(4)
        x, y, z, _ = ss.spinArrays()
        ss.setSpinArrays(z, x, y)
        step(1)
        step(3)
        res.append(state(ss))
    assert_same(res[0], res[1])


def test_individual_calls_between_runs(M):
    dims = (128, 8, 2)
    n = int(np.prod(dims))
    s0 = random_spins(n, 43)
    res = []
    for mode in ("calls", "mixed"):
        ss, ops, l = build(M, dims, s0, llg="Cartesian")
        if mode == "calls":
            calls(ss, ops, l, 10)
        else:
            M.run(ss, ops, l, 4)
            calls(ss, ops, l, 2)
            p = M.Plan(ss, ops, l)
            p.launch(3)
            calls(ss, ops, l, 1)
        res.append(state(ss))
    assert_same(res[0], res[1])


def test_two_systems_share_one_dipole(M):
    dims = (64, 16, 2)
    n = int(np.prod(dims))
    sa, sb = random_spins(n, 44), tilted_spins(n, 45)
    res = []
    for mode in ("calls", "run"):
        dip = M.Dipole(*dims)
        dip.setStrength(0.03)
        A = build(M, dims, sa, dip_op=dip)
        B = build(M, dims, sb, dip_op=dip)
        for k in range(3):
            for ss, ops, l in (A, B):
                if mode == "calls":
                    calls(ss, ops, l, 3)
                else:
                    M.run(ss, ops, l, 3)
        res.append(state(A[0]) + state(B[0]))
    assert_same(res[0], res[1])


def test_run_matches_oracle(M):
    """The fused pass against the FP64 oracle (T = 0, 30 steps)."""
    dims = (64, 24, 2)
    n = int(np.prod(dims))
    s0 = tilted_spins(n, 46, deg=20.0)
    ss, ops, l = build(M, dims, s0, llg="Quaternion", T=0.0)
    M.run(ss, ops, l, 30)
    o = O.SpinSystem(*dims)
    o.set_spins(*s0)
    o.alpha, o.dt = 0.05, 0.005
    f, t, j = O.nn_paths(*dims, pbc=(1, 1, 0))
    sites = np.arange(n, dtype=np.int32)
    lr = O.LongRange(*dims, O.dipole_tensor(*dims))
    O.run_steps(o, 30, paths=(f, t, j), ani=(sites, np.tile([0, 0, 1.0], (n, 1)), np.full(n, 0.05)),
                B=(0.1, 0, 0.02), lr=lr, g=0.03, llg="Quaternion")
    err = float(np.abs(np.stack(ss.spinArrays()[:3]) - o.spins()).max())
    assert err < 2e-6, err


@pytest.mark.parametrize("dims,open_xy", [((32, 256, 4), False), ((16, 512, 2), False), ((8, 128, 3), True)])
def test_wide_plane_dipole_field(M, dims, open_xy):
    """Planes 256 and 512 wide (the register (y,z) kernel): dipole field
    against the oracle, reference-mode lattice sum or open direct sum."""
    from helpers import Pair
    n = int(np.prod(dims))
    p = Pair(*dims, random_spins(n, 47, lengths=True))
    p.dipole(g=0.4, open_xy=open_xy)
    p.o.reset_fields()
    for f in p.oapply:
        f(p.o)
    p.g.resetFields()
    for op in p.ops:
        op.apply(p.g)
    h = np.stack(p.g.fieldArrays("Dipole"))
    ref = p.o.field("Dipole")
    assert float(np.linalg.norm(h - ref) / np.linalg.norm(ref)) <= 1e-5


def test_wide_plane_steps_match_calls_and_oracle(M):
    dims = (32, 256, 4)
    n = int(np.prod(dims))
    s0 = tilted_spins(n, 48, deg=20.0)
    out = []
    for mode in ("calls", "run"):
        ss, ops, l = build(M, dims, s0, llg="Quaternion", T=0.0)
        if mode == "calls":
            calls(ss, ops, l, 6)
        else:
            M.run(ss, ops, l, 6)
        out.append(state(ss))
    assert_same(out[0], out[1])
    o = O.SpinSystem(*dims)
    o.set_spins(*s0)
    o.alpha, o.dt = 0.05, 0.005
    f, t, j = O.nn_paths(*dims, pbc=(1, 1, 0))
    sites = np.arange(n, dtype=np.int32)
    lr = O.LongRange(*dims, O.dipole_tensor(*dims))
    O.run_steps(o, 6, paths=(f, t, j), ani=(sites, np.tile([0, 0, 1.0], (n, 1)), np.full(n, 0.05)),
                B=(0.1, 0, 0.02), lr=lr, g=0.03, llg="Quaternion")
    assert float(np.abs(out[1][0] - o.spins()).max()) < 1e-6


@pytest.mark.parametrize("quirk,llg", [(True, "Quaternion"), (False, "Cartesian")])
def test_uniform_cubic_on_the_fused_pass(M, quirk, llg):
    """One uniform cubic axis set (M/cpu/anisotropy/..._cubic.cpp:308-390)
    on the fused fast kernels: individual calls and captured steps agree
    bitwise, a timed plan runs the fused x pass, and the trajectory follows
    the FP64 oracle."""
    from helpers import Pair
    dims = (64, 16, 4)
    n = int(np.prod(dims))
    s0 = tilted_spins(n, 49, deg=25.0)
    res = []
    for mode in ("calls", "run", "plan"):
        p = Pair(*dims, s0, alpha=0.1, dt=0.02)
        p.exchange(J=1.0, pbc=(1, 1, 0))
        p.cubic(K=(0.3, 0.1, 0.05), quirk=quirk)
        p.dipole(g=0.05)
        l = M.LLG.new(llg)
        if mode == "calls":
            for _ in range(10):
                p.step_gpu(l)
        elif mode == "run":
            M.run(p.g, p.ops, l, 10)
        else:
            plan = M.Plan(p.g, p.ops, l, timing=True)
            plan.launch(10)
            assert "k_xstep" in plan.kernelTimes()
        res.append(np.stack(p.g.spinArrays()[:3]))
    np.testing.assert_array_equal(res[0], res[1])
    np.testing.assert_array_equal(res[0], res[2])
    ol = O.LLG(llg)
    for _ in range(10):
        p.step_oracle(ol)
    err = float(np.abs(res[2] - p.o.spins()).max())
    assert err < 1e-5, err


def test_plan_after_spin_upload_matches_a_fresh_run(M):
    """mlb_system_upload_f32 of the spins alone (magnitudes kept) between plan
    launches: the captured step is reused (no new capture) and the run from
    the uploaded spins equals, bit for bit, a fresh system run from them."""
    dims = (64, 32, 4)
    n = int(np.prod(dims))
    s0 = tilted_spins(n, 51, deg=25.0)
    s1 = tilted_spins(n, 52, deg=35.0).astype(np.float32)
    ssA, opsA, lA = build(M, dims, s0, llg="Quaternion", T=0.0)
    ssA.setSpinArrays(*s0, np.ones(n))          # unit moments on both systems
    plan = M.Plan(ssA, opsA, lA)
    plan.launch(5)
    ssA.uploadF32(*[np.ascontiguousarray(s1[c]) for c in range(3)])
    plan.launch(7)
    ssB, opsB, lB = build(M, dims, s1.astype(np.float64), llg="Quaternion", T=0.0)
    ssB.setSpinArrays(*s1.astype(np.float64), np.ones(n))
    M.run(ssB, opsB, lB, 7)
    np.testing.assert_array_equal(np.stack(ssA.spinArrays()[:3]), np.stack(ssB.spinArrays()[:3]))
    np.testing.assert_array_equal(np.stack(ssA.fieldArrays("Total")), np.stack(ssB.fieldArrays("Total")))


def test_device_timeline_plan(M):
    """A timing=2 plan (device timeline of the fused (y,z) and x passes) steps
    exactly as a plain plan and reports both passes' spans per step; a plan
    without the timeline refuses deviceTimes."""
    dims = (256, 32, 4)
    n = int(np.prod(dims))
    s0 = random_spins(n, 61)
    out = []
    for timing in (False, 2):
        ss, ops, l = build(M, dims, s0, llg="Quaternion", T=0.5)
        p = M.Plan(ss, ops, l, timing=timing)
        spans = []
        for _ in range(4):
            p.launch(1)
            if timing == 2:
                spans.append(p.deviceTimes())
        out.append(state(ss))
        if timing == 2:
            for d in spans[1:]:
                assert set(d) == {"k_conv_yz", "k_xstep"}, d
                assert all(0.0 < v < 5e4 for v in d.values()), d
        else:
            with pytest.raises(M.MagLuaError):
                p.deviceTimes()
    assert_same(out[0], out[1])


def test_fields_after_spin_upload_are_the_steps_fields(M):
    """The fields of the last step (lazy records of the previous spin
    generation) read after a spins-only FP32 upload are, bit for bit, those
    read before it: the upload overwrites the current spin buffer only."""
    dims = (64, 32, 4)
    n = int(np.prod(dims))
    s0 = tilted_spins(n, 53, deg=25.0)
    s1 = tilted_spins(n, 54, deg=35.0).astype(np.float32)
    names = ("Total", "Exchange", "Anisotropy", "Thermal", "Dipole")
    out = []
    for upload in (False, True):
        ss, ops, l = build(M, dims, s0, llg="Quaternion", T=0.4)
        ss.setSpinArrays(*s0, np.ones(n))
        p = M.Plan(ss, ops, l)
        p.launch(3)
        if upload:
            ss.uploadF32(*[np.ascontiguousarray(s1[c]) for c in range(3)])
        out.append([np.stack(ss.fieldArrays(nm)) for nm in names])
        if upload:
            np.testing.assert_array_equal(np.stack(ss.spinArrays()[:3]), s1.astype(np.float64))
    for a, b in zip(*out):
        np.testing.assert_array_equal(a, b)


def test_async_net_moment_overlapping_steps(M):
    """netMomentAsync runs on a stream of its own next to the following steps
    (the next step writes the other spin buffer; the one after waits for the
    read): every step's moment equals the synchronous netMoment of the same
    step (up to the order of the FP64 additions: the side read runs on fewer
    blocks), and the trajectory is unchanged bit for bit."""
    dims = (128, 64, 4)
    n = int(np.prod(dims))
    s0 = tilted_spins(n, 55, deg=30.0)
    moments, spins = [], []
    for mode in ("async", "sync"):
        ss, ops, l = build(M, dims, s0, llg="Quaternion", T=0.3)
        ss.setSpinArrays(*s0, np.ones(n))
        p = M.Plan(ss, ops, l)
        got = []
        for k in range(12):
            p.launch(1)
            if mode == "async":
                ss.netMomentAsync(k % 4)
                if k >= 2:
                    got.append(ss.netMomentWait((k - 2) % 4))
            else:
                got.append(ss.netMoment())
        if mode == "async":
            for k in range(10, 12):
                got.append(ss.netMomentWait(k % 4))
        moments.append(np.array(got))
        spins.append(np.stack(ss.spinArrays()[:3]))
    np.testing.assert_allclose(moments[0], moments[1], rtol=1e-13, atol=1e-12)
    np.testing.assert_array_equal(spins[0], spins[1])
