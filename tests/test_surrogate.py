"""Learned dipolar surrogate (no reference counterpart): the tcgen05 BF16
forward and the FP32 training kernels against the FP64 CPU reference of the
network (oracle/surrogate.py), online training on pairs from the plain
method, what the trained network gains over holding the field between exact
evaluations (and, on the surrogate configuration's film, its field error
against the FP64 field within 1e-3), and the captured run with its exact
schedule and residual check.

Tolerances: the stencil branch with BF16-representable inputs and weights is
exact up to FP32 accumulation (1e-5); the spectral branch rounds its DFT rows
and mixed spectrum to BF16 (2e-2); the stencil gradient is FP32 (1e-4); the
mode gradient uses a BF16 transform of G (2e-2).
"""
import numpy as np
import pytest

from oracle import surrogate as OS
from helpers import random_spins, rel_err


def crel(a, b):
    return rel_err(np.stack([np.real(a), np.imag(a)]), np.stack([np.real(b), np.imag(b)]))

pytestmark = pytest.mark.gpu

DIMS = (128, 16, 2)
N = DIMS[0] * DIMS[1] * DIMS[2]
C = 3 * DIMS[2]
MODES = (8, 8)
RAD = 2


@pytest.fixture(scope="module")
def M():
    import maglua_b200 as M
    M.init(0)
    return M


def bf16(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def _sur(M, dims=DIMS, modes=MODES, radius=RAD):
    d = M.Dipole(*dims)
    d.setStrength(0.05)
    return M.Surrogate(d, modes, radius), d


def _random_params(seed, scale_w=0.1, scale_r=0.3):
    r = np.random.default_rng(seed)
    W = r.normal(size=((2 * RAD + 1) ** 2, C, C)) * scale_w
    R = (r.normal(size=(MODES[0], MODES[1], C, C)) + 1j * r.normal(size=(MODES[0], MODES[1], C, C))) * scale_r
    return W, R


def test_stencil_branch_layout_exact(M):
    S, _ = _sur(M)
    W, _ = _random_params(1)
    W = bf16(W)
    R = np.zeros((MODES[0], MODES[1], C, C), complex)
    S.setParams(W, R)
    x = bf16(np.random.default_rng(2).normal(size=(3, N)))
    got = S.forward(x)
    ref = OS.forward(x, W, R, DIMS, MODES[0], MODES[1], RAD)
    assert rel_err(got, ref) <= 1e-5


def test_spectral_branch(M):
    S, _ = _sur(M)
    _, R = _random_params(3)
    W = np.zeros(((2 * RAD + 1) ** 2, C, C))
    S.setParams(W, R)
    x = np.random.default_rng(4).normal(size=(3, N))
    got = S.forward(x)
    ref = OS.forward(x.astype(np.float32), W, R.astype(np.complex64), DIMS, MODES[0], MODES[1], RAD)
    assert rel_err(got, ref) <= 2e-2


def test_full_forward_two_calls(M):
    S, _ = _sur(M)
    W, R = _random_params(5)
    S.setParams(W, R)
    Wr, Rr = S.params()
    x = np.random.default_rng(6).normal(size=(3, N))
    ref = OS.forward(x.astype(np.float32), Wr, Rr, DIMS, MODES[0], MODES[1], RAD)
    a = S.forward(x)
    b = S.forward(x)
    assert np.array_equal(a, b)
    assert rel_err(a, ref) <= 2e-2


def test_gradients_against_cpu_reference(M):
    S, _ = _sur(M)
    W, R = _random_params(7)
    S.setParams(W, R)
    Wr, Rr = S.params()
    r = np.random.default_rng(8)
    x = r.normal(size=(3, N)).astype(np.float32)
    t = r.normal(size=(3, N)).astype(np.float32)
    dW, dR, P, loss = S.gradients(x, t)
    # backward kernels on the device's own prediction
    L1, dW1, dR1, _ = OS.loss_and_gradients(x, t, Wr, Rr, DIMS, MODES[0], MODES[1], RAD, pred=P)
    assert loss == pytest.approx(L1, rel=1e-6)
    assert rel_err(dW, dW1) <= 1e-4
    assert crel(dR, dR1) <= 2e-2
    # end to end against the FP64 network
    L2, dW2, dR2, P2 = OS.loss_and_gradients(x, t, Wr, Rr, DIMS, MODES[0], MODES[1], RAD)
    assert rel_err(P, P2) <= 2e-2
    assert rel_err(dW, dW2) <= 3e-2
    assert crel(dR, dR2) <= 3e-2


def _film(M, dims, seed, T=0.1):
    n = int(np.prod(dims))
    ss = M.SpinSystem(*dims)
    ss.setSpinArrays(*random_spins(n, seed))
    ss.setAlpha(0.02)
    ss.setTimeStep(0.005)
    ex = M.Exchange(ss)
    import oracle as O
    f, to, j = O.nn_paths(*dims, J=1.0, pbc=(1, 1, 0))
    ex.addPaths(f, to, j)
    ani = M.Anisotropy(ss)
    ani.addMany(np.arange(n, dtype=np.int32), np.tile([0.0, 0.0, 1.0], (n, 1)), np.full(n, 0.02))
    dip = M.Dipole(ss)
    dip.setStrength(0.05)
    ops = [ex, ani, dip]
    if T > 0:
        th = M.Thermal(ss)
        th.setTemperature(T)
        th.setSeed(seed)
        ops.append(th)
    return ss, ops, dip


def test_training_gains_over_holding_the_field(M):
    dims = (128, 128, 2)
    ss, ops, dip = _film(M, dims, 101)
    S = M.Surrogate(dip, (16, 16), 2)
    llg = M.LLG.new("Quaternion")
    loss = S.train(ss, ops, llg, 600, window=10, lr=2e-3)
    v = S.validate(ss, ops, llg, 100, window=10)
    assert loss < 0.2, loss
    # the trained network's field is closer to the exact one than the field
    # held from the last exact evaluation (the method without it)
    assert v["field_mean"] * 4 < v["field_without_mean"], v
    assert v["dh_mean"] < 0.5, v


def _fp64_field_error(M, S, ss, ops, dip, llg, k, windows):
    """Relative dipolar-field error of the surrogate against the FP64 field
    over `windows` windows of k steps: at each window's start m0 and the
    exact FP32 field H0 (what a surrogate run holds); for j = 1 .. k-1 plain
    steps, H0 + net(m_j - m0) against the field of m_j evaluated with FP64
    state (FP64 FFT convolution of the same Dipole tensor).  Returns the mean
    error and the mean error of holding H0."""
    dims = ss._dims
    d64 = M.SpinSystem(*dims, precision="f64")
    dip64 = M.Dipole(*dims)
    dip64.setStrength(dip.strength())
    errs, hold = [], []
    for _ in range(windows):
        m0 = np.stack(ss.spinArrays()[:3])
        ss.resetFields()
        dip.apply(ss)
        h0 = np.stack(ss.fieldArrays("Dipole"))
        for _j in range(1, k):
            M.run(ss, ops, llg, 1)
            mj = np.stack(ss.spinArrays()[:3])
            d64.setSpinArrays(*mj)
            dip64.apply(d64)
            h64 = np.stack(d64.fieldArrays("Dipole"))
            nrm = np.linalg.norm(h64)
            errs.append(np.linalg.norm(h0 + S.forward(mj - m0) - h64) / nrm)
            hold.append(np.linalg.norm(h0 - h64) / nrm)
        M.run(ss, ops, llg, 1)
    return float(np.mean(errs)), float(np.mean(hold))


def test_radius3_network_within_field_error_bar(M):
    """The surrogate configuration's film (512x512x4, J=1, K=0.02, g=0.05,
    T=0.1, alpha=0.02, dt=0.005): a 16x16-mode, radius-3 network trained
    online on the plain method predicts the dipolar field between exact
    evaluations 5 steps apart within 1e-3 relative error against the FP64
    field, more than ten times closer than holding the field."""
    dims = (512, 512, 4)
    ss, ops, dip = _film(M, dims, 1000)
    llg = M.LLG.new("Quaternion")
    M.run(ss, ops, llg, 50)
    S = M.Surrogate(dip, (16, 16), 3)
    S.train(ss, ops, llg, 1000, window=10, lr=2e-3)
    err, hold = _fp64_field_error(M, S, ss, ops, dip, llg, 5, 2)
    assert err <= 1e-3, (err, hold)
    assert err * 10 < hold, (err, hold)


def test_run_with_zero_tolerance_equals_plain_run(M):
    dims = (128, 32, 2)
    ss, ops, dip = _film(M, dims, 202, T=0.0)
    ref, ops_r, dip_r = _film(M, dims, 202, T=0.0)
    S = M.Surrogate(dip, (8, 8), RAD)
    W, R = _random_params(9)
    S.setParams(W * 1e-2, R * 1e-2)
    S.setSchedule(4, tol=0.0, eps=1.0)    # every residual check fails: every step exact
    llg = M.LLG.new("Quaternion")
    S.run(ss, ops, llg, 12)
    M.run(ref, ops_r, M.LLG.new("Quaternion"), 12)
    a = np.stack(ss.spinArrays()[:3])
    b = np.stack(ref.spinArrays()[:3])
    assert np.array_equal(a, b)
    st = S.stats()
    assert st["exact"] == 12 and st["surrogate"] == 0


def test_run_schedule_counts_and_stays_close(M):
    dims = (128, 128, 2)
    ss, ops, dip = _film(M, dims, 303)
    S = M.Surrogate(dip, (16, 16), 2)
    llg = M.LLG.new("Quaternion")
    S.train(ss, ops, llg, 300, window=5, lr=2e-3)
    S.setSchedule(5, tol=1.0)             # no residual failures at this bound
    S.run(ss, ops, llg, 40)
    st = S.stats()
    assert st["exact"] == 8 and st["surrogate"] == 32 and st["failed"] == 0, st


def test_fused_surrogate_step_equals_individual_calls(M):
    """Attached surrogate: steps run through the fused output pass (network
    field + LLG update in one kernel, exact steps through the fused x pass)
    equal the same steps issued as individual calls, which materialise the
    field in the slot and run the separate step kernel."""
    dims = (128, 32, 2)
    res = []
    for mode in ("calls", "run"):
        ss, ops, dip = _film(M, dims, 404)
        S = M.Surrogate(dip, (8, 8), RAD)
        W, R = _random_params(10)
        S.setParams(W * 1e-2, R * 1e-2)
        S.setSchedule(3, tol=1.0, eps=0.05)
        llg = M.LLG.new("Quaternion")
        S.attach(ss)
        if mode == "calls":
            for _ in range(8):
                ss.resetFields()
                for op in ops:
                    op.apply(ss)
                ss.sumFields()
                llg.apply(ss)
        else:
            M.run(ss, ops, llg, 8)
        S.detach(ss)
        res.append((np.stack(ss.spinArrays()[:3]), np.stack(ss.fieldArrays("Dipole")), S.stats()))
    np.testing.assert_array_equal(res[0][0], res[1][0])
    np.testing.assert_array_equal(res[0][1], res[1][1])
    assert res[0][2]["exact"] == res[1][2]["exact"] == 3, res
    assert res[1][2]["surrogate"] == 5, res


def test_completion_wait_limit_reports_and_recovers(M):
    """A tensor-core completion wait that gives up sets the surrogate's error
    flag and the host call returns MLB_ECUDA; the kernel still waits (bounded)
    for its own MMAs before reading and freeing TMEM, so the context stays
    usable: with the default limit the next forward equals a clean one."""
    S, _ = _sur(M)
    W, R = _random_params(12)
    S.setParams(W, R)
    x = random_spins(N, 13)
    clean = S.forward(x)
    S.setWaitLimit(0)            # every completion wait gives up at once
    with pytest.raises(M.MagLuaError) as ei:
        S.forward(x)
    assert ei.value.code == -3 and "gave up" in str(ei.value)
    S.setWaitLimit(1 << 24)
    again = S.forward(x)
    np.testing.assert_array_equal(again, clean)
