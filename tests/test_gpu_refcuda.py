"""Parity pinned to the reference's own arithmetic: the reference's FP64 CUDA
kernels, compiled unchanged from its sources into oracle/_ref/libref_cuda.so
(oracle/Makefile), run beside the oracle and the product on the same seeded
inputs (M/ = src/modules/):

* LLG.Quaternion  -- cuda_llg_quat_apply (M/cuda/llg_cuda/llgquat.cu:283)
* LLG.Cartesian   -- cuda_llg_cart_apply_N (M/cuda/llg_cuda/llgcartesian.cu:133),
                     two replicas in one batched call
* Anisotropy      -- cuda_anisotropy_N (M/cuda/anisotropy_cuda/spinoperationanisotropy.cu:50)
* Thermal         -- cuda_thermal (M/cuda/thermal_cuda/spinoperationthermal.cu:77)
                     with the same FP32 normals injected everywhere

Tolerances: FP64 (oracle and the product's FP64 state) within 1e-12
relative of the reference kernel's output; the product's FP32 state within
2e-6 (one FP32 step).  Known semantic delta, recorded in the anisotropy
test: the reference's GPU anisotropy divides by |s|^2 where its CPU build
(and the oracle and the product) divide by ms^2; inputs with |s| = ms make
them agree, and a site with |s| != ms shows the difference."""
import numpy as np
import pytest

import oracle as O
from oracle import refcuda
from helpers import random_spins, rel_err

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 2e-6
DIMS = (13, 7, 3)          # 273 sites: not a multiple of the reference's 512-thread blocks


@pytest.fixture(scope="module")
def R():
    lib = refcuda.load()
    if lib is None:
        pytest.skip("oracle/_ref/libref_cuda.so not built (no reference tree where the build ran)")
    return lib


@pytest.fixture(scope="module")
def torch():
    import torch
    return torch


@pytest.fixture(scope="module")
def M():
    import maglua_b200 as M
    M.init(0)
    return M


def _dev(torch, a):
    return torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


def _inputs(seed, n):
    r = np.random.default_rng(seed)
    s = random_spins(n, seed, lengths=True)
    h = r.normal(size=(3, n))
    ht = 0.3 * r.normal(size=(3, n))
    return s, h, ht


def _oracle_llg(kind, s, h, ht, alpha, dt, gamma, tfirst, site_alpha=None):
    o = O.SpinSystem(*DIMS)
    o.set_spins(*s)
    o.alpha, o.dt, o.gamma = alpha, dt, gamma
    if site_alpha is not None:
        o.set_site_alpha(site_alpha)
    for name, f in (("Total", h), ("Thermal", ht)):
        v = o.field_views(name)
        for c in range(3):
            v[c][:] = f[c]
        o.set_slot_used(name, True)
    O.LLG(kind, thermal_only_first_term=int(tfirst)).apply(o)
    return o.spins()


def _product_llg(M, kind, s, h, ht, alpha, dt, gamma, tfirst, precision, site_alpha=None):
    ss = M.SpinSystem(*DIMS, precision=precision)
    ss.setSpinArrays(*s)
    ss.setAlpha(alpha)
    ss.setTimeStep(dt)
    ss.setGamma(gamma)
    if site_alpha is not None:
        ss.setSiteAlphaArray(site_alpha)
    ss.setFieldArrays("Total", *h)
    ss.setFieldArrays("Thermal", *ht)
    llg = M.LLG.new(kind)
    llg.setThermalOnlyFirstTerm(bool(tfirst))
    llg.apply(ss)
    return np.stack(ss.spinArrays()[:3])


@pytest.mark.parametrize("tfirst", [1, 0])
@pytest.mark.parametrize("per_site_alpha", [False, True])
def test_quaternion_llg_matches_reference_cuda(R, torch, M, tfirst, per_site_alpha):
    n = int(np.prod(DIMS))
    s, h, ht = _inputs(11 + tfirst, n)
    alpha, dt, gamma = 0.13, 0.05, 1.7
    sa = np.random.default_rng(3).uniform(0.05, 0.3, n) if per_site_alpha else None
    ms = np.linalg.norm(s, axis=0)
    frm = [_dev(torch, s[c]) for c in range(3)] + [_dev(torch, ms)]
    to = [torch.zeros(n, dtype=torch.float64, device="cuda") for _ in range(4)]
    H = [_dev(torch, h[c]) for c in range(3)]
    HT = [_dev(torch, ht[c]) for c in range(3)]
    ws = [torch.zeros(n, dtype=torch.float64, device="cuda") for _ in range(4)]
    d_alpha = None if sa is None else _dev(torch, sa)
    rc = R.ref_llg_quat_apply(*DIMS, refcuda.ptrs(*to), refcuda.ptrs(*frm), refcuda.ptrs(*frm), refcuda.ptrs(*HT),
                              refcuda.ptrs(*H), refcuda.ptrs(*ws), dt, alpha,
                              None if d_alpha is None else d_alpha.data_ptr(), gamma, None, tfirst)
    assert rc == 0
    ref = torch.stack(to[:3]).cpu().numpy()
    assert np.array_equal(to[3].cpu().numpy(), ms)        # the reference copies ms into the destination
    orc = _oracle_llg("Quaternion", s, h, ht, alpha, dt, gamma, tfirst, sa)
    p64 = _product_llg(M, "Quaternion", s, h, ht, alpha, dt, gamma, tfirst, "f64", sa)
    p32 = _product_llg(M, "Quaternion", s, h, ht, alpha, dt, gamma, tfirst, "f32", sa)
    assert rel_err(orc, ref) <= TOL64
    assert rel_err(p64, ref) <= TOL64
    assert rel_err(p32, ref) <= TOL32


@pytest.mark.parametrize("tfirst", [1, 0])
@pytest.mark.parametrize("renorm", [True, False])
def test_cartesian_llg_batched_matches_reference_cuda(R, torch, M, tfirst, renorm):
    n = int(np.prod(DIMS))
    reps = []
    for j, (alpha, dt, gamma) in enumerate(((0.1, 0.02, 1.0), (0.25, 0.01, 2.0))):
        s, h, ht = _inputs(40 + j, n)
        reps.append((s, h, ht, alpha, dt, gamma))
    cols = {k: [] for k in ("to", "frm", "H", "HT")}
    keep = []
    for s, h, ht, *_ in reps:
        ms = np.linalg.norm(s, axis=0)
        cols["frm"].append([_dev(torch, s[c]) for c in range(3)] + [_dev(torch, ms)])
        cols["to"].append([torch.zeros(n, dtype=torch.float64, device="cuda") for _ in range(4)])
        cols["H"].append([_dev(torch, h[c]) for c in range(3)])
        cols["HT"].append([_dev(torch, ht[c]) for c in range(3)])

    def parr(group, c):
        t = torch.tensor([rep[c].data_ptr() for rep in cols[group]], dtype=torch.int64, device="cuda")
        keep.append(t)
        return t

    to = refcuda.ptrs(*[parr("to", c) for c in range(4)])
    frm = refcuda.ptrs(*[parr("frm", c) for c in range(4)])
    H = refcuda.ptrs(*[parr("H", c) for c in range(3)])
    HT = refcuda.ptrs(*[parr("HT", c) for c in range(3)])
    dt = _dev(torch, [r[4] for r in reps])
    alpha = _dev(torch, [r[3] for r in reps])
    gamma = _dev(torch, [r[5] for r in reps])
    nullp = torch.zeros(len(reps), dtype=torch.int64, device="cuda")
    rc = R.ref_llg_cart_apply_n(*DIMS, to, frm, frm, HT, H, dt.data_ptr(), nullp.data_ptr(), alpha.data_ptr(),
                                nullp.data_ptr(), gamma.data_ptr(), tfirst, int(not renorm), len(reps))
    assert rc == 0
    for j, (s, h, ht, a, d, g) in enumerate(reps):
        ref = torch.stack(cols["to"][j][:3]).cpu().numpy()
        o = O.SpinSystem(*DIMS)
        o.set_spins(*s)
        o.alpha, o.dt, o.gamma = a, d, g
        for name, f in (("Total", h), ("Thermal", ht)):
            v = o.field_views(name)
            for c in range(3):
                v[c][:] = f[c]
            o.set_slot_used(name, True)
        O.LLG("Cartesian", thermal_only_first_term=tfirst, disable_renormalization=int(not renorm)).apply(o)
        assert rel_err(o.spins(), ref) <= TOL64
        for prec, tol in (("f64", TOL64), ("f32", TOL32)):
            ss = M.SpinSystem(*DIMS, precision=prec)
            ss.setSpinArrays(*s)
            ss.setAlpha(a)
            ss.setTimeStep(d)
            ss.setGamma(g)
            ss.setFieldArrays("Total", *h)
            ss.setFieldArrays("Thermal", *ht)
            llg = M.LLG.new("Cartesian")
            llg.setThermalOnlyFirstTerm(bool(tfirst))
            llg.setDisableRenormalization(not renorm)
            llg.apply(ss)
            assert rel_err(np.stack(ss.spinArrays()[:3]), ref) <= tol


def test_anisotropy_matches_reference_cuda(R, torch, M):
    n = int(np.prod(DIMS))
    r = np.random.default_rng(7)
    s = random_spins(n, 7, lengths=True)
    axes = r.normal(size=(n, 3))
    axes /= np.linalg.norm(axes, axis=1)[:, None]
    K = r.uniform(-0.5, 0.5, n)
    gs = 0.8
    S = [_dev(torch, s[c]) for c in range(3)]
    Hh = [torch.zeros(n, dtype=torch.float64, device="cuda") for _ in range(3)]
    keep = [torch.tensor([t.data_ptr()], dtype=torch.int64, device="cuda") for t in S + Hh]
    A = [_dev(torch, axes[:, c]) for c in range(3)]
    Kd = _dev(torch, K)
    rc = R.ref_anisotropy_n(gs, *[k.data_ptr() for k in keep[:3]], *[a.data_ptr() for a in A], Kd.data_ptr(),
                            *[k.data_ptr() for k in keep[3:]], n, 1)
    assert rc == 0
    ref = torch.stack(Hh).cpu().numpy()
    sites = np.arange(n, dtype=np.int32)
    o = O.SpinSystem(*DIMS)
    o.set_spins(*s)
    O.anisotropy_apply(o, sites, axes, K, gscale=gs)
    assert rel_err(o.field("Anisotropy"), ref) <= TOL64
    for prec, tol in (("f64", TOL64), ("f32", TOL32)):
        ss = M.SpinSystem(*DIMS, precision=prec)
        ss.setSpinArrays(*s)
        ani = M.Anisotropy(*DIMS)
        ani.addMany(sites, axes, K)
        ani.setScale(gs)
        ani.apply(ss)
        assert rel_err(np.stack(ss.fieldArrays("Anisotropy")), ref) <= tol
    # the delta: a moment magnitude that differs from |s| (the reference's
    # GPU kernel uses |s|^2, its CPU build ms^2)
    ss = M.SpinSystem(*DIMS, precision="f64")
    ms = np.linalg.norm(s, axis=0)
    ms2 = ms.copy()
    ms2[0] *= 2.0
    ss.setSpinArrays(*s, ms2)
    ani = M.Anisotropy(*DIMS)
    ani.addMany(sites, axes, K)
    ani.setScale(gs)
    ani.apply(ss)
    got = np.stack(ss.fieldArrays("Anisotropy"))
    assert np.allclose(got[:, 0], ref[:, 0] / 4.0, rtol=1e-12, atol=1e-15)
    assert rel_err(got[:, 1:], ref[:, 1:]) <= TOL64


@pytest.mark.parametrize("half", [0, 1])
def test_thermal_matches_reference_cuda(R, torch, M, half):
    n = int(np.prod(DIMS))
    r = np.random.default_rng(21 + half)
    rng6 = r.normal(size=(n, 6)).astype(np.float32)
    s = random_spins(n, 22, lengths=True)
    ms = np.linalg.norm(s, axis=0)
    scale = r.uniform(0.5, 2.0, n)
    T, alpha, dt, gamma = 0.7, 0.1, 0.01, 1.3
    Hh = [torch.zeros(n, dtype=torch.float64, device="cuda") for _ in range(3)]
    d_rng = torch.tensor(rng6.reshape(-1), device="cuda")
    d_ms, d_sc = _dev(torch, ms), _dev(torch, scale)
    rc = R.ref_thermal(d_rng.data_ptr(), half, T, *[h.data_ptr() for h in Hh], d_ms.data_ptr(), d_sc.data_ptr(), n,
                       dt, alpha, None, gamma, None)
    assert rc == 0
    ref = torch.stack(Hh).cpu().numpy()
    noise = [rng6[:, 3 * half + c].astype(np.float64) for c in range(3)]
    o = O.SpinSystem(*DIMS)
    o.set_spins(*s)
    o.alpha, o.dt, o.gamma = alpha, dt, gamma
    O.thermal_apply_noise(o, T, noise, scale=scale)
    assert rel_err(o.field("Thermal"), ref) <= TOL64
    for prec, tol in (("f64", TOL64), ("f32", TOL32)):
        ss = M.SpinSystem(*DIMS, precision=prec)
        ss.setSpinArrays(*s)
        ss.setAlpha(alpha)
        ss.setTimeStep(dt)
        ss.setGamma(gamma)
        th = M.Thermal(*DIMS)
        th.setTemperature(T)
        for i in range(n):
            assert M._lib.mlb_thermal_scale_site(th._h, i, float(scale[i])) == 0
        th.inject(*noise)
        th.apply(ss)
        assert rel_err(np.stack(ss.fieldArrays("Thermal")), ref) <= tol
