"""Benchmark of the spin-dynamics step (spin-steps/s) on B200.

Workload (one replica per GPU, weak scaling): 256x256x8 simple-cubic film,
periodic in x/y and open in z (zero-padded FFT in z); nearest-neighbour
exchange J=1; anisotropy K=0.05 along z; dipole g=0.02; applied field 0.1
along x; thermal noise T=0.5; alpha=0.05, dt=0.005; spins +z with a seeded
5-degree random tilt; LLG.Quaternion.  One step = resetFields, the five
operators, sumFields, llg:apply -- the plain fused FFT path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Timing: each timed step is bracketed by CUDA events on the launching stream
and preceded by an L2 flush (a 1 GiB write, then a 512 MiB read sweep so the
flush's dirty lines are written back before the step; excluded from the step
time);
the value is total spin-steps over the max over ranks of the summed step
times.  Rank 0 prints one JSON line.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

NX, NY, NZ = 256, 256, 8
J, K_ANI, G_DIP, BX = 1.0, 0.05, 0.02, 0.1
TEMP, ALPHA, DT = 0.5, 0.05, 0.005
WORKLOAD = "film 256x256x8, periodic x/y, open z (z padded to 16), J=1, K=0.05 z, g=0.02, B=0.1 x, T=0.5, alpha=0.05, dt=0.005, LLG.Quaternion"
METRIC = "spin-steps/s"
UNIT = "spin-steps/s"
FLUSH_BYTES = 1 << 30


def tilted_spins(n, seed, deg=5.0):
    r = np.random.default_rng(seed)
    phi = r.uniform(0, 2 * np.pi, n)
    th = np.deg2rad(deg)
    return np.stack([np.sin(th) * np.cos(phi), np.sin(th) * np.sin(phi), np.full(n, np.cos(th))])


def nn_paths(nx, ny, nz, pbc=(1, 1, 0)):
    """Pathways of the canonical setup loop ex:add({i,j,k},{i+-1,...},J)."""
    idx = np.arange(nx * ny * nz, dtype=np.int32).reshape(nz, ny, nx)
    frm, to = [], []
    for ax, n in ((2, nx), (1, ny), (0, nz)):
        for sgn in (1, -1):
            src = idx
            dst = np.roll(idx, -sgn, axis=ax)
            if not pbc[2 - ax]:
                sl = [slice(None)] * 3
                sl[ax] = slice(0, n - 1) if sgn == 1 else slice(1, n)
                src, dst = src[tuple(sl)], dst[tuple(sl)]
            frm.append(src.ravel())
            to.append(dst.ravel())
    f = np.concatenate(frm).astype(np.int32)
    t = np.concatenate(to).astype(np.int32)
    return f, t, np.full(len(f), J)


def build_system(M, seed, precision="f32"):
    n = NX * NY * NZ
    ss = M.SpinSystem(NX, NY, NZ, precision=precision)
    ss.setSpinArrays(*tilted_spins(n, seed))
    ss.setAlpha(ALPHA)
    ss.setTimeStep(DT)
    ex = M.Exchange(ss)
    ex.addPaths(*nn_paths(NX, NY, NZ))
    ani = M.Anisotropy(ss)
    ani.addMany(np.arange(n), np.tile([0, 0, 1.0], (n, 1)), np.full(n, K_ANI))
    th = M.Thermal(ss, M.Random.Philox(1000 + seed))
    th.setTemperature(TEMP)
    z = M.AppliedField(ss)
    z.set(BX, 0, 0)
    dip = M.Dipole(ss)
    dip.setStrength(G_DIP)
    llg = M.LLG.new("Quaternion")
    return ss, [ex, ani, th, z, dip], llg


# ----------------------------------------------------------------- batched ensemble
ENS_CLASSES = [(16, 16, 16), (32, 32, 4), (48, 48, 2), (64, 64, 4)]
ENS_WORKLOAD = ("512 replicas, sizes drawn (seed 3) from 16^3, 32x32x4, 48x48x2, 64x64x4; open boundaries "
                "(every axis padded x2); J=1, K=0.2 z, dipole g=0.02, T=0.2, alpha=0.1, dt=0.01, all +z, "
                "B_z swept 0 -> -0.5 over 20000 steps; LLG.Cartesian")


def ensemble_dims(nrep=512, seed=3):
    r = np.random.default_rng(seed)
    return [ENS_CLASSES[k] for k in r.integers(0, 4, nrep)]


def _ensemble_configure(e, g):
    e.configure(alpha=0.1, dt=0.01, J=1.0, pbc=(0, 0, 0), K=0.2, axis=(0, 0, 1), T=0.2, seed=7,
                B=(0, 0, 0), dB=(0, 0, -0.5 / 20000), g=g, open_xy=True, llg="Cartesian")


def _time_ensemble(M, torch, dims, g, steps, warmup):
    e = M.Ensemble(dims)
    _ensemble_configure(e, g)
    for r, d in enumerate(dims):
        n = int(np.prod(d))
        e.setSpins(r, np.zeros(n), np.zeros(n), np.ones(n))
    e.run(warmup)
    st = torch.cuda.ExternalStream(e.stream())
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(st)
    e.run(steps)
    b.record(st)
    torch.cuda.synchronize()
    return e, a.elapsed_time(b) / steps


def _plain_replicas(M, torch, dims, steps):
    """The plain path over the same replicas: one SpinSystem per replica
    (each on its own stream) with the operator set shared per size class
    (the reference's op:apply({ss...}) pattern), every replica's captured
    step launched by a host loop; wall clock around whole steps of all
    replicas, synchronised at both ends."""
    ops_by = {}
    systems = []
    for d in dims:
        n = int(np.prod(d))
        ss = M.SpinSystem(*d)
        ss.setSpinArrays(np.zeros(n), np.zeros(n), np.ones(n))
        ss.setAlpha(0.1)
        ss.setTimeStep(0.01)
        if d not in ops_by:
            ex = M.Exchange(*d)
            ex.addPaths(*nn_paths(*d, pbc=(0, 0, 0)))
            ani = M.Anisotropy(*d)
            ani.addMany(np.arange(n), np.tile([0, 0, 1.0], (n, 1)), np.full(n, 0.2))
            th = M.Thermal(*d)
            th.setSeed(7)
            th.setTemperature(0.2)
            z = M.AppliedField(*d)
            z.set(0, 0, 0)
            z.setSweep(0, 0, -0.5 / 20000)
            dip = M.Dipole(*d)
            dip.setOpen(True, True, True)
            dip.setStrength(0.02)
            ops_by[d] = [ex, ani, th, z, dip]
        llg = M.LLG.new("Cartesian")
        systems.append((ss, M.Plan(ss, ops_by[d], llg)))
    for ss, p in systems:
        p.launch(2)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        for ss, p in systems:
            p.launch(1)
    torch.cuda.synchronize()
    return (time.perf_counter() - t0) * 1e3 / steps


def _pow2_at_least(m):
    p = 1
    while p < m:
        p *= 2
    return p


def ensemble_bytes(dims):
    """Algorithmic bytes of one ensemble step by the per-site formula
    B = 36 + 24 + (K/N)(24 + 48 * 2) per replica, K = (Px/2+1) Py Pz stored
    k-points with every axis of an open replica padded to the power of two
    at least 2n - 1 (z: 1 when nz = 1)."""
    total = 0
    for nx, ny, nz in dims:
        n = nx * ny * nz
        Px, Py = _pow2_at_least(2 * nx - 1), _pow2_at_least(2 * ny - 1)
        Pz = 1 if nz == 1 else _pow2_at_least(2 * nz - 1)
        K = (Px // 2 + 1) * Py * Pz
        total += 60 * n + K * (24 + 48 * 2)
    return total


def run_batched(M, torch, steps, warmup):
    """Configuration 3: the packed ensemble (one captured graph per step,
    classes on concurrent branches, tuned tile/grid/(y,z) variant), the same
    replicas through the plain path one SpinSystem per replica, and the
    ensemble without the dipole (the bound any dipole surrogate works under)."""
    dims = ensemble_dims()
    e, ms = _time_ensemble(M, torch, dims, 0.02, steps, warmup)
    info = e.info()
    sites = info["sites"]
    _, ms_nodip = _time_ensemble(M, torch, dims, 0.0, steps, warmup)
    plain_ms = _plain_replicas(M, torch, dims, max(3, min(steps, 10)))
    nbytes = ensemble_bytes(dims)
    peak, peak_kind = measured_peak()
    return {"value": sites * steps / (ms * steps * 1e-3), "unit": UNIT, "ms_per_step": ms,
            "sites": sites, "replicas": len(dims), "fused_block_size": info["block_size"],
            "step_roofline": {"algorithmic_bytes_per_step": nbytes, "achieved_gbs": nbytes / (ms * 1e-3) / 1e9,
                              "frac": nbytes / (ms * 1e-3) / 1e9 / peak, "peak": peak, "peak_kind": peak_kind,
                              "how": "36 + 24 B per site + (24 + 96) B per stored k-point of each replica's padded "
                                     "grid, over the event-timed step"},
            "config": e.configInfo(), "tune_log": e.tuneLog().strip().splitlines(),
            "workload": ENS_WORKLOAD,
            "plain_one_system_per_replica": {"value": sites / (plain_ms * 1e-3), "ms_per_step": plain_ms,
                                             "speedup_of_batched": plain_ms / ms,
                                             "how": "512 SpinSystems, operators shared per size class, one captured "
                                                    "plain step per replica launched by a host loop; wall clock over "
                                                    "whole steps (synchronised at both ends)"},
            "without_dipole": {"ms_per_step": ms_nodip, "value": sites / (ms_nodip * 1e-3),
                               "amdahl_ceiling": ms / ms_nodip,
                               "how": "the same ensemble with g = 0: every dipole pass removed, the bound on what "
                                      "replacing the dipole evaluation by anything can gain"},
            "l2": "working set larger than L2 (no flush)"}


# ----------------------------------------------------------------- learned surrogate
SUR_DIMS = (512, 512, 4)
SUR_WORKLOAD = ("film 512x512x4, periodic x/y, open z (z padded to 8), J=1, K=0.02 z, g=0.05, T=0.1, "
                "alpha=0.02, dt=0.005, LLG.Quaternion; spins from a seeded random start relaxed 200 steps; "
                "surrogate: linear spectral-conv net (BF16 tcgen05, 16x16 modes, radius-3 stencil) trained "
                "online on the plain method over 8 seeded random-start runs")


def _sur_system(M, dims, seed, relax, ops=None):
    """A 512x512x4 film from a seeded random start with the surrogate
    workload's operators (shared between systems of the size), relaxed by
    `relax` plain steps."""
    n = int(np.prod(dims))
    r = np.random.default_rng(seed)
    v = r.normal(size=(3, n))
    v /= np.linalg.norm(v, axis=0)
    ss = M.SpinSystem(*dims)
    ss.setSpinArrays(*v)
    ss.setAlpha(0.02)
    ss.setTimeStep(0.005)
    if ops is None:
        ex = M.Exchange(*dims)
        ex.addPaths(*nn_paths(*dims))
        ani = M.Anisotropy(*dims)
        ani.addMany(np.arange(n), np.tile([0, 0, 1.0], (n, 1)), np.full(n, 0.02))
        th = M.Thermal(*dims)
        th.setSeed(1000)
        th.setTemperature(0.1)
        dip = M.Dipole(*dims)
        dip.setStrength(0.05)
        ops = [ex, ani, th, dip]
    llg = M.LLG.new("Quaternion")
    if relax:
        M.run(ss, ops, llg, relax)
    return ss, ops, llg


def _sur_error_fp64(M, S, ss, ops, llg, k, windows):
    """Relative dipolar-field error of the surrogate against the FP64 field:
    per window, m0 and the exact FP32 field H0 at its start (what a surrogate
    run holds), then for j = 1 .. k-1 plain steps H0 + net(m_j - m0) against
    the field of m_j evaluated with FP64 state (FP64 FFT convolution of the
    same Dipole tensor).  Returns mean and max of the error and the same for
    holding H0 (the method without the network)."""
    dims = ss._dims
    d64 = M.SpinSystem(*dims, precision="f64")
    dip64 = M.Dipole(*dims)
    dip64.setStrength(ops[-1].strength())
    dip = ops[-1]
    errs, hold = [], []
    for _ in range(windows):
        m0 = np.stack(ss.spinArrays()[:3])
        ss.resetFields()
        dip.apply(ss)
        h0 = np.stack(ss.fieldArrays("Dipole"))
        for j in range(1, k):
            M.run(ss, ops, llg, 1)
            mj = np.stack(ss.spinArrays()[:3])
            d64.setSpinArrays(*mj)
            dip64.apply(d64)
            h64 = np.stack(d64.fieldArrays("Dipole"))
            pred = h0 + S.forward(mj - m0)
            nrm = np.linalg.norm(h64)
            errs.append(float(np.linalg.norm(pred - h64) / nrm))
            hold.append(float(np.linalg.norm(h0 - h64) / nrm))
        M.run(ss, ops, llg, 1)
    return float(np.mean(errs)), float(np.max(errs)), float(np.mean(hold))


def run_surrogate(M, torch, steps, train_runs=8, train_steps=250, radius=3):
    """Plain fused FFT path vs the learned surrogate on the 512x512x4 film:
    spin-steps/s of both on the same system; the surrogate trained on the
    plain method over `train_runs` seeded random-start runs; its relative
    dipolar-field error against the FP64 field at each exact-evaluation
    period k (and the run's own residual-check statistics)."""
    dims = SUR_DIMS
    n = int(np.prod(dims))
    ss, ops, llg = _sur_system(M, dims, 1000, 200)
    st = torch.cuda.ExternalStream(ss.stream())

    def timed(fn, k):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ss.synchronize()
        a.record(st)
        fn(k)
        b.record(st)
        ss.synchronize()
        return a.elapsed_time(b) / k

    plan = M.Plan(ss, ops, llg)
    plan.launch(3)
    plain_ms = timed(plan.launch, steps)
    plan_nd = M.Plan(ss, ops[:3], llg)
    plan_nd.launch(3)
    nodip_ms = timed(plan_nd.launch, steps)
    del plan_nd
    S = M.Surrogate(ops[-1], (16, 16), radius)
    t0 = time.perf_counter()
    losses = []
    for r in range(train_runs):
        tss, _, tl = _sur_system(M, dims, 2000 + r, 50, ops)
        losses.append(S.train(tss, ops, tl, train_steps, window=10, lr=2e-3))
        del tss
    train_s = time.perf_counter() - t0
    out = {"workload": SUR_WORKLOAD, "sites": n, "radius": radius, "modes": [16, 16],
           "plain": {"value": n / (plain_ms * 1e-3), "ms_per_step": plain_ms},
           "without_dipole": {"ms_per_step": nodip_ms, "amdahl_ceiling": plain_ms / nodip_ms,
                              "how": "the same film's captured step without the Dipole operator: the bound on what "
                                     "replacing the dipole evaluation by anything can gain"},
           "train": {"runs": train_runs, "steps_per_run": train_steps, "seconds": train_s,
                     "final_rel_loss_per_run": losses,
                     "how": "online training on the plain method, one seeded random-start run after another "
                            "(seeds 2000..), each relaxed 50 steps first"},
           "by_k": {}}
    for k in (5, 10, 20):
        val = S.validate(ss, ops, llg, 4 * k, window=k)
        e64 = _sur_error_fp64(M, S, ss, ops, llg, k, 2)
        S.setSchedule(k, tol=1e-3)
        S.run(ss, ops, llg, k)
        ms = timed(lambda m: S.run(ss, ops, llg, m), max(steps, 10 * k))
        st_ = S.stats()
        out["by_k"][str(k)] = {"value": n / (ms * 1e-3), "ms_per_step": ms, "speedup_vs_plain": plain_ms / ms,
                               "field_rel_err_vs_fp64_mean": e64[0], "field_rel_err_vs_fp64_max": e64[1],
                               "field_rel_err_vs_fp64_without_net_mean": e64[2],
                               "field_rel_err_vs_fp32_mean": val["field_mean"],
                               "field_rel_err_vs_fp32_max": val["field_max"],
                               "exact": st_["exact"], "surrogate": st_["surrogate"], "failed_checks": st_["failed"]}
    out["l2"] = "working set about 100 MB: L2-resident, no flush (both paths measured the same way)"
    return out


def run_fno_study(M, torch, runs=64, snaps=24, window=8, steps_per_eval=20, lin_radius=2):
    """The network the learned-surrogate configuration names -- a 4-layer
    spectral-convolution network (FNO: lift 1x1 to 32 channels, four layers
    of a spectral convolution over 16 x 16 retained modes plus a 1x1
    convolution, GELU between layers, projection to the 12 channels), BF16
    1x1 convolutions, FP32 FFTs -- trained on (dm, dH_dip) pairs of the
    plain method from `runs` seeded random-start runs of the 512x512x4 film,
    against the library's linear stencil + spectral network (stencil radius
    lin_radius) trained on the same runs.  Reports both networks' relative dipolar-field error against
    the FP64 field at k = 5, 10, 20 and their cost per evaluation.  A
    comparison study in PyTorch (torch.fft, cuBLAS 1x1 convolutions): the
    product's surrogate is the library's own network and kernels."""
    import torch.nn.functional as Fn
    dims = SUR_DIMS
    nx, ny, nz = dims
    n = int(np.prod(dims))
    C, W, MD, L = 3 * nz, 32, 16, 4
    dev = "cuda"
    g = torch.Generator(device="cpu").manual_seed(5)

    def prm(*shape, scale):
        return torch.nn.Parameter((torch.randn(*shape, generator=g) * scale).to(dev))

    P = {"lift_w": prm(W, C, scale=1 / np.sqrt(C)), "lift_b": prm(W, scale=0.0),
         "proj_w": prm(C, W, scale=1 / np.sqrt(W)), "proj_b": prm(C, scale=0.0)}
    for l in range(L):
        P[f"spec{l}"] = prm(W, W, MD, MD, 2, scale=1 / W)
        P[f"pw{l}"] = prm(W, W, scale=1 / np.sqrt(W))
        P[f"pb{l}"] = prm(W, scale=0.0)

    def fno(x):   # x [B, C, ny, nx] (normalised dm) -> [B, C, ny, nx]
        with torch.autocast("cuda", dtype=torch.bfloat16):
            h = torch.einsum("oc,bcyx->boyx", P["lift_w"], x) + P["lift_b"][None, :, None, None]
        h = h.float()
        for l in range(L):
            X = torch.fft.rfft2(h)
            Wc = torch.view_as_complex(P[f"spec{l}"])       # [W, W, ky 16, kx 16]
            Y = torch.zeros_like(X)
            Y[:, :, :MD // 2, :MD] = torch.einsum("biyx,ioyx->boyx", X[:, :, :MD // 2, :MD], Wc[:, :, :MD // 2])
            Y[:, :, -MD // 2:, :MD] = torch.einsum("biyx,ioyx->boyx", X[:, :, -MD // 2:, :MD], Wc[:, :, MD // 2:])
            sp = torch.fft.irfft2(Y, s=h.shape[-2:])
            with torch.autocast("cuda", dtype=torch.bfloat16):
                pw = torch.einsum("oc,bcyx->boyx", P[f"pw{l}"], h) + P[f"pb{l}"][None, :, None, None]
            h = sp + pw.float()
            if l < L - 1:
                h = Fn.gelu(h)
        with torch.autocast("cuda", dtype=torch.bfloat16):
            out = torch.einsum("oc,bcyx->boyx", P["proj_w"], h) + P["proj_b"][None, :, None, None]
        return out.float()

    def chan(v):   # (3, n) numpy -> [1, C, ny, nx] on the GPU
        return torch.as_tensor(np.asarray(v, np.float32).reshape(3 * nz, ny, nx), device=dev)[None]

    ops = None
    S = None
    opt = torch.optim.Adam(list(P.values()), lr=1e-3)
    sx = sy = None
    losses = []
    t0 = time.perf_counter()
    for r in range(runs):
        tss, ops, tl = _sur_system(M, dims, 3000 + r, 50, ops)
        if S is None:
            S = M.Surrogate(ops[-1], (16, 16), lin_radius)
        # the library's network on this run (its own online training)
        S.train(tss, ops, tl, snaps, window=window, lr=2e-3)
        dip = ops[-1]
        for w in range(max(1, snaps // window)):
            tss.resetFields(); dip.apply(tss)
            m0 = np.stack(tss.spinArrays()[:3]); h0 = np.stack(tss.fieldArrays("Dipole"))
            for j in range(1, window + 1):
                M.run(tss, ops, tl, 1)
                tss.resetFields(); dip.apply(tss)
                x = chan(np.stack(tss.spinArrays()[:3]) - m0)
                t = chan(np.stack(tss.fieldArrays("Dipole")) - h0)
                if sx is None:   # normalisation from the first pair
                    sx = float(x.std()) + 1e-12
                    sy = float(t.std()) + 1e-12
                pred = fno(x / sx)
                loss = ((pred - t / sy) ** 2).sum() / ((t / sy) ** 2).sum()
                opt.zero_grad()
                loss.backward()
                opt.step()
                losses.append(loss.item())
        del tss
    train_s = time.perf_counter() - t0

    # errors against the FP64 field on the held-out film (seed 1000), as the
    # surrogate leg measures them
    ss, _, llg = _sur_system(M, dims, 1000, 200, ops)
    with torch.no_grad():
        fno_np = lambda d: (fno(chan(d) / sx) * sy).cpu().numpy()[0].reshape(3, n).astype(np.float64)
        q = max(1, len(losses) // 8)
        out = {"workload": SUR_WORKLOAD, "linear_radius": lin_radius, "runs": runs,
               "pairs_per_run": max(1, snaps // window) * window,
               "train_seconds": train_s, "fno_final_rel_loss": float(np.mean(losses[-window:])),
               "fno_rel_loss_by_eighth": [float(np.mean(losses[i * q:(i + 1) * q])) for i in range(8)], "by_k": {}}
        for k in (5, 10, 20):
            e_lin = _sur_error_fp64(M, S, ss, ops, llg, k, 2)
            F = type("FNOFwd", (), {"forward": staticmethod(fno_np)})
            e_fno = _sur_error_fp64(M, F, ss, ops, llg, k, 2)
            out["by_k"][str(k)] = {"linear_err_mean": e_lin[0], "linear_err_max": e_lin[1],
                                   "fno_err_mean": e_fno[0], "fno_err_max": e_fno[1], "hold_err_mean": e_lin[2]}
        # cost per evaluation: the FNO's forward (batch 1) and the library
        # network's forward, CUDA events; the exact FP32 dipole evaluation
        x = torch.randn(1, C, ny, nx, device=dev)
        for _ in range(3):
            fno(x)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(); a.record()
        for _ in range(steps_per_eval):
            fno(x)
        b.record(); torch.cuda.synchronize()
        out["fno_us_per_eval"] = a.elapsed_time(b) * 1e3 / steps_per_eval
    st = torch.cuda.ExternalStream(ss.stream())
    plan = M.Plan(ss, ops, llg)
    plan.launch(3)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ss.synchronize(); a.record(st); plan.launch(steps_per_eval); b.record(st); ss.synchronize()
    out["plain_step_us"] = a.elapsed_time(b) * 1e3 / steps_per_eval
    plan_nd = M.Plan(ss, ops[:3], llg)
    plan_nd.launch(3)
    ss.synchronize(); a.record(st); plan_nd.launch(steps_per_eval); b.record(st); ss.synchronize()
    out["step_without_dipole_us"] = a.elapsed_time(b) * 1e3 / steps_per_eval
    out["fno_step_lower_bound_us"] = out["step_without_dipole_us"] + out["fno_us_per_eval"]
    # HBM bound of any implementation of the network: BF16 activations, each
    # layer fused into one read and one write of its W channels (truncated
    # DFTs as GEMMs, spectral inverse + 1x1 + GELU in one pass), lift and
    # projection one pass each over their inputs and outputs
    act = 2.0 * n / nz   # bytes per channel plane (BF16)
    fno_bytes = L * 2 * W * act + (C + W) * act * 2
    out["fno_hbm_bound_us"] = fno_bytes / (measured_peak()[0] * 1e9) * 1e6
    out["fno_hbm_bound_step_us"] = out["step_without_dipole_us"] + out["fno_hbm_bound_us"]
    out["fno_speedup_bound"] = out["plain_step_us"] / out["fno_step_lower_bound_us"]
    out["how"] = ("both networks trained on the plain method over the same seeded random-start runs (seeds 3000..); "
                  "errors: |H0 + net(m_j - m0) - H64(m_j)| / |H64(m_j)| over two windows of each k on the held-out "
                  "film; fno_step_lower_bound_us: the step without the dipole plus one FNO evaluation (no exact "
                  "evaluations, no residual check)")
    return out


# ----------------------------------------------------------------- Runge-Kutta
def run_rk(M, torch, steps=20):
    """The 256x256x8 film stepped by the native RK4 scheme (RungeKutta.lua's
    make_rk_step_function with the deterministic operators as the field and
    the Thermal operator as the kick): spin-steps/s of full RK4 steps (four
    field evaluations each), the steps run as captured graphs (the default)
    and eagerly."""
    ss, ops, _ = build_system(M, 0)
    th = [o for o in ops if isinstance(o, M.Thermal)][0]
    det = [o for o in ops if o is not th]
    rk = M.RungeKutta(ss, "RK4", det, M.LLG.new("Quaternion"), temp=th)
    rk.step(3)
    st = torch.cuda.ExternalStream(ss.stream())
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed():
        ss.synchronize()
        a.record(st)
        rk.step(steps)
        b.record(st)
        ss.synchronize()
        return a.elapsed_time(b) / steps

    g0 = rk.graphSteps()
    ms = timed()
    graph_steps = rk.graphSteps() - g0
    rk.setGraph(False)
    ms_eager = timed()
    with M.profile() as prof:
        rk.step(steps)
        ss.synchronize()
    rk.setGraph(True)
    kern_ms = sum(t for t, c in prof.kernels.values()) / steps
    launches = sum(c for t, c in prof.kernels.values()) / steps
    n = NX * NY * NZ
    return {"workload": WORKLOAD.replace("LLG.Quaternion", "RK4 (LLG.Quaternion stages) + thermal kick"),
            "value": n / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms, "graph_steps": graph_steps,
            "eager_ms_per_step": ms_eager, "kernel_ms_per_step": kern_ms, "launches_per_step": launches,
            "how": "mlb_rk_step, L2 not flushed: each step after the first runs as a captured CUDA graph (the eager "
                   "step's kernels and arguments recorded with their dependent-launch edges, the step graph "
                   "updated in place; results equal the eager steps bit for bit); eager_ms_per_step the same steps "
                   "launched one by one; kernel_ms_per_step sums the eager kernels' own event-timed durations"}


# ----------------------------------------------------------------- FP64 film
def run_fp64_film(M, torch, steps=20):
    """The headline workload with FP64 state (every term, the convolution
    and the LLG update in double, as the reference computes): captured steps,
    no flush."""
    ss, ops, llg = build_system(M, 0, precision="f64")
    M.run(ss, ops, llg, 3)
    plan = M.Plan(ss, ops, llg)
    plan.launch(2)
    st = torch.cuda.ExternalStream(ss.stream())
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ss.synchronize()
    a.record(st)
    plan.launch(steps)
    b.record(st)
    ss.synchronize()
    ms = a.elapsed_time(b) / steps
    n = NX * NY * NZ
    return {"workload": WORKLOAD + " in FP64", "value": n / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms,
            "how": "one captured step per graph launch, back to back, CUDA events; FP64 register split (y,z) "
                   "passes, x passes and fused step"}


# ----------------------------------------------------------------- LongRange2D / Dipole2D
def run_lr2d(M, torch, calls=20):
    """Dipole2D on the 256x256x8 film (builder truncation 25 x 8 x 8 x 8):
    field evaluations per second and the layer-mixing kernel against the
    HBM roofline.  Algorithmic bytes per evaluation: spins in and field out
    (24 B/site), the x passes' spectrum write and read and the mixing pass's
    read and write (4 x 24 B per (kx, y, z)), and the tensor spectrum
    (9 complex per (kx, ky, source, destination))."""
    ss, _, _ = build_system(M, 0)
    dip = M.Dipole2D(ss)
    dip.setTruncation(25, 8, 8, 8)
    dip.apply(ss)
    for _ in range(3):
        dip.apply(ss)
    st = torch.cuda.ExternalStream(ss.stream())
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ss.synchronize()
    a.record(st)
    for _ in range(calls):
        dip.apply(ss)
    b.record(st)
    ss.synchronize()
    ms = a.elapsed_time(b) / calls
    with M.profile() as prof:
        for _ in range(calls):
            dip.apply(ss)
        ss.synchronize()
    n = NX * NY * NZ
    K = (NX // 2 + 1) * NY * NZ
    q_bytes = 72 * NZ * K
    total = 24 * n + 96 * K + q_bytes
    kern = {k: {"avg_us": 1e3 * t / c, "launches": c} for k, (t, c) in prof.kernels.items()}
    out = {"workload": "Dipole2D (layer-pair tensors, periodic in-plane) on the 256x256x8 film, FP32",
           "evaluations_per_s": 1e3 / ms, "ms_per_evaluation": ms,
           "algorithmic_bytes_per_evaluation": total, "achieved_gbs": total / (ms * 1e-3) / 1e9,
           "kernels": kern, "how": "eager mlb_op_apply calls, CUDA events on the system's stream"}
    if "k_lr2d_mix" in kern:
        mix = 48 * K + q_bytes
        out["k_lr2d_mix_gbs"] = mix / (kern["k_lr2d_mix"]["avg_us"] * 1e-6) / 1e9
        out["k_lr2d_mix_frac"] = out["k_lr2d_mix_gbs"] / measured_peak()[0]
    return out


# ----------------------------------------------------------------- DipoleEwald3D
def run_ewald(M, edge=32):
    """The Ewald tensor of an edge^3 simple-cubic lattice (NSites 10: 9261
    real and reciprocal terms per element, 9 elements per site) computed on
    the GPU (one warp per site, all nine components from shared
    transcendentals), against the library's host path
    timed on a sample of elements (the reference evaluates elements one by
    one on the CPU)."""
    ew = M.DipoleEwald3D(edge, edge, edge)
    ew.calculateTensorElement("XX", (1, 0, 0))   # the eta search
    t0 = time.perf_counter()
    ew.tensorArrays()
    gpu_s = time.perf_counter() - t0
    k = 12
    t0 = time.perf_counter()
    for i in range(k):
        ew.calculateTensorElement(["XX", "XY", "ZZ"][i % 3], (i % edge, (3 * i) % edge, (5 * i) % edge))
    host_per = (time.perf_counter() - t0) / k
    n_el = 9 * edge ** 3
    return {"workload": f"DipoleEwald3D tensor of a {edge}^3 simple-cubic lattice, NSites 10, FP64",
            "elements": n_el, "gpu_seconds": gpu_s, "host_seconds_per_element": host_per,
            "host_seconds_estimate": host_per * n_el, "speedup": host_per * n_el / gpu_s,
            "how": "wall clock around mlb_ewald3d_tensor (kernel + copy of 9 x edge^3 doubles) vs "
                   "mlb_ewald3d_element on one host thread"}


# ----------------------------------------------------------------- 256^3 open cube
CUBE_DIMS = (256, 256, 256)
CUBE_WORKLOAD = ("256^3 simple-cubic cube, open boundaries (512^3 padded transform, split (y,z) passes), "
                 "J=1, cubic anisotropy K_c=0.05 (axes x, y, z), g=0.03, T=0.3, alpha=0.05, dt=0.005, "
                 "LLG.Quaternion; spins +z with a seeded 20-degree tilt")


def cube_system(M, prec, spins):
    """The open cube of CUBE_DIMS sites with its operators and integrator."""
    dims = CUBE_DIMS
    n = int(np.prod(dims))
    f, t, j = nn_paths(*dims, pbc=(0, 0, 0))
    ss = M.SpinSystem(*dims, precision=prec)
    ss.setSpinArrays(*spins)
    ss.setAlpha(0.05)
    ss.setTimeStep(0.005)
    ex = M.Exchange(ss)
    ex.addPaths(f, t, j)
    cub = M.AnisotropyCubic(ss)
    cub.addMany(np.arange(n), np.tile([1.0, 0, 0], (n, 1)), np.tile([0, 1.0, 0], (n, 1)),
                np.tile([0.05, 0, 0], (n, 1)))
    th = M.Thermal(ss, M.Random.Philox(5))
    th.setTemperature(0.3)
    dip = M.Dipole(ss)
    dip.setStrength(0.03)
    dip.setOpen(True, True, True)
    return ss, [ex, cub, th, dip], M.LLG.new("Quaternion")


def run_cube_steps(M, nsteps):
    """Profiling driver: eager FP32 steps of the cube."""
    n = int(np.prod(CUBE_DIMS))
    ss, ops, llg = cube_system(M, "f32", tilted_spins(n, 5, deg=20.0))
    for _ in range(nsteps):
        M.run(ss, ops, llg, 1)
    ss.synchronize()


def run_cube(M, torch, steps=20):
    """Configuration 5 on one GPU: FP32 and FP64 step rates, and the FP32
    fields and energies of one state against the FP64 run's (both from the
    same spins: the FP64 state after 2 steps, rounded to FP32)."""
    dims = CUBE_DIMS
    n = int(np.prod(dims))
    s0 = tilted_spins(n, 5, deg=20.0)
    build = lambda prec, spins: cube_system(M, prec, spins)   # noqa: E731

    def timed(ss, fn, k):
        st = torch.cuda.ExternalStream(ss.stream())
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ss.synchronize()
        a.record(st)
        fn(k)
        b.record(st)
        ss.synchronize()
        return a.elapsed_time(b) / k

    d, dops, dl = build("f64", s0)
    M.run(d, dops, dl, 2)
    f64_ms = timed(d, lambda k: M.run(d, dops, dl, k), 3)
    x, y, z, _ = d.spinArrays()
    g, gops, gl = build("f32", np.stack([x, y, z]))
    for ss in (d, g):
        ops = dops if ss is d else gops
        ss.resetFields()
        for op in ops[:2] + ops[3:]:
            op.apply(ss)
        ss.sumFields()
    hd, hg = np.stack(d.fieldArrays("Dipole")), np.stack(g.fieldArrays("Dipole"))
    out = {"workload": CUBE_WORKLOAD, "sites": n,
           "dipole_field_rel_err_f32_vs_f64": float(np.linalg.norm(hg - hd) / np.linalg.norm(hd)), "energy_rel_err": {}}
    for nm in ("Exchange", "CubicAnisotropy", "Dipole"):
        ed, eg = d.fieldDot(nm), g.fieldDot(nm)
        out["energy_rel_err"][nm] = abs(eg - ed) / abs(ed)
    del d, dops, hd, hg
    M.run(g, gops, gl, 3)
    f32_ms = timed(g, lambda k: M.run(g, gops, gl, k), steps)
    out["f32"] = {"value": n / (f32_ms * 1e-3), "ms_per_step": f32_ms}
    out["f64"] = {"value": n / (f64_ms * 1e-3), "ms_per_step": f64_ms}
    out["l2"] = "working set several GB: larger than L2 (no flush)"
    return out


# ----------------------------------------------------------------- algorithmic bytes
def algorithmic_bytes():
    """Per-launch algorithmic bytes of each kernel, split from the per
    spin-step figure B = 36 + 24 + (K/N)(24 + 48*2) with K = (Px/2+1)*Py*Pz:
    fused stencil/LLG 36 B/site; forward x pass 12 B/site + 24 B/k;
    (y,z) pass with the tensor multiply 24+24+24 B/k; inverse x pass 24 B/k
    + 12 B/site.  The fused x pass (inverse x, step, forward x of the new
    spins) carries the three: 48 B/k + 60 B/site."""
    n = NX * NY * NZ
    Px, Py, Pz = NX, NY, 16
    Kk = (Px // 2 + 1) * Py * Pz
    return {
        "k_fused_step": 36 * n,
        "k_conv_fx": 12 * n + 24 * Kk,
        "k_conv_yz": 72 * Kk,
        "k_conv_ix": 24 * Kk + 12 * n,
        "k_xstep": 48 * Kk + 60 * n,
    }, (36 + 24) * n + Kk * (24 + 48 * 2), n, Kk


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic():
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(p) as f:
            return json.load(f)
    except Exception:
        return {}


# ----------------------------------------------------------------- clocks
class ClockSampler:
    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def wait_first(self, timeout_s=5.0):
        """Until the sampler has produced its first line (nvidia-smi takes a
        moment to start)."""
        t_end = time.perf_counter() + timeout_s
        while self.proc and not self.lines and time.perf_counter() < t_end:
            time.sleep(0.01)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------- CPU baseline (oracle)
def _cpu_worker(args):
    seed, steps = args
    import oracle as O
    n = NX * NY * NZ
    ss = O.SpinSystem(NX, NY, NZ)
    ss.set_spins(*tilted_spins(n, seed))
    ss.alpha, ss.dt = ALPHA, DT
    f, t, j = nn_paths(NX, NY, NZ)
    sites = np.arange(n, dtype=np.int32)
    ani = (sites, np.tile([0, 0, 1.0], (n, 1)), np.full(n, K_ANI))
    lr = O.LongRange(NX, NY, NZ, O.dipole_tensor(NX, NY, NZ))
    rng = O.MT(1000 + seed)
    O.run_steps(ss, 1, paths=(f, t, j), ani=ani, T=TEMP, rng=rng, B=(BX, 0, 0), lr=lr, g=G_DIP,
                llg="Quaternion")
    t0 = time.perf_counter()
    O.run_steps(ss, steps, paths=(f, t, j), ani=ani, T=TEMP, rng=rng, B=(BX, 0, 0), lr=lr, g=G_DIP,
                llg="Quaternion")
    return time.perf_counter() - t0


def cpu_baseline(procs=1, target_s=15.0):
    """The FP64 CPU restatement of the reference's modules on the host cores:
    `procs` independent replicas in parallel (one process each)."""
    import multiprocessing as mp
    import oracle as O  # noqa: F401  (builds liboracle.so if needed)
    ctx = mp.get_context("spawn")
    with ctx.Pool(1) as pool:
        t1 = pool.map(_cpu_worker, [(0, 1)])[0]
    steps = int(max(2, min(200, target_s / max(t1, 1e-6))))
    with ctx.Pool(procs) as pool:
        times = pool.map(_cpu_worker, [(r, steps) for r in range(procs)])
    n = NX * NY * NZ
    val = procs * n * steps / max(times)
    return {"value": val, "unit": UNIT, "cores": procs, "kind": "port",
            "sample": f"{steps} steps of the full {NX}x{NY}x{NZ} workload per process, {procs} process(es), "
                      f"FP64 C restatement (gcc -O2), Mersenne-Twister thermal noise, own FFT in place of FFTW"}


# ----------------------------------------------------------------- ranks
def reduce_max(v, dist):
    """The maximum of v over the process group's ranks (every rank gets it):
    the device time of a weak-scaling run is the slowest rank's."""
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(v)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ----------------------------------------------------------------- main
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=20.0,
                    help="reference arm: seconds of CPU work per process in its bounded sample")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-surrogate", action="store_true", help="skip the learned-surrogate comparison")
    ap.add_argument("--no-cube", action="store_true", help="skip the 256^3 open-cube precision study")
    ap.add_argument("--fno-study", action="store_true",
                    help="only the study of the 4-layer spectral-convolution network (PyTorch) against the library's "
                         "surrogate network; prints its JSON line")
    ap.add_argument("--ncu-steps", type=int, default=0,
                    help="profiling driver: run this many eager steps of the workload and exit (for ncu)")
    ap.add_argument("--ncu-surrogate", type=int, default=0,
                    help="profiling driver: this many surrogate steps on the 512x512x4 film (small random "
                         "network weights, every step after the first a surrogate step) and exit")
    ap.add_argument("--ncu-ensemble", type=int, default=0,
                    help="profiling driver: this many captured steps of the packed ensemble and exit")
    ap.add_argument("--ncu-cube", type=int, default=0,
                    help="profiling driver: this many eager FP32 steps of the open cube (edge --cube-edge) and exit")
    ap.add_argument("--cube-edge", type=int, default=256, help="edge of the cube for --ncu-cube")
    ap.add_argument("--ncu-lr2d", type=int, default=0,
                    help="profiling driver: this many Dipole2D evaluations on the 256x256x8 film and exit")
    ap.add_argument("--ncu-ewald", type=int, default=0,
                    help="profiling driver: the Ewald tensor of an edge^3 simple-cubic lattice (NSites 10) and exit")
    ap.add_argument("--ncu-f64", type=int, default=0,
                    help="profiling driver: this many eager steps of the 256x256x8 film in FP64 and exit")
    ap.add_argument("--ncu-rk4", type=int, default=0,
                    help="profiling driver: this many RK4 steps (+ thermal kick) of the 256x256x8 film and exit")
    args = ap.parse_args()
    if args.ncu_rk4:
        import maglua_b200 as M
        M.init(int(os.environ.get("LOCAL_RANK", "0")))
        ss, ops, _ = build_system(M, 0)
        th = [o for o in ops if isinstance(o, M.Thermal)][0]
        rk = M.RungeKutta(ss, "RK4", [o for o in ops if o is not th], M.LLG.new("Quaternion"), temp=th)
        rk.step(args.ncu_rk4)
        ss.synchronize()
        return
    if args.fno_study:
        import torch
        import maglua_b200 as M
        M.init(int(os.environ.get("LOCAL_RANK", "0")))
        print(json.dumps({"fno_study": run_fno_study(M, torch)}), flush=True)
        return
    if args.ncu_f64:
        import maglua_b200 as M
        M.init(int(os.environ.get("LOCAL_RANK", "0")))
        ss, ops, llg = build_system(M, 0, precision="f64")
        for _ in range(args.ncu_f64):
            M.run(ss, ops, llg, 1)
        ss.synchronize()
        return
    if args.ncu_lr2d or args.ncu_ewald:
        import maglua_b200 as M
        M.init(int(os.environ.get("LOCAL_RANK", "0")))
        if args.ncu_lr2d:
            ss, _, _ = build_system(M, 0)
            dip = M.Dipole2D(ss)
            dip.setTruncation(25, 8, 8, 8)
            for _ in range(args.ncu_lr2d):
                dip.apply(ss)
            ss.synchronize()
        else:
            M.DipoleEwald3D(args.ncu_ewald, args.ncu_ewald, args.ncu_ewald).tensorArrays()
        return
    if args.ncu_cube:
        import maglua_b200 as M
        M.init(int(os.environ.get("LOCAL_RANK", "0")))
        global CUBE_DIMS
        CUBE_DIMS = (args.cube_edge,) * 3
        run_cube_steps(M, args.ncu_cube)
        return
    if args.ncu_steps or args.ncu_surrogate or args.ncu_ensemble:
        import maglua_b200 as M
        M.init(int(os.environ.get("LOCAL_RANK", "0")))
        if args.ncu_steps:
            ss, ops, llg = build_system(M, 0)
            for _ in range(args.ncu_steps):
                M.run(ss, ops, llg, 1)
            ss.synchronize()
        if args.ncu_surrogate:
            dims = SUR_DIMS
            n = int(np.prod(dims))
            ss = M.SpinSystem(*dims)
            ss.setSpinArrays(*tilted_spins(n, 9, deg=30.0))
            ss.setAlpha(0.02)
            ss.setTimeStep(0.005)
            ex = M.Exchange(ss)
            ex.addPaths(*nn_paths(*dims))
            dip = M.Dipole(ss)
            dip.setStrength(0.05)
            ops, llg = [ex, dip], M.LLG.new("Quaternion")
            S = M.Surrogate(dip, (16, 16), 3)   # the surrogate leg's network
            r = np.random.default_rng(9)
            W = r.normal(size=(49, S.C, S.C)) * 1e-3
            R = (r.normal(size=(16, 16, S.C, S.C)) + 1j * r.normal(size=(16, 16, S.C, S.C))) * 1e-3
            S.setParams(W, R)
            S.setSchedule(1 << 30, tol=1e30, eps=1e-6)
            S.attach(ss)
            for _ in range(args.ncu_surrogate):
                M.run(ss, ops, llg, 1)
            S.detach(ss)
            ss.synchronize()
        if args.ncu_ensemble:
            import torch
            _time_ensemble(M, torch, ensemble_dims(), 0.02, args.ncu_ensemble, 3)
        return
    args.warmup = max(3, args.warmup)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        procs = os.cpu_count() or 1
        cb = cpu_baseline(procs=procs, target_s=args.cpu_seconds)
        line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": WORKLOAD, "replicas": procs, "parallelism": f"replicas{procs}"},
                "cpu_baseline": cb,
                "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))

    import maglua_b200 as M
    M.init(local)
    ss, ops, llg = build_system(M, seed=rank)
    stream = torch.cuda.ExternalStream(ss.stream())
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    sweep = torch.ones(FLUSH_BYTES // 8, dtype=torch.float32, device="cuda")
    n = NX * NY * NZ

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    # warm-up (tensor setup, graph capture)
    M.run(ss, ops, llg, args.warmup)
    plan_nt = M.Plan(ss, ops, llg, timing=False)
    plan_nt.launch(2)
    ss.synchronize()

    def flush_l2():
        with torch.cuda.stream(stream):
            flush.zero_()          # write 1 GiB (> L2)
            sweep.sum()            # read 512 MiB: evicts the dirty flush lines

    # timed region: one captured step per launch, per-step events, L2 flush
    # (write then read sweep) before every step, outside the events
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    # clocks: nvidia-smi samples every 50 ms, longer than the timed region,
    # so the sampling window runs from a quarter second of load (L2 flush
    # sweeps) before the timed region to a quarter second after it
    clocks = ClockSampler(local)
    clocks.start()
    clocks.wait_first()

    def load(seconds):
        t_end = time.perf_counter() + seconds
        while time.perf_counter() < t_end:
            flush_l2()
            ss.synchronize()

    load(0.25)
    barrier()
    for k in range(args.steps):
        flush_l2()
        evs[k][0].record(stream)
        plan_nt.launch(1)
        evs[k][1].record(stream)
    ss.synchronize()
    barrier()
    load(0.25)
    clk = clocks.stop()
    clk["window"] = "0.25 s of load before the timed region to 0.25 s after it (samples every 50 ms)"
    step_ms = [a.elapsed_time(b) for a, b in evs]
    total_ms = sum(step_ms)
    if dist:
        total_ms = reduce_max(total_ms, dist)
    value = world * n * args.steps / (total_ms * 1e-3)

    # per-kernel times: the same step captured with event nodes around each
    # kernel (the nodes add a little time of their own), same flushes
    plan = M.Plan(ss, ops, llg, timing=True)
    plan.launch(2)
    kern_ms = {}
    kern_n = {}
    ksteps = min(args.steps, 200)
    for k in range(ksteps):
        flush_l2()
        plan.launch(1)
        for nm, ms in plan.kernelTimes().items():
            kern_ms[nm] = kern_ms.get(nm, 0.0) + ms
            kern_n[nm] = kern_n.get(nm, 0) + 1
    ss.synchronize()

    # device timeline of the same flushed steps with the step's dependent
    # launches kept (no event nodes): each pass from its first CTA released
    # from the dependency wait to its last CTA's end (%globaltimer)
    plan_dt = M.Plan(ss, ops, llg, timing=2)
    plan_dt.launch(2)
    plan_dt.deviceTimes()
    dev_us = {}
    for k in range(ksteps):
        flush_l2()
        plan_dt.launch(1)
        for nm, us in plan_dt.deviceTimes().items():
            dev_us.setdefault(nm, []).append(us)
    ss.synchronize()
    del plan_dt

    # steady state without flushes (L2-resident state), same plan
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    e0.record(stream)
    plan_nt.launch(args.steps)
    e1.record(stream)
    ss.synchronize()
    ss_ms = e0.elapsed_time(e1)

    # the same film without the dipole operator (the Amdahl bound of any
    # dipole surrogate): the same plan shape, back to back, no flush
    ss_nd, ops_nd, llg_nd = build_system(M, seed=rank)
    plan_nd = M.Plan(ss_nd, ops_nd[:4], llg_nd)
    plan_nd.launch(3)
    st_nd = torch.cuda.ExternalStream(ss_nd.stream())
    e0.record(st_nd)
    plan_nd.launch(args.steps)
    e1.record(st_nd)
    ss_nd.synchronize()
    nodip_ms = e0.elapsed_time(e1)
    del plan_nd, ss_nd, ops_nd

    # end to end through the C ABI with host buffers
    hx, hy, hz = (torch.empty(n, dtype=torch.float32).pin_memory().numpy() for _ in range(3))
    s0 = tilted_spins(n, rank)
    hx[:], hy[:], hz[:] = s0
    # warm-up: the netMoment slot graphs of both spin buffers
    for k in range(8):
        plan_nt.launch(1)
        ss.netMomentAsync(k % 4)
        ss.netMomentWait(k % 4)
    ss.synchronize()

    def e2e_run():
        barrier()
        t0 = time.perf_counter()
        ss.uploadF32(hx, hy, hz)   # the spins; the moment magnitudes stay (all 1)
        # each step's netMoment is read on the host; the read of step k waits
        # while steps k + 1 and k + 2 are already queued on the GPU
        depth = 2
        for k in range(args.steps):
            plan_nt.launch(1)
            ss.netMomentAsync(k % 4)
            if k >= depth:
                ss.netMomentWait((k - depth) % 4)
        # the final spins' download is queued behind the last step before the
        # host waits for the last two steps' moments
        ss.downloadF32(hx, hy, hz)
        for k in range(max(0, args.steps - depth), args.steps):
            ss.netMomentWait(k % 4)
        ss.synchronize()
        return time.perf_counter() - t0

    # the host loop shares its cores with other work on the box: the median
    # of three complete runs
    e2e_runs = sorted(e2e_run() for _ in range(3))
    e2e_s = e2e_runs[1]

    # the same run split into its parts (each synchronised on its own): the
    # one-off upload and download, and the per-step API loop
    def e2e_parts():
        barrier()
        t0 = time.perf_counter()
        ss.uploadF32(hx, hy, hz)   # the spins; the moment magnitudes stay (all 1)
        ss.synchronize()
        t1 = time.perf_counter()
        depth = 2
        for k in range(args.steps):
            plan_nt.launch(1)
            ss.netMomentAsync(k % 4)
            if k >= depth:
                ss.netMomentWait((k - depth) % 4)
        for k in range(max(0, args.steps - depth), args.steps):
            ss.netMomentWait(k % 4)
        ss.synchronize()
        t2 = time.perf_counter()
        ss.downloadF32(hx, hy, hz)
        ss.synchronize()
        t3 = time.perf_counter()
        return t1 - t0, t2 - t1, t3 - t2

    parts = sorted((e2e_parts() for _ in range(3)), key=lambda p: p[1])[1]
    if dist:
        e2e_s = reduce_max(e2e_s, dist)
    e2e_val = world * n * args.steps / e2e_s

    batched = run_batched(M, torch, args.steps, args.warmup)
    surrogate = run_surrogate(M, torch, min(args.steps, 200)) if not args.no_surrogate else None
    cube = run_cube(M, torch) if not args.no_cube else None
    rk = run_rk(M, torch)
    lr2d = run_lr2d(M, torch)
    fp64 = run_fp64_film(M, torch)
    ewald = run_ewald(M)

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return

    per_launch, bytes_step, _, Kk = algorithmic_bytes()
    peak, peak_kind = measured_peak()
    traffic = ncu_traffic()
    kern = {k: (kern_ms[k], kern_n[k]) for k in kern_ms if k in per_launch}
    dom = max(kern, key=lambda k: kern[k][0]) if kern else None
    roof = None
    kernels_out = {}
    for k, (ms, nl) in kern.items():
        avg = ms / nl
        ach = per_launch[k] / (avg * 1e-3) / 1e9
        kernels_out[k] = {"avg_us": avg * 1e3, "launches": nl, "share": ms / sum(v[0] for v in kern.values()),
                          "algorithmic_bytes": per_launch[k], "achieved_gbs": ach}
    if dom:
        ms, nl = kern[dom]
        avg = ms / nl
        ach = per_launch[dom] / (avg * 1e-3) / 1e9
        tr = traffic.get(dom)
        roof = {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": peak, "unit": "GB/s",
                "frac": ach / peak, "peak_kind": peak_kind + " (burst copy)",
                "traffic": tr, "algorithmic_bytes_per_launch": per_launch[dom],
                "timing": "CUDA event nodes around the kernel in a timing copy of the captured step (the "
                          "kernel's own launch latency included)"}
        if dev_us.get(dom):
            dus = float(np.median(dev_us[dom]))
            dach = per_launch[dom] / (dus * 1e-6) / 1e9
            roof["device_timeline"] = {
                "us": dus, "achieved": dach, "frac": dach / peak,
                "how": "median over the flushed timed steps of the captured step with its dependent launches "
                       "(no event nodes): %globaltimer from the first CTA released from the dependency wait to "
                       "the last CTA's end"}
    for k, v in dev_us.items():
        if k in kernels_out:
            kernels_out[k]["device_us"] = float(np.median(v))
    step_bytes_gbs = bytes_step / (total_ms / args.steps * 1e-3) / 1e9
    cpu = None
    if not args.no_cpu and world == 1:
        cpu = cpu_baseline(procs=1, target_s=15.0)
    # our kernels in the timed region: the step kernels, counted per step in
    # the timing pass (the fused x pass also writes the next step's device
    # block, so a captured step has no other kernel)
    launches = int(round(sum(kern_n.values()) / ksteps * args.steps))
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "sites_per_gpu": n, "parallelism": f"replicas{world}",
                   "l2": "flushed between steps (1 GiB write then a 512 MiB read sweep, excluded by per-step CUDA events)",
                   "llg": "Quaternion", "path": "plain fused FFT path"},
        "clocks": clk,
        "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": (12 * n) / args.steps,
                "d2h_bytes_per_step": 48 + (12 * n) / args.steps, "steps": args.steps,
                "how": "C-ABI calls from host: pinned FP32 upload of the spins, per step mlb_plan_launch(1) + netMoment of that "
                       "step read into pinned memory and waited for once two more steps are queued, final download; median of "
                       "three complete runs; the upload and download are once per run, so the figure depends on "
                       "the step count",
                "parts": {"upload_ms": parts[0] * 1e3, "loop_ms_per_step": parts[1] * 1e3 / args.steps,
                          "download_ms": parts[2] * 1e3,
                          "loop_value": n / (parts[1] / args.steps),
                          "how": "the same run with a synchronisation after the upload and before the download: "
                                 "upload, the per-step API loop (launch + netMoment read), download"}},
        "gpu_launches": launches,
        "roofline": roof,
        "kernels": kernels_out,
        "step_roofline": {"bytes_per_spin_step": bytes_step / n, "achieved_gbs": step_bytes_gbs,
                          "frac": step_bytes_gbs / peak, "K_points": Kk},
        "steady_state_l2_resident": {"value": n * args.steps / (ss_ms * 1e-3), "ms_per_step": ss_ms / args.steps,
                                     "how": "the same plan launched for all the steps back to back (carried steps four to a graph), no flush"},
        "film_without_dipole": {"ms_per_step": nodip_ms / args.steps, "amdahl_ceiling": ss_ms / nodip_ms,
                                "how": "the film's captured step without the Dipole operator, back to back, no flush: "
                                       "the bound on what replacing the dipole evaluation by anything can gain"},
        "cpu_baseline": cpu,
        "plain_vs_surrogate_batched": {
            "batched_vs_plain_one_system_per_replica": batched["plain_one_system_per_replica"]["speedup_of_batched"],
            "batched_value": batched["value"],
            "plain_one_system_per_replica_value": batched["plain_one_system_per_replica"]["value"],
            "ensemble_no_dipole_ceiling": batched["without_dipole"]["amdahl_ceiling"],
            "film_no_dipole_ceiling": ss_ms / nodip_ms,
            "surrogate_film_speedup_by_k": ({k: v["speedup_vs_plain"] for k, v in surrogate["by_k"].items()}
                                            if surrogate else None),
            "surrogate_film_field_err_vs_fp64_by_k": ({k: v["field_rel_err_vs_fp64_mean"]
                                                       for k, v in surrogate["by_k"].items()} if surrogate else None),
            "how": "configuration 3's replicas: the packed ensemble (exact FFT dipole, FP32) against the same "
                   "replicas through the plain path one SpinSystem each; the learned surrogate on configuration "
                   "4's film against that film's plain path, its field error against the FP64 field; the "
                   "no-dipole ceilings bound what any dipole surrogate can gain on each workload"},
        "batched_ensemble": batched,
        "surrogate": surrogate,
        "cube_256": cube,
        "rk4": rk,
        "fp64_film": fp64,
        "dipole2d": lr2d,
        "ewald3d": ewald,
    }
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
