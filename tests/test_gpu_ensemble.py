"""Packed ensembles beyond one shared parameter set: per-replica temperature
and applied field (start and sweep), size classes outside the power-of-two
fast passes (generic passes replica by replica), and the tuner's choices and
cache file.  Each replica is compared with the same lattice run as a single
SpinSystem through the operator API (itself checked against the oracle in
test_gpu_parity.py and test_gpu_physics.py).  Reference batching:
SpinOperation::apply(SpinSystem**, n) (M/cpu/core/spinoperation.cpp:288-300)
and the CUDA build's batched LLG (M/cuda/llg_cuda/llgcartesian.cu:133)."""
import os

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


def _single(M, dims, s, cfg, nsteps, B, dB, T=0.0, seed=0):
    n = int(np.prod(dims))
    ss = M.SpinSystem(*dims)
    ss.setSpinArrays(*s)
    ss.setAlpha(cfg["alpha"])
    ss.setTimeStep(cfg["dt"])
    ex = M.Exchange(ss)
    ex.addPaths(*O.nn_paths(*dims, pbc=(0, 0, 0)))
    ani = M.Anisotropy(ss)
    ani.addMany(np.arange(n), np.tile([0, 0, 1.0], (n, 1)), np.full(n, cfg["K"]))
    z = M.AppliedField(ss)
    z.set(*B)
    z.setSweep(*dB)
    ops = [ex, ani, z]
    if cfg["g"]:
        dip = M.Dipole(ss)
        dip.setOpen(True, True, True)
        dip.setStrength(cfg["g"])
        ops.append(dip)
    l = M.LLG.new(cfg["llg"])
    M.run(ss, ops, l, nsteps)
    return np.stack(ss.spinArrays()[:3])


CFG = dict(alpha=0.1, dt=0.01, K=0.2, g=0.05, llg="Cartesian")


def _ensemble(M, dims, cfg, T=0.0, seed=0):
    e = M.Ensemble(dims)
    e.configure(alpha=cfg["alpha"], dt=cfg["dt"], J=1.0, pbc=(0, 0, 0), K=cfg["K"], axis=(0, 0, 1.0), T=T,
                seed=seed, B=(0, 0, 0), dB=(0, 0, 0), g=cfg["g"], open_xy=True, llg=cfg["llg"])
    return e


def test_per_replica_applied_field_and_sweep(M):
    dims = [(16, 16, 4), (8, 8, 2), (16, 16, 4), (32, 16, 1)]
    fields = [((0.0, 0.1, -0.2), (0.0, 0.0, -1e-3)), ((0.05, 0.0, 0.0), (1e-3, 0.0, 0.0)),
              ((0.0, 0.0, 0.3), (0.0, 2e-3, 0.0)), ((-0.1, 0.0, 0.1), (0.0, 0.0, 0.0))]
    e = _ensemble(M, dims, CFG)
    starts = [random_spins(int(np.prod(d)), 90 + r) for r, d in enumerate(dims)]
    for r, (s, (B, dB)) in enumerate(zip(starts, fields)):
        e.setSpins(r, *s)
        e.setReplicaParams(r, 0.0, B, dB)
    e.run(10)
    e.run(20)
    for r, (d, (B, dB)) in enumerate(zip(dims, fields)):
        ref = _single(M, d, starts[r], CFG, 30, B, dB)
        got = np.stack(e.spins(r))
        assert np.abs(got - ref).max() <= 1e-5, (r, np.abs(got - ref).max())
        np.testing.assert_allclose(e.replicaField(r), np.array(B) + 30 * np.array(dB), rtol=0, atol=1e-12)


def test_per_replica_temperature(M):
    """Replicas at T = 0 in an ensemble whose other replicas are thermal step
    exactly as deterministic single systems; thermal replicas differ from
    them and from each other, with unit moments kept."""
    dims = [(16, 16, 4)] * 4
    n = 16 * 16 * 4
    e = _ensemble(M, dims, CFG, T=0.0, seed=11)
    s0 = random_spins(n, 5)
    for r in range(4):
        e.setSpins(r, *s0)
    e.setReplicaParams(1, 0.4, (0, 0, 0), (0, 0, 0))
    e.setReplicaParams(3, 0.4, (0, 0, 0), (0, 0, 0))
    e.run(25)
    ref = _single(M, dims[0], s0, CFG, 25, (0, 0, 0), (0, 0, 0))
    for r in (0, 2):
        assert np.abs(np.stack(e.spins(r)) - ref).max() <= 1e-5
    a, b = np.stack(e.spins(1)), np.stack(e.spins(3))
    assert np.abs(a - ref).max() > 1e-3 and np.abs(a - b).max() > 1e-3
    assert np.allclose(np.sqrt((a ** 2).sum(0)), 1.0, atol=1e-5)


def test_size_classes_outside_fast_passes(M):
    """Classes whose padded grid is outside the power-of-two fast kernels
    (x padded to 8 < 16; z padded to 64 > 32) run the generic passes replica
    by replica, next to fast classes, in the same captured step."""
    dims = [(4, 6, 2), (16, 16, 4), (4, 6, 2), (6, 5, 20), (8, 8, 2)]
    e = _ensemble(M, dims, CFG)
    starts = [random_spins(int(np.prod(d)), 120 + r) for r, d in enumerate(dims)]
    for r, s in enumerate(starts):
        e.setSpins(r, *s)
        e.setReplicaParams(r, 0.0, (0.0, 0.02 * r, -0.1), (0.0, 0.0, -1e-3))
    e.run(15)
    info = e.configInfo()
    assert info["classes"] == 4 and info["generic_classes"] == 2
    for r, d in enumerate(dims):
        ref = _single(M, d, starts[r], CFG, 15, (0.0, 0.02 * r, -0.1), (0.0, 0.0, -1e-3))
        got = np.stack(e.spins(r))
        assert np.abs(got - ref).max() <= 1e-5, (d, np.abs(got - ref).max())


def test_tuner_log_and_cache_file(M, tmp_path, monkeypatch):
    cache = tmp_path / "tune.txt"
    monkeypatch.setenv("MLB_TUNE_CACHE", str(cache))
    # a class set no other test tunes in this process
    dims = [(24, 24, 3), (12, 12, 6), (24, 24, 3)]
    starts = [random_spins(int(np.prod(d)), 140 + r) for r, d in enumerate(dims)]
    outs = []
    for attempt in range(2):
        e = _ensemble(M, dims, dict(CFG, llg="Quaternion"))
        for r, s in enumerate(starts):
            e.setSpins(r, *s)
        e.run(12)
        outs.append([np.stack(e.spins(r)) for r in range(len(dims))])
        log = e.tuneLog()
        if attempt == 0:
            assert "fused step" in log and "chosen" in log
    assert cache.exists() and len(cache.read_text().strip().splitlines()) == 1
    for a, b in zip(*outs):
        np.testing.assert_array_equal(a, b)
    # a fresh process reads the file instead of timing again
    import subprocess
    import sys
    code = ("import sys; sys.path.insert(0, %r); import numpy as np, maglua_b200 as M; M.init(0);"
            "e = M.Ensemble(%r); e.configure(alpha=0.1, dt=0.01, K=0.2, g=0.05, llg='Quaternion');"
            "[e.setSpins(r, np.zeros(int(np.prod(d))), np.zeros(int(np.prod(d))), np.ones(int(np.prod(d))))"
            " for r, d in enumerate(%r)]; e.run(1); print(e.tuneLog())") % (
        os.path.dirname(os.path.dirname(os.path.abspath(__file__))), dims, dims)
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300,
                         env=dict(os.environ, MLB_TUNE_CACHE=str(cache)))
    assert out.returncode == 0, out.stderr
    assert "cached choices" in out.stdout
