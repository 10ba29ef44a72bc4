"""CPU checks of the surrogate network's FP64 reference (oracle/surrogate.py):
its analytic gradients against central finite differences, and its
spectral branch against a direct double sum over the retained modes."""
import numpy as np

from oracle import surrogate as OS

DIMS = (8, 6, 2)
C = 6
MX, MY, RAD = 3, 4, 1


def _setup(seed):
    r = np.random.default_rng(seed)
    n = DIMS[0] * DIMS[1] * DIMS[2]
    W = r.normal(size=((2 * RAD + 1) ** 2, C, C))
    R = r.normal(size=(MX, MY, C, C)) + 1j * r.normal(size=(MX, MY, C, C))
    x = r.normal(size=(3, n))
    t = r.normal(size=(3, n))
    return W, R, x, t


def _loss(x, t, W, R):
    return OS.loss_and_gradients(x, t, W, R, DIMS, MX, MY, RAD)[0]


def test_gradients_match_finite_differences():
    W, R, x, t = _setup(1)
    L, dW, dR, _ = OS.loss_and_gradients(x, t, W, R, DIMS, MX, MY, RAD)
    h = 1e-6
    r = np.random.default_rng(2)
    for _ in range(6):
        o, a, b = r.integers(0, W.shape[0]), r.integers(0, C), r.integers(0, C)
        Wp, Wm = W.copy(), W.copy()
        Wp[o, a, b] += h
        Wm[o, a, b] -= h
        fd = (_loss(x, t, Wp, R) - _loss(x, t, Wm, R)) / (2 * h)
        assert abs(fd - dW[o, a, b]) <= 1e-6 * max(1.0, abs(fd))
    for _ in range(6):
        kx, j, a, b = r.integers(0, MX), r.integers(0, MY), r.integers(0, C), r.integers(0, C)
        for part, unit in ((np.real, 1.0), (np.imag, 1j)):
            Rp, Rm = R.copy(), R.copy()
            Rp[kx, j, a, b] += h * unit
            Rm[kx, j, a, b] -= h * unit
            fd = (_loss(x, t, W, Rp) - _loss(x, t, W, Rm)) / (2 * h)
            assert abs(fd - part(dR[kx, j, a, b])) <= 1e-6 * max(1.0, abs(fd))


def test_spectral_branch_direct_sum():
    W, R, x, _ = _setup(3)
    W0 = np.zeros_like(W)
    got = OS.to_channels(OS.forward(x, W0, R, DIMS, MX, MY, RAD), DIMS)
    X = OS.to_channels(x, DIMS)
    nx, ny = DIMS[0], DIMS[1]
    yy, xx = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    ref = np.zeros_like(got)
    for kx in range(MX):
        w = 1.0 if kx == 0 else 2.0
        for j, ky in enumerate(OS.ky_list(ny, MY)):
            ph = np.exp(-2j * np.pi * (kx * xx / nx + ky * yy / ny))
            Xh = np.array([np.sum(X[c] * ph) for c in range(C)])
            A = R[kx, j] @ Xh
            ref += w / (nx * ny) * np.real(A[:, None, None] * np.conj(ph)[None])
    assert np.abs(got - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max())
