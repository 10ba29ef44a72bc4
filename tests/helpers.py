"""Shared set-up for the parity tests: one configuration built twice, on the
FP64 oracle and on the CUDA product, from the same seeded inputs."""
import numpy as np

import oracle as O


def random_spins(n, seed, lengths=False):
    """Spins uniform on the sphere (normalised Gaussians); optional random
    lengths in [0.5, 1.5]."""
    r = np.random.default_rng(seed)
    v = r.normal(size=(3, n))
    v /= np.linalg.norm(v, axis=0)
    if lengths:
        v *= r.uniform(0.5, 1.5, size=n)
    return v


def tilted_spins(n, seed, deg=5.0):
    """+z with a seeded tilt of `deg` degrees and uniform azimuth."""
    r = np.random.default_rng(seed)
    phi = r.uniform(0, 2 * np.pi, n)
    th = np.deg2rad(deg)
    return np.stack([np.sin(th) * np.cos(phi), np.sin(th) * np.sin(phi), np.full(n, np.cos(th))])


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


class Pair:
    """Oracle and product objects for the same lattice."""

    def __init__(self, nx, ny, nz, spins, alpha=0.1, dt=0.01, gamma=1.0, precision="f32"):
        import maglua_b200 as M
        self.M = M
        self.dims = (nx, ny, nz)
        self.n = nx * ny * nz
        self.o = O.SpinSystem(nx, ny, nz)
        self.o.set_spins(*spins)
        self.o.alpha, self.o.dt, self.o.gamma = alpha, dt, gamma
        self.g = M.SpinSystem(nx, ny, nz, precision=precision)
        self.g.setSpinArrays(*spins)
        self.g.setAlpha(alpha)
        self.g.setTimeStep(dt)
        self.g.setGamma(gamma)
        self.ops = []      # product operators
        self.oapply = []   # oracle callables f(ss)

    def exchange(self, J=1.0, pbc=(1, 1, 1), normalize=True, paths=None):
        M = self.M
        f, t, j = paths if paths is not None else O.nn_paths(*self.dims, J=J, pbc=pbc)
        ex = M.Exchange(*self.dims)
        ex.normalizeMoments(bool(normalize))
        ex.addPaths(f, t, j)
        self.ops.append(ex)
        self.oapply.append(lambda ss, f=f, t=t, j=j: O.exchange_apply(ss, f, t, j, normalize))
        return ex

    def anisotropy(self, axis=(0, 0, 1), K=0.1):
        M = self.M
        ani = M.Anisotropy(*self.dims)
        ax = np.asarray(axis, float) / np.linalg.norm(axis)
        sites = np.arange(self.n, dtype=np.int32)
        axes = np.tile(ax, (self.n, 1))
        Ks = np.full(self.n, K)
        ani.addMany(sites, axes, Ks)
        self.ops.append(ani)
        self.oapply.append(lambda ss: O.anisotropy_apply(ss, sites, axes, Ks))
        return ani

    def cubic(self, K=(0.05, 0.0, 0.0), quirk=True):
        M = self.M
        cub = M.AnisotropyCubic(*self.dims)
        cub.setQuirks(quirk)
        sites = np.arange(self.n, dtype=np.int32)
        a1 = np.tile([1.0, 0, 0], (self.n, 1))
        a2 = np.tile([0, 1.0, 0], (self.n, 1))
        KK = np.tile(K, (self.n, 1))
        cub.addMany(sites, a1, a2, KK)
        rc, axes = O.cubic_axes([1.0, 0, 0], [0, 1.0, 0])
        AX = np.tile(axes, (self.n, 1))
        self.ops.append(cub)
        self.oapply.append(lambda ss: O.anisotropy_cubic_apply(ss, sites, AX, KK, quirk=quirk))
        return cub

    def zeeman(self, B):
        M = self.M
        z = M.AppliedField(*self.dims)
        z.set(*B)
        self.ops.append(z)
        self.oapply.append(lambda ss, B=tuple(B): O.zeeman_apply(ss, B))
        return z

    def dipole(self, g, open_xy=False):
        M = self.M
        nx, ny, nz = self.dims
        dip = M.Dipole(*self.dims)
        dip.setStrength(g)
        if open_xy:
            dip.setOpen(True, True, True)
            self.ops.append(dip)
            self.oapply.append(lambda ss: _open_dipole_oracle(ss, g))
        else:
            T6 = O.dipole_tensor(nx, ny, nz)
            lr = O.LongRange(nx, ny, nz, T6)
            self._lr = lr
            self.ops.append(dip)
            self.oapply.append(lambda ss: lr.apply(ss, g))
        return dip

    def step_oracle(self, llg):
        self.o.reset_fields()
        for f in self.oapply:
            f(self.o)
        self.o.sum_fields()
        llg.apply(self.o)

    def step_gpu(self, llg):
        self.g.resetFields()
        for op in self.ops:
            op.apply(self.g)
        self.g.sumFields()
        llg.apply(self.g)


def _open_dipole_oracle(ss, g):
    h = O.dipole_direct(ss, g, periodic=(0, 0, 0))
    views = ss.field_views("Dipole")
    for c in range(3):
        views[c][:] = h[c]
    ss.set_slot_used("Dipole", True)
