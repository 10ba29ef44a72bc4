"""Generate the golden fixtures in this folder from the FP64 oracle.

    python tests/golden/make_golden.py

The reference publishes no numeric fixtures and cannot be built here (no Lua
5.1, no FFTW3), so these pin the oracle's outputs on seeded inputs.  The
oracle is checked against published vectors and closed forms in
tests/test_oracle.py; the GPU parity tests read these fixtures.

Workload (the CPU-runnable configuration): 32x32x1 simple-cubic film of unit
spins, periodic in x/y, spins uniform on the sphere (seed 1), nearest-
neighbour exchange J=1, anisotropy K=0.1 along z, dipole g=0.01 (periodic
images, cut-off 1000), LLG alpha=0.1, dt=0.01, T=0.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402

NX, NY, NZ = 32, 32, 1
J, K, G = 1.0, 0.1, 0.01
ALPHA, DT = 0.1, 0.01


def c1_spins(seed=1):
    r = np.random.default_rng(seed)
    v = r.normal(size=(3, NX * NY * NZ))
    return v / np.linalg.norm(v, axis=0)


def c1_setup():
    n = NX * NY * NZ
    ss = O.SpinSystem(NX, NY, NZ)
    ss.set_spins(*c1_spins())
    ss.alpha, ss.dt = ALPHA, DT
    paths = O.nn_paths(NX, NY, NZ, J=J, pbc=(1, 1, 1), dirs=4)
    sites = np.arange(n, dtype=np.int32)
    ani = (sites, np.tile([0, 0, 1.0], (n, 1)), np.full(n, K))
    T6 = O.dipole_tensor(NX, NY, NZ)
    lr = O.LongRange(NX, NY, NZ, T6)
    return ss, paths, ani, lr, T6


def compute(quick=False):
    out = {}
    m = O.MT(5489)
    out["mt5489_first8"] = [float(m.randint()) for _ in range(8)]
    ss, paths, ani, lr, T6 = c1_setup()
    # one field evaluation
    ss.reset_fields()
    O.exchange_apply(ss, *paths)
    O.anisotropy_apply(ss, *ani)
    lr.apply(ss, G)
    ss.sum_fields()
    for name in ("Exchange", "Anisotropy", "Dipole", "Total"):
        out["c1_field_" + name] = ss.field(name).tolist()
    out["c1_tensor_XX_row0"] = T6[0][0, 0, :].tolist()
    out["c1_tensor_XY_row1"] = T6[1][0, 1, :].tolist()
    steps = 100 if quick else 1000
    for kind in ("Cartesian", "Quaternion"):
        ss, paths, ani, lr, _ = c1_setup()
        O.run_steps(ss, steps, paths=paths, ani=ani, lr=lr, g=G, llg=kind)
        out[f"c1_{kind}_{steps}"] = ss.spins().tolist()
        if not quick:
            ss2, paths, ani, lr, _ = c1_setup()
            O.run_steps(ss2, 100, paths=paths, ani=ani, lr=lr, g=G, llg=kind)
            out[f"c1_{kind}_100"] = ss2.spins().tolist()
    return out


if __name__ == "__main__":
    data = compute(quick=False)
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(data, f)
    print("wrote", os.path.join(HERE, "golden.json"), sorted(data))
