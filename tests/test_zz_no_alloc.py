"""mlb_dipole_field_noalloc: the Dipole field of caller-owned FP32 device
arrays with the spectrum scratch in a static device array (no allocation in
the call).  Compared, through the C ABI, with the field the ordinary
operator apply (mlb_op_apply) writes into the SpinSystem's "Dipole" slot, on
consecutive calls.  The device arrays handed to it are torch tensors (the
test allocates; the call under test does not)."""
import ctypes as C

import numpy as np
import pytest

from helpers import random_spins, rel_err

pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-5


@pytest.fixture(scope="module")
def M():
    import maglua_b200 as M
    M.init(0)
    return M


@pytest.fixture(scope="module")
def torch():
    import torch
    return torch


def _reference_field(M, dims, spins, g, open_xy):
    ss = M.SpinSystem(*dims)
    ss.setSpinArrays(*spins)
    dip = M.Dipole(ss)
    dip.setStrength(g)
    if open_xy:
        dip.setOpen(True, True, True)
    dip.apply(ss)
    return ss, dip, np.stack(ss.fieldArrays("Dipole"))


def _noalloc(M, torch, op, spins):
    dev = torch.device("cuda", 0)
    s = [torch.tensor(np.ascontiguousarray(spins[c]), dtype=torch.float32, device=dev) for c in range(3)]
    h = [torch.full_like(s[0], float("nan")) for _ in range(3)]
    torch.cuda.synchronize()
    rc = M._lib.mlb_dipole_field_noalloc(op._h, *[t.data_ptr() for t in s], *[t.data_ptr() for t in h], None)
    torch.cuda.synchronize()
    assert rc == 0, M._lib.mlb_last_error().decode()
    return np.stack([t.double().cpu().numpy() for t in h])


@pytest.mark.parametrize("dims,open_xy", [((32, 32, 4), False),   # power-of-two sizes: register/Stockham FFT passes
                                          ((7, 5, 3), False),     # general FFT kernels
                                          ((12, 10, 2), True)])   # open in-plane boundaries (zero padded)
def test_noalloc_matches_operator_apply_on_consecutive_calls(M, torch, dims, open_xy):
    n = int(np.prod(dims))
    s1 = random_spins(n, 71, lengths=True)
    s2 = random_spins(n, 72, lengths=True)
    ss, dip, ref1 = _reference_field(M, dims, s1, 0.3, open_xy)
    ss.setSpinArrays(*s2)
    dip.apply(ss)
    ref2 = np.stack(ss.fieldArrays("Dipole"))
    first = _noalloc(M, torch, dip, s1)
    second = _noalloc(M, torch, dip, s1)
    third = _noalloc(M, torch, dip, s2)
    for got, ref in ((first, ref1), (second, ref1), (third, ref2)):
        assert np.isfinite(got).all()
        assert rel_err(got, ref) <= FIELD_TOL


def _user_tensor_op(M, kind, dims, g):
    """A LongRange with random elements at a few offsets, or a Dipole with
    one element edited after its lattice sum: both take the general
    (9-component complex) tensor multiply."""
    nx, ny, nz = dims
    r = np.random.default_rng(5)
    if kind == "longrange":
        op = M.LongRange(*dims)
        for ab in ("XX", "XY", "XZ", "YY", "YZ", "ZZ"):
            for off in ((0, 0, 0), (1, 0, 0), (0, -1, 0), (2, 1, 1 if nz > 1 else 0), (-1, 2, -1 if nz > 1 else 0)):
                op.setMatrix(ab, off, float(r.normal()))
    else:
        op = M.Dipole(*dims)
        op.getMatrix("XY", (1, 1, 0))        # builds the lattice sum
        op.setMatrix("XY", (1, 1, 0), 0.37)
    op.setStrength(g)
    return op


@pytest.mark.parametrize("kind", ["longrange", "edited_dipole"])
@pytest.mark.parametrize("dims", [(16, 8, 3), (6, 5, 2)])
def test_noalloc_matches_operator_apply_with_user_tensors(M, torch, kind, dims):
    n = int(np.prod(dims))
    s1 = random_spins(n, 81, lengths=True)
    s2 = random_spins(n, 82)
    op = _user_tensor_op(M, kind, dims, 0.2)
    refs = []
    for s in (s1, s2):
        ss = M.SpinSystem(*dims)
        ss.setSpinArrays(*s)
        op.apply(ss)
        refs.append(np.stack(ss.fieldArrays(op.slotName())))
    got = [_noalloc(M, torch, op, s1), _noalloc(M, torch, op, s2)]
    for g_, ref in zip(got, refs):
        assert np.isfinite(g_).all()
        assert rel_err(g_, ref) <= FIELD_TOL


def test_noalloc_rejects_lattice_beyond_scratch(M):
    # 1024 x 256 x 8 periodic: (513 kx) x 3 x 8 x 256 complex FP32 = 25.2 MB > 16 MiB
    dip = M.Dipole(1024, 256, 8)
    rc = M._lib.mlb_dipole_field_noalloc(dip._h, None, None, None, None, None, None, None)
    assert rc == -6  # MLB_ERANGE
    assert "16777216-byte static scratch" in M._lib.mlb_last_error().decode()


def test_noalloc_requires_built_tensor(M):
    dip = M.Dipole(8, 8, 2)
    rc = M._lib.mlb_dipole_field_noalloc(dip._h, None, None, None, None, None, None, None)
    assert rc == -4  # MLB_ESTATE


def test_noalloc_rejects_another_current_device(M, torch):
    # the tensor spectrum lives on device 0; with device 1 current the call
    # must refuse before launching anything
    if torch.cuda.device_count() < 2:
        pytest.skip("needs two visible devices")
    dims = (8, 8, 2)
    n = int(np.prod(dims))
    dip = M.Dipole(*dims)
    dip.setStrength(0.1)
    ss = M.SpinSystem(*dims)
    ss.setSpinArrays(*random_spins(n, 3))
    dip.apply(ss)
    ss.synchronize()
    with torch.cuda.device(1):
        t = [torch.zeros(n, device="cuda:1") for _ in range(6)]
        rc = M._lib.mlb_dipole_field_noalloc(dip._h, *[x.data_ptr() for x in t], None)
    assert rc == -1  # MLB_EINVAL
    assert "holds the operator's tensor spectrum" in M._lib.mlb_last_error().decode()
