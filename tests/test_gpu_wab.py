"""The Dipole tensor cache files of the reference (WAB_<nx>x<ny>.<v>.lua,
M/cpu/dipole/dipolesupport.cpp:256-643): the layout the writer produces
(header, one "NAME[k] = [[...]]" or "NAME[k] = 0" block per z offset and
component, % .16g numbers), the tensor it holds against the oracle's lattice
sum, and a file read back as the operator's tensor (parameters checked as
dipoleParamsMatch does)."""
import re

import numpy as np
import pytest

import oracle as O
from helpers import random_spins, rel_err

pytestmark = pytest.mark.gpu
NAMES = ["XX", "XY", "XZ", "YY", "YZ", "ZZ"]


@pytest.fixture(scope="module")
def M():
    import maglua_b200 as M
    M.init(0)
    return M


def parse_wab(text, dims):
    nx, ny, nz = dims
    T = {q: np.zeros((2 * nz - 1, ny, nx)) for q in NAMES}
    for m in re.finditer(r"\n(XX|XY|XZ|YY|YZ|ZZ)\[(-?\d+)\] = (0|\[\[(.*?)\]\])", text, re.S):
        q, k, body = m.group(1), int(m.group(2)), m.group(4)
        if body is not None:
            rows = [[float(v) for v in line.split(",") if v.strip()] for line in body.strip().split("\n")]
            T[q][k + nz - 1] = np.array(rows)
    return [T[q] for q in NAMES]


def test_wab_written_layout_and_tensor(M, tmp_path):
    dims = (8, 6, 3)
    dip = M.Dipole(*dims)
    f = tmp_path / "WAB_8x6.1.lua"
    dip.writeWAB(f)
    text = f.read_text()
    assert "gmax = {1000, 1000, 1000, 1000}" in text
    assert "nx, ny, nz = 8, 6, 3" in text
    assert "function parse()" in text
    blocks = re.findall(r"\n(XX|XY|XZ|YY|YZ|ZZ)\[(-?\d+)\] = ", text)
    assert len(blocks) == 6 * 5
    got = parse_wab(text, dims)
    ref = O.dipole_tensor(*dims)
    for g, r in zip(got, ref):
        np.testing.assert_allclose(g, r, rtol=1e-12, atol=1e-14)


def test_wab_read_becomes_the_tensor(M, tmp_path):
    dims = (8, 6, 3)
    n = int(np.prod(dims))
    s = random_spins(n, 80)
    src = M.Dipole(*dims)
    f = tmp_path / "WAB_8x6.1.lua"
    src.writeWAB(f)
    # alter one layer: the read tensor, not a recomputed one, must be used
    text = f.read_text()
    T6 = parse_wab(text, dims)
    T6[0][2] *= 1.5
    lines = text.split("\n")
    out, skip = [], False
    for line in lines:
        if line.startswith("XX[0] = "):
            rows = "\n".join(",".join(f"{v:.16g}" for v in row) for row in T6[0][2])
            out.append("XX[0] = [[\n" + rows + "\n]]")
            skip = not line.endswith("= 0")
            continue
        if skip:
            if line == "]]":
                skip = False
            continue
        out.append(line)
    f2 = tmp_path / "WAB_8x6.2.lua"
    f2.write_text("\n".join(out))
    dip = M.Dipole(*dims)
    dip.setStrength(0.3)
    dip.readWAB(f2)
    ss = M.SpinSystem(*dims)
    ss.setSpinArrays(*s)
    dip.apply(ss)
    o = O.SpinSystem(*dims)
    o.set_spins(*s)
    O.LongRange(*dims, T6).apply(o, 0.3)
    assert rel_err(np.stack(ss.fieldArrays("Dipole")), o.field("Dipole")) <= 1e-5


def test_wab_parameters_must_match(M, tmp_path):
    f = tmp_path / "WAB_8x6.1.lua"
    M.Dipole(8, 6, 3).writeWAB(f)
    with pytest.raises(M.MagLuaError, match="nx, ny, nz"):
        M.Dipole(8, 6, 2).readWAB(f)
    d = M.Dipole(8, 6, 3)
    d.setTruncation(50)
    with pytest.raises(M.MagLuaError, match="gmax"):
        d.readWAB(f)


# ---------------------------------------------------------------- truncation math.huge
@pytest.mark.parametrize("dims,rings", [((6, 5, 3), 7), ((16, 4, 2), 3)])
def test_huge_truncation_ring_sum_matches_oracle(M, dims, rings):
    """Truncation math.huge (dipoleLoad, dipolesupport.cpp:771-835): the image
    sum in rings of 5 lattices, here over a few rings (the ring count is a
    parameter of the check; the reference's is 1000)."""
    dip = M.Dipole(*dims)
    dip.setTruncation(float("inf"))
    assert dip.truncation() == (float("inf"),) * 4
    dip.setHugeRings(rings)
    got = dip.tensorArrays()
    ref = O.dipole_tensor_rings(*dims, nrings=rings)
    scale = max(np.abs(r).max() for r in ref)
    for g, r in zip(got, ref):
        assert np.abs(g - r).max() <= 1e-12 * scale


def test_huge_truncation_full_ring_count_and_field(M, tmp_path):
    """The reference's full count, 1000 rings (|X|, |Y| <= 4999), on a 2x2x1
    lattice against the oracle; the field it gives; a WAB file written with
    gmax = {math.huge, ...} read back by another operator of truncation
    math.huge."""
    dims = (2, 2, 1)
    dip = M.Dipole(*dims)
    dip.setTruncation(float("inf"))
    got = dip.tensorArrays()
    ref = O.dipole_tensor_rings(*dims, nrings=1000)
    scale = max(np.abs(r).max() for r in ref)
    for g, r in zip(got, ref):
        assert np.abs(g - r).max() <= 1e-11 * scale
    n = 4
    s = random_spins(n, 81)
    ss = M.SpinSystem(*dims)
    ss.setSpinArrays(*s)
    dip.setStrength(0.3)
    dip.apply(ss)
    o = O.SpinSystem(*dims)
    o.set_spins(*s)
    O.LongRange(*dims, ref).apply(o, 0.3)
    assert rel_err(np.stack(ss.fieldArrays("Dipole")), o.field("Dipole")) <= 1e-5
    f = tmp_path / "WAB_2x2.1.lua"
    dip.writeWAB(f)
    assert "gmax = {math.huge, math.huge, math.huge, math.huge}" in f.read_text()
    other = M.Dipole(*dims)
    other.setTruncation(float("inf"))
    other.setHugeRings(1)          # a read file replaces the sum
    other.readWAB(f)
    for g, r in zip(other.tensorArrays(), ref):
        assert np.abs(g - r).max() <= 1e-11 * scale
