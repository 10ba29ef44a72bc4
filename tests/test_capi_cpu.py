"""CPU checks of the C ABI library: it loads, exports every symbol that
include/mlb200.h declares, its host-side pieces give published answers, and
without a GPU it fails loudly instead of computing anything on the CPU."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "mlb200.h")


def _declared():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mlb_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    import maglua_b200
    return maglua_b200._lib.load()


def test_library_exports_every_declared_symbol(lib):
    names = _declared()
    assert len(names) > 60
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_mirror_binds_every_declared_symbol():
    import maglua_b200
    assert sorted(maglua_b200.EXPORTED) == _declared()


def test_philox_known_answers():
    # Random123 kat_vectors for philox4x32_10 (Salmon et al., SC'11)
    import maglua_b200 as M
    assert M.philox4x32_10((0, 0, 0, 0), (0, 0)) == (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)
    assert M.philox4x32_10((0xffffffff,) * 4, (0xffffffff,) * 2) == (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)
    assert M.philox4x32_10((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0)) == (
        0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1)


def test_box_muller_uniforms_in_open_interval():
    # the 24-bit uniforms used before log(): (k + 0.5) * 2^-24 never hits 0 or 1
    k = np.array([0, 2 ** 24 - 1], dtype=np.float64)
    u = (k + 0.5) * 2.0 ** -24
    assert (u > 0).all() and (u < 1).all()


@pytest.mark.skipif(os.path.exists("/dev/nvidia0"), reason="a GPU is present")
def test_without_gpu_calls_fail_loudly(lib):
    import maglua_b200 as M
    rc = lib.mlb_init(0)
    assert rc != 0
    assert len(lib.mlb_last_error()) > 0
    with pytest.raises(M.MagLuaError):
        M.init(0)


def test_error_codes_are_distinct():
    text = open(HEADER).read()
    codes = re.findall(r"#define MLB_E[A-Z]+ (-\d+)", text)
    assert len(codes) == len(set(codes)) >= 6
