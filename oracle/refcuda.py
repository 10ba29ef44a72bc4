"""The reference's own FP64 CUDA kernels (LLG quaternion and Cartesian,
Anisotropy, Thermal), compiled unchanged from the reference tree by
oracle/Makefile into oracle/_ref/libref_cuda.so with the C ABI of
oracle/ref_cuda_shim.cu.

TEST INFRASTRUCTURE ONLY: tests/ use it to pin the oracle and the product
against the reference's own arithmetic.  Every pointer it takes is a device
pointer (the tests pass torch tensors' data_ptr()).  load() returns None when
the library was not built (no reference tree where it was built).
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(_HERE, "_ref", "libref_cuda.so")

_P = C.c_void_p
_P4 = _P * 4
_P3 = _P * 3
_lib = None


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        return None
    lib = C.CDLL(LIB)
    lib.ref_llg_quat_apply.argtypes = [C.c_int, C.c_int, C.c_int, _P4, _P4, _P4, _P3, _P3, _P4, C.c_double,
                                       C.c_double, _P, C.c_double, _P, C.c_int]
    lib.ref_llg_cart_apply_n.argtypes = [C.c_int, C.c_int, C.c_int, _P4, _P4, _P4, _P3, _P3, _P, _P, _P, _P, _P,
                                         C.c_int, C.c_int, C.c_int]
    lib.ref_anisotropy_n.argtypes = [C.c_double, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, C.c_int, C.c_int]
    lib.ref_thermal.argtypes = [_P, C.c_int, C.c_double, _P, _P, _P, _P, _P, C.c_int, C.c_double, C.c_double, _P,
                                C.c_double, _P]
    for f in (lib.ref_llg_quat_apply, lib.ref_llg_cart_apply_n, lib.ref_anisotropy_n, lib.ref_thermal):
        f.restype = C.c_int
    _lib = lib
    return lib


def ptrs(*tensors):
    """Host array of the tensors' device addresses (None -> NULL)."""
    vals = [0 if t is None else t.data_ptr() for t in tensors]
    return (_P * len(vals))(*vals)
