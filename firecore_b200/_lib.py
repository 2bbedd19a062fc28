"""Loader for the native library (``libMMFFmulti_lib.so``, built in-tree)."""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libMMFFmulti_lib.so")
_lib = None


def load() -> ctypes.CDLL:
    """Load the library (RTLD_LOCAL, as pyBall/cpp_utils_.py loads the reference's)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run `python -m firecore_b200.build` first")
        lib = ctypes.CDLL(LIB_PATH, mode=ctypes.RTLD_LOCAL)
        _declare(lib)
        _lib = lib
    return _lib


def ptr(a):
    """ctypes void pointer to a numpy array or torch tensor (None -> NULL)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
        return ctypes.c_void_p(a.ctypes.data)
    return ctypes.c_void_p(a.data_ptr())


def _declare(lib):
    c_int, c_double, c_void = ctypes.c_int, ctypes.c_double, ctypes.c_void_p
    lib.mmff_gen_nnode.argtypes = [c_int]
    lib.mmff_gen_nnode.restype = c_int
    lib.mmff_gen_systems.argtypes = [c_int, c_void, ctypes.c_uint64, c_int, c_double, c_int, c_double, c_void,
                                     c_int] + [c_void] * 11 + [c_int]
    lib.mmff_gen_systems.restype = c_int
    lib.mmff_gen_slab.argtypes = [c_double, c_int, c_int, c_double, c_double, c_void, c_void, c_void, c_void]
    lib.mmff_gen_slab.restype = c_int
