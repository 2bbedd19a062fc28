"""Loader for the native library (``libMMFFmulti_lib.so``, built in-tree)."""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("MMFF_LIB", os.path.join(HERE, "libMMFFmulti_lib.so"))
GEN_PATH = os.path.join(HERE, "libmmff_gen.so")
_lib = None
_gen = None


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


def gen() -> ctypes.CDLL:
    """Load the host-only workload generator (``libmmff_gen.so``: the seeded
    molecules and slabs of ``csrc/molgen.cpp``, no CUDA)."""
    global _gen
    if _gen is None:
        if not os.path.exists(GEN_PATH):
            raise RuntimeError(f"{GEN_PATH} is missing: run `python -m firecore_b200.build` first")
        g = ctypes.CDLL(GEN_PATH, mode=ctypes.RTLD_LOCAL)
        _declare_gen(g)
        _gen = g
    return _gen


def _declare_gen(lib):
    c_int, c_double, c_void = ctypes.c_int, ctypes.c_double, ctypes.c_void_p
    lib.mmff_gen_nnode.argtypes = [c_int]
    lib.mmff_gen_nnode.restype = c_int
    lib.mmff_gen_systems.argtypes = [c_int, c_void, ctypes.c_uint64, c_int, c_double, c_int, c_double, c_void,
                                     c_int] + [c_void] * 11 + [c_int]
    lib.mmff_gen_systems.restype = c_int
    lib.mmff_gen_slab.argtypes = [c_double, c_int, c_int, c_double, c_double, c_void, c_void, c_void, c_void]
    lib.mmff_gen_slab.restype = c_int


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
    _declare_gen(lib)
    lib.mmff_last_error.argtypes = []
    lib.mmff_last_error.restype = ctypes.c_char_p
    sig = {
        "mmff_init_device": [c_int], "mmff_sync": [], "mmff_set_params": [c_int, c_void, c_double, c_double, c_double],
        "mmff_set_fire": [c_double] * 6 + [c_int, c_double, c_double, c_int], "mmff_set_launch": [c_int, c_int],
        "mmff_grid_upload": [c_int, c_int, c_int, c_void, c_void, c_void],
        "mmff_grid_build": [c_int, c_void, c_void, c_void, c_void, c_void, c_double, c_int, c_int, c_int, c_void,
                            c_void, c_void],
        "mmff_grid_sample": [c_int, c_void, c_void, c_void],
        "mmff_systems_upload": [c_int] + [c_void] * 14, "mmff_systems_restore": [],
        "mmff_systems_set_state": [c_void, c_void, c_int], "mmff_eval": [c_int],
        "mmff_set_constraints": [c_void, c_void], "mmff_set_bond_constraints": [c_int, c_void, c_void, c_int, c_void, c_void], "mmff_set_grid_cache": [c_int], "mmff_set_pair_lists": [c_int, c_double],
        "mmff_relax": [c_int, c_double, c_int], "mmff_get_forces": [c_void], "mmff_get_energies": [c_void],
        "mmff_get_state": [c_void] * 6, "mmff_timer_start": [], "mmff_num_buckets": [],
        "mmff_bucket_info": [c_int, c_void], "mmff_set_counting": [c_int], "mmff_get_counters": [c_void],
        "mmff_mlp_set_params": [c_void, c_void, c_void, c_double], "mmff_mlp_get_params": [c_void],
        "mmff_mlp_grad": [c_int, c_void, c_void, c_void, c_void], "mmff_mlp_adamw": [c_void, c_double, c_double],
        "mmff_mlp_infer": [c_int, c_void, c_void], "mmff_mlp_set_data": [c_int, c_void, c_void],
        "mmff_mlp_train": [c_int, c_int, c_double, c_double, c_void], "mmff_mlp_set_elements": [c_void],
        "mmff_mlp_features": [c_double, c_void], "mmff_mlp_warmstart": [c_int, c_double, c_void],
        "mmff_mlp_set_projection": [c_int], "mmff_mlp_project": [c_void, c_void], "mmff_mlp_wait_test": [],
        "mmff_mlp_plan": [c_void], "mmff_mlp_layout": [c_void],
        "mmff_set_graph": [c_int], "mmff_set_md": [c_double, c_double, c_double, ctypes.c_ulonglong],
        "mmff_md": [c_int], "mmff_set_explore": [c_int, c_int, c_int], "mmff_explore": [c_int, c_double, c_int],
        "mmff_get_explore": [c_void, c_void], "mmff_surf_upload": [c_int, c_void, c_void, c_void, c_void, c_double], "mmff_autotune": [c_int, c_int, c_void, c_int],
        "mmff_get_tuning": [c_int, c_void], "mmff_set_tuning": [c_int, c_int, c_int, c_int, c_int],
        "mmff_build_xyz": [ctypes.c_char_p] * 5 + [c_int, c_void, c_int] + [c_void] * 12,
    }
    for name, args in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = c_int
    lib.mmff_kernel_launches.argtypes = []
    lib.mmff_kernel_launches.restype = ctypes.c_ulonglong
    lib.mmff_timer_stop.argtypes = []
    lib.mmff_timer_stop.restype = c_double
    lib.mmff_peak_fp32.argtypes = []
    lib.mmff_peak_fp32.restype = c_double
    lib.mmff_peak_l2.argtypes = [c_int]
    lib.mmff_peak_l2.restype = c_double
    lib.mmff_mlp_smem_desc.argtypes = [ctypes.c_uint, ctypes.c_uint, ctypes.c_uint]
    lib.mmff_mlp_smem_desc.restype = ctypes.c_ulonglong
    lib.mmff_mlp_instr_desc.argtypes = [c_int, c_int, c_int]
    lib.mmff_mlp_instr_desc.restype = ctypes.c_uint
