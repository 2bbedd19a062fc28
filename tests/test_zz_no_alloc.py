"""mmff_bspline_fit_noalloc: the B-spline fit for callers that may not allocate
device memory (they own every buffer, e.g. through a fixed arena of their
own).  The caller passes a device array of node values; the call fits it in
place without any cudaMalloc, keeping its per-axis solver coefficients in a
static device array.

Checked against the allocating path, mmff_grid_build, on the golden small grid,
for two calls in a row (the second reuses the scratch the first left behind).
Runs last in the suite (file name) and also alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from conftest import grid_from_golden

pytestmark = pytest.mark.gpu


def test_noalloc_fit_matches_grid_build(golden):
    import torch
    from firecore_b200 import _lib
    from firecore_b200.systems import Substrate
    from firecore_b200.world import World

    lib = _lib.load()
    lib.mmff_bspline_fit_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    lib.mmff_bspline_fit_noalloc.restype = ctypes.c_int

    grid = grid_from_golden(golden)
    sub = Substrate(golden["spos"], golden["sREQ"], golden["slvec"], grid, 1.5, (1, 1, 0), (4, 4, 0))
    ref = World(0).grid_build(sub, return_coefs=True)          # existing, allocating entry point
    nx, ny, nz = grid.n
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    for call in range(2):
        d = torch.from_numpy(np.ascontiguousarray(golden["V"])).to("cuda")   # caller-owned node values
        rc = lib.mmff_bspline_fit_noalloc(ctypes.c_void_p(d.data_ptr()), nx, ny, nz, ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, lib.mmff_last_error().decode()
        torch.cuda.synchronize()
        C = d.cpu().numpy()
        assert np.abs(C - ref).max() <= 1e-9 * np.abs(ref).max(), f"call {call}"


def test_noalloc_fit_rejects_oversized_grid():
    from firecore_b200 import _lib
    lib = _lib.load()
    lib.mmff_bspline_fit_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    lib.mmff_bspline_fit_noalloc.restype = ctypes.c_int
    rc = lib.mmff_bspline_fit_noalloc(ctypes.c_void_p(16), 5000, 8, 8, None)   # rejected before any device access
    assert rc < 0 and b"exceeds" in lib.mmff_last_error()
