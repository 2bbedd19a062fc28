"""mmff_bspline_fit_noalloc: the B-spline fit for callers that may not allocate
device memory (they own every buffer, e.g. through a fixed arena of their
own).  The caller passes a device array of node values; the call fits it in
place without any cudaMalloc, keeping its per-axis solver coefficients in a
static device array.

Checked against the allocating path, mmff_grid_build, on the golden small grid,
for two calls in a row (the second reuses the scratch the first left behind);
on grids whose three axes differ (and on the smallest grid the entry point
accepts) against a dense numpy solve of the same periodic / open systems; and
a host pointer must come back as an argument error.  Runs last in the suite
(file name) and also alone in a fresh process.
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


def _dense_fit(V):
    """Coefficients C with V = (Mx (x) My (x) Mz) C: (c[i-1] + 4 c[i] + c[i+1]) / 6
    per axis, periodic along x and y, zero outside the grid along z."""
    def mat(n, periodic):
        M = np.zeros((n, n))
        for i in range(n):
            M[i, i] += 4.0 / 6.0
            for j in (i - 1, i + 1):
                if 0 <= j < n:
                    M[i, j] += 1.0 / 6.0
                elif periodic:
                    M[i, j % n] += 1.0 / 6.0
        return np.linalg.inv(M)
    nx, ny, nz = V.shape[:3]
    return np.einsum("ia,jb,kc,abcd->ijkd", mat(nx, True), mat(ny, True), mat(nz, False), V)


@pytest.mark.parametrize("shape", [(12, 10, 8), (3, 3, 2), (5, 7, 16)])
def test_noalloc_fit_uneven_axes_vs_dense_solve(shape):
    import torch
    from firecore_b200 import _lib
    lib = _lib.load()
    lib.mmff_bspline_fit_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    lib.mmff_bspline_fit_noalloc.restype = ctypes.c_int
    V = np.random.default_rng(sum(shape)).normal(size=shape + (3,))
    ref = _dense_fit(V)
    torch.cuda.set_device(0)
    for call in range(2):
        d = torch.from_numpy(V.copy()).to("cuda")
        rc = lib.mmff_bspline_fit_noalloc(ctypes.c_void_p(d.data_ptr()), *shape, None)
        assert rc == 0, lib.mmff_last_error().decode()
        torch.cuda.synchronize()
        assert np.abs(d.cpu().numpy() - ref).max() <= 1e-12 * np.abs(ref).max() + 1e-13, (shape, call)


def test_noalloc_fit_rejects_host_pointer():
    from firecore_b200 import _lib
    lib = _lib.load()
    lib.mmff_bspline_fit_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    lib.mmff_bspline_fit_noalloc.restype = ctypes.c_int
    h = np.zeros((8, 8, 8, 3))
    rc = lib.mmff_bspline_fit_noalloc(ctypes.c_void_p(h.ctypes.data), 8, 8, 8, None)
    assert rc < 0 and b"not device memory" in lib.mmff_last_error()
