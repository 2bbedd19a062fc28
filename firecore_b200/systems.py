"""Seeded synthetic workloads for multi-system MMFF relaxation.

Molecules: heavy-atom trees with C:N:O:H = 10:2:2:10, heavy-heavy bonds
1.40 +- 0.05 A, X-H caps 1.09 A, angle / pi terms by hybridisation, charges
N(0, 0.2) e re-centred to zero net (native generator ``mmff_gen_systems`` of the
host-only ``libmmff_gen.so``).
Substrate: rigid rock-salt (001) slab, a = 5.64 A, 3 layers, 4 x 4 cells,
ions +-0.9 e, periodic in x, y.

Arrays follow the layout of the reference's MMFFsp3_loc
(cpp/common/molecular/MMFFsp3_loc.h:43-139): per system ``natoms`` atoms with
the ``nnode`` node atoms first, then caps, and ``nvecs = natoms + nnode``
vectors (atoms, then one pi orbital per node).  Systems are packed back to
back (CSR) and all topology indices are local to their system.
"""
from __future__ import annotations

import ctypes
import math
import os
from dataclasses import dataclass, field
from typing import Sequence

import numpy as np

from . import _lib

# MMFFsp3_loc neighbour-cell index of the zero image for nPBC = (1,1,0)
# (NBFF.h:42 makePBCshifts_ ordering: iz outer, iy, ix inner).
def central_cell(npbc: Sequence[int]) -> int:
    nx, ny = 2 * npbc[0] + 1, 2 * npbc[1] + 1
    return (npbc[2] * ny + npbc[1]) * nx + npbc[0]


@dataclass
class SystemBatch:
    natoms: np.ndarray            # [nsys] int32
    nnode: np.ndarray             # [nsys] int32
    pos: np.ndarray               # [sum nvecs, 3] float64
    neighs: np.ndarray            # [sum natoms, 4] int32
    neighCell: np.ndarray         # [sum natoms, 4] int32
    bkneighs: np.ndarray          # [sum natoms, 4] int32
    REQs: np.ndarray              # [sum natoms, 4] float64  (R0, sqrt(E0), Q, Hb)
    apars: np.ndarray             # [sum nnode, 4]
    bLs: np.ndarray
    bKs: np.ndarray
    Ksp: np.ndarray
    Kpp: np.ndarray
    lvec: np.ndarray              # [nsys, 3, 3]
    elements: np.ndarray          # [sum natoms] int32 (0 H, 1 C, 2 N, 3 O)

    @property
    def nsys(self) -> int:
        return int(self.natoms.shape[0])

    @property
    def nvecs(self) -> np.ndarray:
        return self.natoms + self.nnode

    def offsets(self):
        a = np.zeros(self.nsys + 1, np.int64); a[1:] = np.cumsum(self.natoms)
        n = np.zeros(self.nsys + 1, np.int64); n[1:] = np.cumsum(self.nnode)
        v = np.zeros(self.nsys + 1, np.int64); v[1:] = np.cumsum(self.nvecs)
        return a, n, v

    def subset(self, idx: Sequence[int]) -> "SystemBatch":
        a, n, v = self.offsets()
        idx = list(idx)
        cat = lambda arr, off: np.concatenate([arr[off[i]:off[i + 1]] for i in idx]) if idx else arr[:0]
        return SystemBatch(self.natoms[idx].copy(), self.nnode[idx].copy(), cat(self.pos, v),
                           cat(self.neighs, a), cat(self.neighCell, a), cat(self.bkneighs, a),
                           cat(self.REQs, a), cat(self.apars, n), cat(self.bLs, n), cat(self.bKs, n),
                           cat(self.Ksp, n), cat(self.Kpp, n), self.lvec[idx].copy(), cat(self.elements, a))


def make_systems(natoms: Sequence[int], seed: int, topo_mode: int = 1, sigma: float = 0.1,
                 rotate: bool = True, zplace: float = 3.0, cell=(22.56, 22.56, 40.0),
                 hbond: bool = False, npbc=(1, 1, 0)) -> SystemBatch:
    """Generate ``len(natoms)`` seeded molecules (see module docstring)."""
    lib = _lib.gen()
    natoms = np.ascontiguousarray(natoms, dtype=np.int32)
    nsys = natoms.shape[0]
    nnode = np.array([lib.mmff_gen_nnode(int(n)) for n in natoms], np.int32)
    na, nn, nv = int(natoms.sum()), int(nnode.sum()), int((natoms + nnode).sum())
    pos = np.zeros((nv, 3)); neighs = np.zeros((na, 4), np.int32); neighCell = np.zeros((na, 4), np.int32)
    bk = np.zeros((na, 4), np.int32); REQs = np.zeros((na, 4)); el = np.zeros(na, np.int32)
    apars, bLs, bKs, Ksp, Kpp = (np.zeros((nn, 4)) for _ in range(5))
    cxy = np.array(cell[:2], np.float64)
    rc = lib.mmff_gen_systems(nsys, _lib.ptr(natoms), ctypes.c_uint64(seed), topo_mode, sigma, int(rotate),
                              zplace, _lib.ptr(cxy), int(hbond), _lib.ptr(pos), _lib.ptr(neighs),
                              _lib.ptr(neighCell), _lib.ptr(bk), _lib.ptr(REQs), _lib.ptr(apars),
                              _lib.ptr(bLs), _lib.ptr(bKs), _lib.ptr(Ksp), _lib.ptr(Kpp), _lib.ptr(el),
                              central_cell(npbc))
    if rc != 0:
        raise RuntimeError(f"mmff_gen_systems failed for system {-rc - 1}")
    lvec = np.tile(np.diag(np.array(cell, np.float64)), (nsys, 1, 1))
    return SystemBatch(natoms, nnode, pos, neighs, neighCell, bk, REQs, apars, bLs, bKs, Ksp, Kpp, lvec, el)


@dataclass
class GridSpec:
    n: tuple                      # (nx, ny, nz)
    pos0: tuple                   # grid origin [A]
    step: tuple                   # orthorhombic voxel edges [A]

    @property
    def npoints(self) -> int:
        return int(self.n[0]) * int(self.n[1]) * int(self.n[2])


@dataclass
class Substrate:
    spos: np.ndarray              # [nsub, 3]
    sREQ: np.ndarray              # [nsub, 4]
    lvec: np.ndarray              # [3, 3]
    grid: GridSpec
    alphaMorse: float = 1.5
    nPBC_mors: tuple = (1, 1, 0)
    nPBC_coul: tuple = (25, 25, 0)


def make_slab(a: float = 5.64, ncell: int = 4, layers: int = 3, q: float = 0.9, z_top: float = 0.0,
              grid_step: float = 0.1, nz: int = 200, z0: float = 0.5,
              REQ_cation=(1.6, math.sqrt(0.004), 0.0, 0.0), REQ_anion=(2.0, math.sqrt(0.010), 0.0, 0.0),
              nPBC_coul=(25, 25, 0), nPBC_mors=(1, 1, 0)) -> Substrate:
    """Rigid rock-salt slab with its B-spline grid specification.

    The x, y grid spacing is the cell edge divided by round(L / grid_step), so the
    grid is commensurate with the periodic cell; z starts ``z0`` above the top
    layer (no grid node sits on an ion)."""
    lib = _lib.gen()
    nsub = 4 * ncell * ncell * layers
    spos = np.zeros((nsub, 3)); sREQ = np.zeros((nsub, 4))
    rc = np.array(REQ_cation, np.float64); ra = np.array(REQ_anion, np.float64)
    n = lib.mmff_gen_slab(a, ncell, layers, z_top, q, _lib.ptr(rc), _lib.ptr(ra), _lib.ptr(spos), _lib.ptr(sREQ))
    assert n == nsub
    L = a * ncell
    nx = int(round(L / grid_step))
    g = GridSpec((nx, nx, nz), (0.0, 0.0, z_top + z0), (L / nx, L / nx, grid_step))
    lvec = np.diag([L, L, max(40.0, nz * grid_step + 10.0)])
    return Substrate(spos, sREQ, lvec, g, 1.5, tuple(nPBC_mors), tuple(nPBC_coul))


# ---------------------------------------------------------------- workloads

def config_small(seed: int = 0, nrep: int = 16, natoms: int = 24, sigma: float = 0.1, hbond=False):
    """16 replicas of one 24-atom molecule, sigma = 0.1 A, 3.0 A above the slab."""
    return make_systems([natoms] * nrep, seed, topo_mode=0, sigma=sigma, rotate=False, hbond=hbond)


def config_replicas(seed: int = 1, nrep: int = 4096, natoms: int = 60, sigma: float = 0.15):
    """Replicas of one seeded 60-atom molecule, random rigid rotation + sigma = 0.15 A."""
    return make_systems([natoms] * nrep, seed, topo_mode=0, sigma=sigma, rotate=True)


def loguniform_sizes(n: int, seed: int, lo: int = 20, hi: int = 400) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.exp(rng.uniform(math.log(lo), math.log(hi + 1), n)).astype(np.int32).clip(lo, hi)


def config_uneven(seed: int = 2, nsys: int = 32768, sigma: float = 0.15):
    """Distinct molecules with atom counts log-uniform in [20, 400]."""
    return make_systems(loguniform_sizes(nsys, seed), seed, topo_mode=1, sigma=sigma, rotate=True)
