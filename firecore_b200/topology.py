"""FireCore-typed molecules from an xyz file and FireCore's parameter tables.

``build_xyz`` calls the library's ``mmff_build_xyz`` (host code, no device):
the result of FireCore's ``MolWorld_sp3::initParams`` -> ``buildMolecule_xyz``
-> ``makeFFs`` (cpp/common/molecular/MolWorld_sp3.h:1298-1586, typing by
``MM::Builder``, MMFFBuilder.h) as ``MMFFsp3_loc`` arrays: nodes first, then
capping atoms, pi orientations after the atoms.
"""
import ctypes
import os

import numpy as np

from . import _lib

TABLES = ("ElementTypes.dat", "AtomTypes.dat", "BondTypes.dat", "AngleTypes.dat")


def table_paths(directory):
    """The four table files of a FireCore ``common_resources`` directory."""
    return tuple(os.path.join(directory, f) for f in TABLES)


def build_xyz(xyz, tables, epairs=False, nPBC=(1, 1, 0), cap=None):
    """Type ``xyz`` with the four table files ``tables``; returns a dict of arrays
    (natoms, nnode, pbc, apos [(natoms+nnode),3], REQs [natoms,4], atypes, type_names,
    neighs / neighCell [natoms,4], apars / bLs / bKs / Ksp / Kpp [nnode,4]).
    Raises RuntimeError with the library's message when the files or the
    molecule are rejected."""
    lib = _lib.load()
    if cap is None:
        with open(xyz) as f:
            try:
                cap = 4 * max(1, int(f.readline().split()[0])) + 8
            except (ValueError, IndexError):
                cap = 64
    cnt = np.zeros(4, np.int32)
    apos = np.zeros((2 * cap, 3))
    REQs = np.zeros((cap, 4))
    at = np.zeros(cap, np.int32)
    ng = np.zeros((cap, 4), np.int32)
    nc = np.zeros((cap, 4), np.int32)
    par = [np.zeros((cap, 4)) for _ in range(5)]
    names = ctypes.create_string_buffer(8 * cap)
    npbc = np.asarray(nPBC, np.int32)
    n = lib.mmff_build_xyz(*(str(t).encode() for t in tables), str(xyz).encode(), int(bool(epairs)), _lib.ptr(npbc), cap,
                           _lib.ptr(cnt), _lib.ptr(apos), _lib.ptr(REQs), _lib.ptr(at), _lib.ptr(ng), _lib.ptr(nc),
                           *(_lib.ptr(a) for a in par), names)
    if n < 0:
        raise RuntimeError(lib.mmff_last_error().decode())
    na, nn = int(cnt[0]), int(cnt[1])
    lvec = np.eye(3) * 20.0
    if cnt[3]:
        with open(xyz) as f:
            f.readline()
            lvec = np.array(f.readline().split()[1:10], float).reshape(3, 3)
    return dict(lvec=lvec, natoms=na, nnode=nn, pbc=bool(cnt[3]), apos=apos[:na + nn].copy(), REQs=REQs[:na].copy(),
                atypes=at[:na].copy(), type_names=[names.raw[8 * i:8 * i + 8].split(b"\0")[0].decode() for i in range(na)],
                neighs=ng[:na].copy(), neighCell=nc[:na].copy(), apars=par[0][:nn].copy(), bLs=par[1][:nn].copy(),
                bKs=par[2][:nn].copy(), Ksp=par[3][:nn].copy(), Kpp=par[4][:nn].copy())


def to_batch(d, nPBC=(1, 1, 0), lvec=None, nsys=1):
    """``nsys`` copies of a ``build_xyz`` result as a ``systems.SystemBatch`` for
    the CSR world (``world.World.upload``) and the oracle: back neighbours as
    ``MMFFsp3_loc::makeBackNeighs`` builds them, neighbour cells from the xyz
    cell where it had one (else the central image), ``lvec`` = the xyz cell,
    the given 3x3 cell, or a 20 A cube."""
    from . import systems as S
    na, nn = d["natoms"], d["nnode"]
    ng = d["neighs"].astype(np.int32)
    bk = -np.ones((na, 4), np.int32)
    for ia in range(nn):
        for j in range(4):
            ja = ng[ia, j]
            if ja < 0:
                continue
            q = int(np.argmax(bk[ja] < 0))
            if bk[ja, q] >= 0:
                raise ValueError(f"atom {ja} has more than 4 back-neighbours")
            bk[ja, q] = ia * 4 + j
    c0 = S.central_cell(nPBC)
    nc = d["neighCell"].astype(np.int32) if d["pbc"] else np.where(ng >= 0, c0, -1).astype(np.int32)
    if lvec is None:
        lvec = d.get("lvec", np.eye(3) * 20.0)
    lv = np.asarray(lvec, np.float64).reshape(3, 3)
    el = np.array([{"H": 0, "C": 1, "N": 2, "O": 3}.get(t.split("_")[0], 1) for t in d["type_names"]], np.int32)
    rep = lambda a: np.concatenate([a] * nsys)  # noqa: E731
    return S.SystemBatch(np.full(nsys, na, np.int32), np.full(nsys, nn, np.int32), rep(d["apos"]), rep(ng), rep(nc),
                         rep(bk), rep(d["REQs"]), rep(d["apars"]), rep(d["bLs"]), rep(d["bKs"]), rep(d["Ksp"]),
                         rep(d["Kpp"]), np.repeat(lv[None], nsys, 0), rep(el))
