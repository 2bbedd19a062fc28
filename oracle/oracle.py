"""Python bindings of the FP64 oracle (mmff_oracle.c) and of the reference
harness (oracle/_ref/libref_harness.so, FireCore's own C++ physics).

TEST INFRASTRUCTURE: the checker.  Imported only by tests/, by
__graft_entry__.smoke() and by bench.py's CPU-baseline / reference arm.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORC_LIB = os.path.join(HERE, "_build", "libmmff_oracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libref_harness.so")

# flag bits (mmff_oracle.h)
BONDS, PIPI, PISIGMA, ANGLES = 1, 2, 4, 8
SUB_ANGLE_NB, SUB_BOND_NB, CLAMP_NB = 16, 32, 64
NONBONDED, GRID, PBC = 128, 256, 512
# run_no_omp with bNonBondNeighs: bSubtractAngleNonBond on, bond subtraction and
# clamping off (ForceField.h:170-186 setNonBondStrategy(+1))
DEFAULT_FLAGS = BONDS | PIPI | PISIGMA | ANGLES | SUB_ANGLE_NB | NONBONDED | GRID | PBC


class ORCParams(ctypes.Structure):
    _fields_ = [("flags", ctypes.c_int), ("npbc", ctypes.c_int * 3), ("Rcut", ctypes.c_double),
                ("Ron", ctypes.c_double), ("FmaxNonBonded", ctypes.c_double), ("alphaMorse", ctypes.c_double),
                ("gn", ctypes.c_int * 3), ("gpos0", ctypes.c_double * 3), ("gstep", ctypes.c_double * 3)]


class ORCFire(ctypes.Structure):
    _fields_ = [("dt_max", ctypes.c_double), ("dt_min", ctypes.c_double), ("damp_max", ctypes.c_double),
                ("finc", ctypes.c_double), ("fdec", ctypes.c_double), ("falpha", ctypes.c_double),
                ("cv_kill", ctypes.c_double), ("minLastNeg", ctypes.c_int), ("variant", ctypes.c_int),
                ("Flim", ctypes.c_double)]


def _p(a):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return ctypes.c_void_p(a.ctypes.data)


_orc = None
_ref = None


def build_oracle(with_ref: bool = False):
    """Compile the checkers (make in oracle/); the reference harness only where
    the reference tree is present."""
    subprocess.check_call(["make", "-s", "-C", HERE, "all"])
    ref_root = os.environ.get("REF_ROOT", "/root/reference")
    if with_ref and os.path.isdir(os.path.join(ref_root, "cpp")):
        subprocess.check_call(["make", "-s", "-C", HERE, "ref", f"REF_ROOT={ref_root}"])


def orc():
    global _orc
    if _orc is None:
        if not os.path.exists(ORC_LIB):
            build_oracle()
        _orc = ctypes.CDLL(ORC_LIB)
    return _orc


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def ref():
    global _ref
    if _ref is None:
        _ref = ctypes.CDLL(REF_LIB)
        _ref.ref_setup.restype = ctypes.c_int
        _ref.ref_setup.argtypes = [ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 11 + [ctypes.c_int, ctypes.c_double] + \
            [ctypes.c_void_p] * 6
        _ref.ref_relax.restype = ctypes.c_int
        _ref.ref_relax.argtypes = [ctypes.c_int, ctypes.c_double] + [ctypes.c_void_p] * 5
        _ref.ref_eval.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        _ref.ref_grid_sample.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        _ref.ref_req2plq.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p]
        _ref.ref_fit3d.restype = ctypes.c_int
        _ref.ref_fit3d.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double, ctypes.c_int,
                                   ctypes.c_double]
        _ref.ref_grid_points.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double,
                                         ctypes.c_void_p]
    return _ref


def make_params(grid=None, flags=DEFAULT_FLAGS, npbc=(1, 1, 0), Rcut=-1.0, Ron=-1.0, alphaMorse=1.5,
                FmaxNonBonded=10.0) -> ORCParams:
    P = ORCParams()
    P.flags = flags
    P.npbc[:] = list(npbc)
    P.Rcut = Rcut
    P.Ron = Ron
    P.FmaxNonBonded = FmaxNonBonded
    P.alphaMorse = alphaMorse
    if grid is not None:
        P.gn[:] = [int(x) for x in grid.n]
        P.gpos0[:] = [float(x) for x in grid.pos0]
        P.gstep[:] = [float(x) for x in grid.step]
    else:
        P.flags &= ~GRID
    return P


def make_fire(dt_max=0.1, dt_min=0.01, damp_max=0.1, finc=1.1, fdec=0.5, falpha=0.8, minLastNeg=3,
              cv_kill=0.0, Flim=-1.0, variant=0) -> ORCFire:
    """Defaults = DynamicOpt after setTimeSteps(0.1) / initOpt (DynamicOpt.h:73-95, 199-205)."""
    F = ORCFire()
    F.dt_max, F.dt_min, F.damp_max, F.finc, F.fdec, F.falpha, F.cv_kill = dt_max, dt_min, damp_max, finc, fdec, falpha, cv_kill
    F.minLastNeg = minLastNeg
    F.Flim = Flim
    F.variant = variant
    return F


def _sysarrays(b):
    """Contiguous copies of the topology/parameter arrays (the caller keeps them
    alive for the duration of the native call)."""
    return [np.ascontiguousarray(b.neighs, np.int32), np.ascontiguousarray(b.neighCell, np.int32),
            np.ascontiguousarray(b.bkneighs, np.int32), np.ascontiguousarray(b.REQs, np.float64),
            np.ascontiguousarray(b.apars, np.float64), np.ascontiguousarray(b.bLs, np.float64),
            np.ascontiguousarray(b.bKs, np.float64), np.ascontiguousarray(b.Ksp, np.float64),
            np.ascontiguousarray(b.Kpp, np.float64), np.ascontiguousarray(b.lvec.reshape(-1, 9), np.float64)]


def eval_forces(b, P: ORCParams, gridC=None, pos=None, nthreads=0):
    """Forces [sum nvecs, 3] and energies [nsys, 4] (bonded, non-bonded, grid, total)."""
    lib = orc()
    pos = np.ascontiguousarray(b.pos if pos is None else pos, np.float64)
    force = np.zeros_like(pos)
    Es = np.zeros((b.nsys, 4))
    keep = [np.ascontiguousarray(b.natoms, np.int32), np.ascontiguousarray(b.nnode, np.int32)]
    g = None if gridC is None else np.ascontiguousarray(gridC, np.float64)
    arrs = _sysarrays(b)
    lib.orc_eval(ctypes.c_int(b.nsys), _p(keep[0]), _p(keep[1]), _p(pos), _p(force), _p(Es), *[_p(a) for a in arrs],
                 _p(g), ctypes.byref(P), ctypes.c_int(nthreads))
    return force, Es


def relax(b, P: ORCParams, F: ORCFire, gridC=None, niter=1000, Fconv=1e-4, conv_mode=0, pos=None, vel=None,
          fire_state=None, nthreads=0, constr=None, constrK=None, dist=(), angles=()):
    """FIRE relaxation (run_no_omp semantics). Returns dict of arrays.
    constr / constrK [sum natoms, 4] (optional): per-atom position springs,
    anchor (x, y, z, on if w > 0) and constants (kx, ky, kz, -) in the same
    frame as pos.  dist / angles: distance and angle constraints as
    World.set_bond_constraints takes them."""
    lib = orc()
    pos = np.array(b.pos if pos is None else pos, np.float64, order="C")
    vel = np.zeros_like(pos) if vel is None else np.array(vel, np.float64, order="C")
    if fire_state is None:
        fire_state = np.zeros((b.nsys, 4))
        fire_state[:, 0] = F.dt_max
        fire_state[:, 1] = F.damp_max
    fire_state = np.array(fire_state, np.float64, order="C")
    nsteps = np.zeros(b.nsys, np.int32); conv = np.zeros(b.nsys, np.int32)
    Fout = np.zeros(b.nsys); Eout = np.zeros((b.nsys, 4))
    keep = [np.ascontiguousarray(b.natoms, np.int32), np.ascontiguousarray(b.nnode, np.int32)]
    g = None if gridC is None else np.ascontiguousarray(gridC, np.float64)
    arrs = _sysarrays(b)
    di = np.array([[int(x) for x in d[:3]] for d in dist], np.int32).reshape(-1, 3)
    dp = np.zeros((len(dist), 8))
    for r, d in enumerate(dist):
        dp[r, :len(d) - 3] = d[3:]
    ai = np.array([[int(x) for x in a[:4]] for a in angles], np.int32).reshape(-1, 4)
    ap = np.array([a[4:6] for a in angles], np.float64).reshape(-1, 2)
    cs = None if constr is None else np.ascontiguousarray(constr, np.float64)
    ck = None if constrK is None else np.ascontiguousarray(constrK, np.float64)
    lib.orc_relax(ctypes.c_int(b.nsys), _p(keep[0]), _p(keep[1]), _p(pos), _p(vel), _p(fire_state), *[_p(a) for a in arrs],
                  _p(g), ctypes.byref(P), ctypes.byref(F), ctypes.c_int(niter), ctypes.c_double(Fconv),
                  ctypes.c_int(conv_mode), _p(nsteps), _p(conv), _p(Fout), _p(Eout), ctypes.c_int(nthreads),
                  _p(cs), _p(ck), ctypes.c_int(len(dist)), _p(di), _p(dp), ctypes.c_int(len(angles)), _p(ai), _p(ap))
    return dict(pos=pos, vel=vel, fire_state=fire_state, nsteps=nsteps, converged=conv, F=Fout, E=Eout)


def md(b, P: ORCParams, gridC=None, nsteps=10, dt=0.05, gamma=0.1, T=300.0, seed=12345, step0=0, pos=None,
       vel=None, Flim=-1.0, nthreads=0):
    """Langevin dynamics (MMFFsp3_loc::move_atom_Langevin) with the counter-based
    noise stream of the device kernels. Returns dict(pos, vel)."""
    lib = orc()
    pos = np.array(b.pos if pos is None else pos, np.float64, order="C")
    vel = np.zeros_like(pos) if vel is None else np.array(vel, np.float64, order="C")
    keep = [np.ascontiguousarray(b.natoms, np.int32), np.ascontiguousarray(b.nnode, np.int32)]
    g = None if gridC is None else np.ascontiguousarray(gridC, np.float64)
    arrs = _sysarrays(b)
    lib.orc_md(ctypes.c_int(b.nsys), _p(keep[0]), _p(keep[1]), _p(pos), _p(vel), *[_p(a) for a in arrs], _p(g),
               ctypes.byref(P), ctypes.c_int(nsteps), ctypes.c_double(dt), ctypes.c_double(gamma), ctypes.c_double(T),
               ctypes.c_ulonglong(seed), ctypes.c_int(step0), ctypes.c_double(Flim), ctypes.c_int(nthreads))
    return dict(pos=pos, vel=vel)


def explore(b, P: ORCParams, F: ORCFire, gridC=None, nsteps=10, Fconv=1e-4, conv_mode=1, n_explore=10, n_relax=0,
            dt=0.05, gamma=0.1, T=300.0, seed=12345, step0=0, pos=None, vel=None, fire_state=None, gopt=None,
            minpos=None, nthreads=0):
    """Exploring cycle of GOpt (orc_explore): FIRE relaxation, a Langevin phase of
    n_explore steps after every minimum found or after n_relax FIRE steps without
    one. Returns dict(pos, vel, fire_state, gopt [nsys, 4], minpos)."""
    lib = orc()
    pos = np.array(b.pos if pos is None else pos, np.float64, order="C")
    vel = np.zeros_like(pos) if vel is None else np.array(vel, np.float64, order="C")
    if fire_state is None:
        fire_state = np.zeros((b.nsys, 4))
        fire_state[:, 0] = F.dt_max
        fire_state[:, 1] = F.damp_max
    fire_state = np.array(fire_state, np.float64, order="C")
    gopt = np.zeros((b.nsys, 4), np.int32) if gopt is None else np.array(gopt, np.int32, order="C")
    minpos = pos.copy() if minpos is None else np.array(minpos, np.float64, order="C")
    keep = [np.ascontiguousarray(b.natoms, np.int32), np.ascontiguousarray(b.nnode, np.int32)]
    g = None if gridC is None else np.ascontiguousarray(gridC, np.float64)
    arrs = _sysarrays(b)
    lib.orc_explore(ctypes.c_int(b.nsys), _p(keep[0]), _p(keep[1]), _p(pos), _p(vel), _p(fire_state), _p(gopt),
                    _p(minpos), *[_p(a) for a in arrs], _p(g), ctypes.byref(P), ctypes.byref(F), ctypes.c_int(nsteps),
                    ctypes.c_double(Fconv), ctypes.c_int(conv_mode), ctypes.c_int(n_explore), ctypes.c_int(n_relax),
                    ctypes.c_double(dt), ctypes.c_double(gamma), ctypes.c_double(T), ctypes.c_ulonglong(seed),
                    ctypes.c_int(step0), ctypes.c_int(nthreads))
    return dict(pos=pos, vel=vel, fire_state=fire_state, gopt=gopt, minpos=minpos)


def surf(pos, REQ, sub, Rdamp=1.0):
    """Direct substrate term of atoms at pos [n,3] with REQ [n,4]: [n,4] (F, E)."""
    lib = orc()
    pos = np.ascontiguousarray(pos, np.float64); REQ = np.ascontiguousarray(REQ, np.float64)
    spos = np.ascontiguousarray(sub.spos, np.float64); sREQ = np.ascontiguousarray(sub.sREQ, np.float64)
    lv = np.ascontiguousarray(sub.lvec.reshape(9), np.float64); nm = np.array(sub.nPBC_mors, np.int32)
    fe = np.zeros((pos.shape[0], 4))
    lib.orc_surf(ctypes.c_int(pos.shape[0]), _p(pos), _p(REQ), ctypes.c_int(spos.shape[0]), _p(spos), _p(sREQ),
                 _p(lv), _p(nm), ctypes.c_double(sub.alphaMorse), ctypes.c_double(Rdamp), _p(fe))
    return fe


def langevin_rand(seed, vec, step, comp):
    lib = orc()
    lib.orc_langevin_rand.restype = ctypes.c_double
    lib.orc_langevin_rand.argtypes = [ctypes.c_ulonglong, ctypes.c_longlong, ctypes.c_int, ctypes.c_int]
    return lib.orc_langevin_rand(seed, vec, step, comp)


def grid_sample(pos, PLQ, gridC, P: ORCParams):
    pos = np.ascontiguousarray(pos, np.float64); PLQ = np.ascontiguousarray(PLQ, np.float64)
    fe = np.zeros((pos.shape[0], 4))
    C = np.ascontiguousarray(gridC, np.float64)      # held for the duration of the call
    orc().orc_grid_sample(ctypes.c_int(pos.shape[0]), _p(pos), _p(PLQ), _p(C), ctypes.byref(P), _p(fe))
    return fe


def req2plq(REQ, K=1.5):
    REQ = np.ascontiguousarray(REQ, np.float64)
    out = np.zeros_like(REQ)
    orc().orc_req2plq(ctypes.c_int(REQ.shape[0]), _p(REQ), ctypes.c_double(K), _p(out))
    return out


def grid_potentials(sub, nthreads=0):
    """FP64 node potentials [nx, ny, nz, 3] of a Substrate (direct sums)."""
    P = make_params(sub.grid, alphaMorse=sub.alphaMorse)
    nx, ny, nz = sub.grid.n
    V = np.zeros((nx, ny, nz, 3))
    nm = np.array(sub.nPBC_mors, np.int32); nc = np.array(sub.nPBC_coul, np.int32)
    sp = np.ascontiguousarray(sub.spos, np.float64); sq = np.ascontiguousarray(sub.sREQ, np.float64)
    lv = np.ascontiguousarray(sub.lvec.reshape(9), np.float64)   # held for the duration of the call
    orc().orc_grid_potentials(ctypes.c_int(sub.spos.shape[0]), _p(sp), _p(sq), _p(lv),
                              _p(nm), _p(nc), ctypes.byref(P), _p(V), ctypes.c_int(nthreads))
    return V


def bspline_fit(V):
    V = np.ascontiguousarray(V, np.float64)
    gn = np.array(V.shape[:3], np.int32)
    C = np.zeros_like(V)
    orc().orc_bspline_fit(_p(gn), _p(V), _p(C))
    return C

