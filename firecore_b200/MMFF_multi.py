"""Drop-in for ``pyBall.MMFF_multi``: the same functions, argument names,
defaults and numpy buffer views, bound to ``libMMFFmulti_lib.so`` of this
package instead of FireCore's OpenCL library.

    from firecore_b200 import MMFF_multi as mmff
    mmff.init(nSys_=100, xyz_name="mol.xyz", surf_name="NaCl_4x4_L3.xyz", gridStep=0.1)
    mmff.getBuffs()
    nsteps = mmff.run(nstepMax=2000, Fconv=1e-4)
    E = mmff.eval()

The reference module's interface (pyBall/MMFF_multi.py) is mirrored function
by function.  ``init`` types the molecule as FireCore does: with FireCore's
tables from ``common_resources/`` under the working directory (the files the
reference reads), else with the four table names passed to ``init``; only when
neither exists does the library fall back to its own parameter table.
"""
from __future__ import annotations

import ctypes
from ctypes import c_bool, c_char_p, c_double, c_float, c_int, c_void_p, POINTER

import numpy as np

from . import _lib

c_double_p = POINTER(c_double)
c_float_p = POINTER(c_float)
c_int_p = POINTER(c_int)

lib = _lib.load()


def _np_as(arr, atype):
    return None if arr is None else arr.ctypes.data_as(atype)


def cstr(s):
    return None if s is None else s.encode("utf8")


def _sig(name, args, res=None):
    f = getattr(lib, name)
    f.argtypes = args
    f.restype = res
    return f


_sig("sample_DistConstr", [c_double] * 5 + [c_int, c_double_p, c_double_p, c_double_p])
for _n in ("sample_evalPiAling", "sample_evalAngleCos", "sample_evalAngleCosHalf"):
    _sig(_n, [c_double] * 4 + [c_int, c_double_p, c_double_p, c_double_p])
_sig("sampleNonBond", [c_int, c_double_p, c_double_p, c_double_p, c_int, c_double_p, c_double_p, c_double, c_double])
_sig("sampleSurf", [c_char_p, c_int, c_double_p, c_double_p, c_double_p, c_int, c_int, c_double, c_double, c_double,
                    c_double_p, c_bool])
_sig("sampleSurf_vecs", [c_char_p, c_int, c_double_p, c_double_p, c_double_p, c_int, c_int, c_double, c_double,
                         c_double, c_double_p, c_bool])
_sig("printBuffNames", [])
_sig("getIBuff", [c_char_p], c_int_p)
_sig("getBuff", [c_char_p], c_double_p)
_sig("getfBuff", [c_char_p], c_float_p)
_sig("init_buffers", [])
_sig("setVerbosity", [c_int, c_int])
_sig("init", [c_int, c_char_p, c_char_p, c_char_p, c_bool, c_bool, c_void_p, c_void_p, c_double, c_char_p, c_char_p,
              c_char_p, c_char_p, c_double, c_double, c_int, c_int, c_double, c_double, c_int], c_void_p)
_sig("insertSMILES", [c_char_p])
_sig("setSwitches_multi", [c_int] * 9)
_sig("checkInvariants", [c_double] * 3, c_bool)
_sig("set_opt", [c_double] * 6 + [c_int, c_double, c_double])
_sig("setOptLog", [c_int] + [c_double_p] * 5)
_sig("setTrjName", [c_char_p, c_int], c_bool)
_sig("saveXYZ", [c_char_p, c_char_p, c_int], c_int)
_sig("getTypeName", [c_int, c_bool], c_char_p)
_sig("eval", [], c_double)
_sig("run", [c_int, c_double, c_double, c_int, c_double_p, c_double_p, c_int], c_int)
_sig("MDloop", [c_int, c_double, c_int, c_int])
_sig("pack_system", [c_int, c_bool, c_bool, c_bool, c_bool])
_sig("unpack_system", [c_int, c_bool, c_bool])
_sig("upload_sys", [c_int, c_bool, c_bool, c_bool, c_bool])
_sig("download_sys", [c_int, c_bool, c_bool])
_sig("upload", [c_bool, c_bool, c_bool, c_bool])
_sig("download", [c_bool, c_bool])
_sig("change_lvec", [c_double_p, c_bool, c_bool])
_sig("optimizeLattice_1d", [c_double_p, c_int, c_int, c_int, c_double])
_sig("optimizeLattice_2d_multi", [c_double_p, c_int, c_int, c_double])
_sig("upload_pop", [c_char_p])
_sig("addDistConstrain", [c_int, c_int] + [c_double] * 5 + [c_double_p, c_bool])
_sig("addAngConstrain", [c_int, c_int, c_int, c_double, c_double])
_sig("shift_atoms_ax", [c_int, c_int_p, c_double_p])
_sig("shift_atoms", [c_int, c_int_p, c_int, c_int, c_double])
_sig("rotate_atoms_ax", [c_int, c_int_p, c_double_p, c_double_p, c_double])
_sig("rotate_atoms", [c_int, c_int_p, c_int, c_int, c_int, c_double])
_sig("scanTranslation_ax", [c_int, c_int_p, c_double_p, c_int, c_double_p, c_char_p, c_bool])
_sig("scanTranslation", [c_int, c_int_p, c_int, c_int, c_double, c_int, c_double_p, c_char_p, c_bool])
_sig("scanRotation_ax", [c_int, c_int_p, c_double_p, c_double_p, c_double, c_int, c_double_p, c_char_p])
_sig("scanRotation", [c_int, c_int_p, c_int, c_int, c_int, c_double, c_int, c_double_p, c_char_p])
_sig("scan", [c_int] + [c_double_p] * 5 + [c_bool, c_bool, c_int, c_double, c_double, c_double])

isInitialized = False


def addDistConstrain(i0, i1, lmin=1, lmax=1, kmin=1, kmax=1, flim=1e+300, l=None, k=None, shift=(0., 0., 0.),
                     bOldIndex=False):
    """Flat-bottom spring between atoms i0 and i1 of every replica (l / k set
    both bounds / both constants), applied by the next relaxations.
    bOldIndex: indices count atoms in the input order."""
    if l is not None:
        lmin = lmax = l
    if k is not None:
        kmin = kmax = k
    sh = np.ascontiguousarray(shift, np.float64)
    return lib.addDistConstrain(i0, i1, lmin, lmax, kmin, kmax, flim, _np_as(sh, c_double_p), bOldIndex)


def addAngConstrain(i0, i1, i2, ang0=0.0, k=1.0):
    """Hold the angle i1-i0-i2 (i0 the centre) at ang0 [rad]; active once a
    distance constraint exists, as in FireCore."""
    return lib.addAngConstrain(i0, i1, i2, ang0, k)


glob_bMMFF = True
nSys = 0


def _samp(fn, xs, *args, Es=None, Fs=None):
    n = len(xs)
    Es = np.zeros(n) if Es is None else Es
    Fs = np.zeros(n) if Fs is None else Fs
    xs = np.ascontiguousarray(xs, np.float64)
    fn(*args, n, _np_as(xs, c_double_p), _np_as(Es, c_double_p), _np_as(Fs, c_double_p))
    return Es, Fs


def sample_DistConstr(xs, lmin=1, lmax=1, kmin=1, kmax=1, flim=1e+300, Es=None, Fs=None):
    return _samp(lib.sample_DistConstr, xs, lmin, lmax, kmin, kmax, flim, Es=Es, Fs=Fs)


def sample_evalPiAling(angles, K=1.0, ang0=0.0, r1=1., r2=1., Es=None, Fs=None):
    return _samp(lib.sample_evalPiAling, angles, K, ang0, r1, r2, Es=Es, Fs=Fs)


def sample_evalAngleCos(angles, K=1.0, ang0=0.0, r1=1., r2=1., Es=None, Fs=None):
    return _samp(lib.sample_evalAngleCos, angles, K, ang0, r1, r2, Es=Es, Fs=Fs)


def sample_evalAngleCosHalf(angles, K=1.0, ang0=0.0, r1=1., r2=1., Es=None, Fs=None):
    return _samp(lib.sample_evalAngleCosHalf, angles, K, ang0, r1, r2, Es=Es, Fs=Fs)


def sampleNonBond(rs, Es=None, fs=None, kind=1, REQi=(1.487, 0.0006808, 0.0, 0.), REQj=(1.487, 0.0006808, 0.0, 0.), K=-1.,
                  Rdamp=1.0):
    n = len(rs)
    Es = np.zeros(n) if Es is None else Es
    fs = np.zeros(n) if fs is None else fs
    rs = np.ascontiguousarray(rs, np.float64)
    ri = np.array(REQi, np.float64); rj = np.array(REQj, np.float64)
    lib.sampleNonBond(n, _np_as(rs, c_double_p), _np_as(Es, c_double_p), _np_as(fs, c_double_p), kind,
                      _np_as(ri, c_double_p), _np_as(rj, c_double_p), K, Rdamp)
    return Es, fs


def sampleSurf(name, rs, Es=None, fs=None, kind=1, atyp=0, Q=0.0, K=-1.0, Rdamp=1.0, pos0=(0., 0., 0.), bSave=False):
    n = len(rs)
    Es = np.zeros(n) if Es is None else Es
    fs = np.zeros(n) if fs is None else fs
    rs = np.ascontiguousarray(rs, np.float64); p0 = np.array(pos0, np.float64)
    lib.sampleSurf(cstr(name), n, _np_as(rs, c_double_p), _np_as(Es, c_double_p), _np_as(fs, c_double_p), kind, atyp, Q, K,
                   Rdamp, _np_as(p0, c_double_p), bSave)
    return Es, fs


def sampleSurf_vecs(ps, Es=None, fs=None, kind=1, atyp=0, Q=0.0, K=-1.0, Rdamp=1.0, pos0=(0., 0., 0.), name=None,
                    bSave=False):
    ps = np.ascontiguousarray(ps, np.float64)
    n = len(ps)
    Es = np.zeros(n) if Es is None else Es
    fs = np.zeros((n, 3)) if fs is None else fs
    p0 = np.array(pos0, np.float64)
    lib.sampleSurf_vecs(cstr(name), n, _np_as(ps, c_double_p), _np_as(Es, c_double_p), _np_as(fs, c_double_p), kind, atyp,
                        Q, K, Rdamp, _np_as(p0, c_double_p), bSave)
    return Es, fs


def getBuff(name, sh):
    sh = sh if isinstance(sh, tuple) else (sh,)
    return np.ctypeslib.as_array(lib.getBuff(name.encode("utf8")), shape=sh)


def getfBuff(name, sh):
    sh = sh if isinstance(sh, tuple) else (sh,)
    return np.ctypeslib.as_array(lib.getfBuff(name.encode("utf8")), shape=sh)


def getIBuff(name, sh):
    sh = sh if isinstance(sh, tuple) else (sh,)
    return np.ctypeslib.as_array(lib.getIBuff(name.encode("utf8")), shape=sh)


def getBuffs(NEIGH_MAX=4):
    """Numpy views of the host mirrors (shapes as pyBall/MMFF_multi.py:210-257;
    the FP32 GPU mirrors are float4 per entry)."""
    global ndims, Es, nDOFs, natoms, nnode, ncap, npi, nvecs
    global DOFs, fDOFs, vDOFs, apos, fapos, pipos, fpipos, neighs, selection
    global gpu_neighs, gpu_neighCell, gpu_bkNeighs, gpu_atoms, gpu_aforces, gpu_avel, gpu_constr
    global gpu_REQs, gpu_MMpars, gpu_BLs, gpu_BKs, gpu_Ksp, gpu_Kpp, gpu_lvecs, gpu_ilvecs
    ndims = getIBuff("ndims", (6,))
    Es = getBuff("Es", (6,))
    nDOFs, nnode, ncap, nvecs = int(ndims[0]), int(ndims[1]), int(ndims[2]), int(ndims[3])
    natoms = nnode + ncap
    npi = nnode
    apos = getBuff("apos", (natoms, 3))
    fapos = getBuff("fapos", (natoms, 3))
    DOFs = getBuff("DOFs", (nvecs, 3))
    fDOFs = getBuff("fDOFs", (nvecs, 3))
    vDOFs = getBuff("vDOFs", (nvecs, 3))
    pipos = getBuff("pipos", (npi, 3))
    fpipos = getBuff("fpipos", (npi, 3))
    neighs = getIBuff("neighs", (nnode, NEIGH_MAX))
    selection = getIBuff("selection", (natoms,))
    gpu_neighs = getIBuff("gpu_neighs", (nSys, nvecs, 4))
    gpu_neighCell = getIBuff("gpu_neighCell", (nSys, nvecs, 4))
    gpu_bkNeighs = getIBuff("gpu_bkNeighs", (nSys, nvecs, 4))
    gpu_atoms = getfBuff("gpu_atoms", (nSys, nvecs, 4))
    gpu_aforces = getfBuff("gpu_aforces", (nSys, nvecs, 4))
    gpu_avel = getfBuff("gpu_avel", (nSys, nvecs, 4))
    gpu_constr = getfBuff("gpu_constr", (nSys, natoms, 4))
    gpu_REQs = getfBuff("gpu_REQs", (nSys, natoms, 4))
    gpu_MMpars = getfBuff("gpu_MMpars", (nSys, nnode, 4))
    gpu_BLs = getfBuff("gpu_BLs", (nSys, nnode, 4))
    gpu_BKs = getfBuff("gpu_BKs", (nSys, nnode, 4))
    gpu_Ksp = getfBuff("gpu_Ksp", (nSys, nnode, 4))
    gpu_Kpp = getfBuff("gpu_Kpp", (nSys, nnode, 4))
    gpu_lvecs = getfBuff("gpu_lvecs", (nSys, 3, 4))
    gpu_ilvecs = getfBuff("gpu_ilvecs", (nSys, 3, 4))


def init_buffers():
    return lib.init_buffers()


def setVerbosity(verbosity=1, idebug=0):
    return lib.setVerbosity(verbosity, idebug)


def init(nSys_=10, xyz_name="input.xyz", surf_name=None, smile_name=None, sElementTypes="data/ElementTypes.dat",
         sAtomTypes="data/AtomTypes.dat", sBondTypes="data/BondTypes.dat", sAngleTypes="data/AngleTypes.dat", bMMFF=True,
         bEpairs=False, nPBC=(1, 1, 0), gridnPBC=(1, 1, 0), gridStep=0.1, T=-1, gamma=-1, nExplore=0, nRelax=0,
         pos_kick=0.0, vel_kick=0.0, GridFF=5):
    global glob_bMMFF, nSys, isInitialized
    nSys = nSys_
    glob_bMMFF = bMMFF
    npbc = np.array(nPBC, np.int32)
    gnpbc = np.array(gridnPBC, np.int32)
    r = lib.init(nSys, cstr(xyz_name), cstr(surf_name), cstr(smile_name), bMMFF, bEpairs, _lib.ptr(npbc), _lib.ptr(gnpbc),
                 gridStep, cstr(sElementTypes), cstr(sAtomTypes), cstr(sBondTypes), cstr(sAngleTypes), T, gamma, nExplore,
                 nRelax, pos_kick, vel_kick, GridFF)
    if not r:
        raise RuntimeError("init failed: " + lib.mmff_last_error().decode())
    isInitialized = True
    return r


def tryInit():
    if not isInitialized:
        init()


def insertSMILES(s):
    return lib.insertSMILES(s.encode("utf8"))


def setSwitches_multi(doAngles=0, doPiPiT=0, doPiSigma=0, doPiPiI=0, doBonded=0, PBC=0, CheckInvariants=0, dovdW=0,
                      bSaveToDatabase=0):
    return lib.setSwitches_multi(doAngles, doPiPiT, doPiSigma, doPiPiI, doBonded, PBC, CheckInvariants, dovdW,
                                 bSaveToDatabase)


def checkInvariants(maxVcog=1e-9, maxFcog=1e-9, maxTg=1e-1):
    return lib.checkInvariants(maxVcog, maxFcog, maxTg)


def set_opt(dt_max=0.1, dt_min=0.02, damp_max=0.2, finc=1.1, fdec=0.5, falpha=0.8, minLastNeg=5, cvf_min=-0.1,
            cvf_max=+0.1):
    return lib.set_opt(dt_max, dt_min, damp_max, finc, fdec, falpha, minLastNeg, cvf_min, cvf_max)


def setOptLog(n):
    arrs = [np.zeros(n) for _ in range(5)]
    lib.setOptLog(n, *[_np_as(a, c_double_p) for a in arrs])
    return tuple(arrs)


def setTrjName(trj_fname_="trj.xyz", savePerNsteps=1, bDel=True):
    if bDel:
        open(trj_fname_, "w").close()
    return lib.setTrjName(cstr(trj_fname_), savePerNsteps)


def saveXYZ(fname, comment, imod=1):
    return lib.saveXYZ(cstr(fname), cstr(comment), imod)


def getTypeName(ia, fromFF=True):
    return lib.getTypeName(ia, fromFF).decode()


def eval():
    return lib.eval()


def run(nstepMax=1000, dt=-1, Fconv=1e-3, ialg=2, outE=None, outF=None, iParalel=1):
    return lib.run(nstepMax, dt, Fconv, ialg, _np_as(outE, c_double_p), _np_as(outF, c_double_p), iParalel)


def MDloop(perframe=100, Ftol=-1, iParalel=3, perVF=100):
    return lib.MDloop(perframe, Ftol, iParalel, perVF)


def pack_system(isys, bParams=False, bForces=False, bVel=False, blvec=True):
    return lib.pack_system(isys, bParams, bForces, bVel, blvec)


def unpack_system(isys, bForces=True, bVel=True):
    return lib.unpack_system(isys, bForces, bVel)


def upload_sys(isys, bParams=False, bForces=False, bVel=True, blvec=True):
    return lib.upload_sys(isys, bParams, bForces, bVel, blvec)


def download_sys(isys, bForces=False, bVel=False):
    return lib.download_sys(isys, bForces, bVel)


def upload(bParams=False, bForces=False, bVel=True, blvec=True):
    return lib.upload(bParams, bForces, bVel, blvec)


def download(bForces=False, bVel=False):
    return lib.download(bForces, bVel)


def change_lvec(lvec, bAdd=False, bUpdatePi=False):
    lv = np.ascontiguousarray(lvec, np.float64).reshape(9)
    return lib.change_lvec(_np_as(lv, c_double_p), bAdd, bUpdatePi)


def optimizeLattice_1d(dlvec, n1=5, n2=5, initMode=0, tol=1e-6):
    dl = np.ascontiguousarray(dlvec, np.float64).reshape(9)
    return lib.optimizeLattice_1d(_np_as(dl, c_double_p), n1, n2, initMode, tol)


def optimizeLattice_2d_multi(dlvec, nstesp=10, initMode=0, tol=1e-6):
    dl = np.ascontiguousarray(dlvec, np.float64).reshape(9)
    return lib.optimizeLattice_2d_multi(_np_as(dl, c_double_p), nstesp, initMode, tol)


def upload_pop(fname):
    return lib.upload_pop(cstr(fname))


def scan(poss, rots=None, Es=None, aforces=None, aposs=None, bF=False, bP=False, omp=False, bRelax=False, niter_max=10000,
         dt=0.05, Fconv=1e-5, Flim=100.0):
    poss = np.ascontiguousarray(poss, np.float64)
    nconf = len(poss)
    if rots is None:
        rots = np.tile(np.eye(3), (nconf, 1, 1))
    rots = np.ascontiguousarray(rots, np.float64)
    Es = np.zeros(nconf) if Es is None else Es
    if bF and aforces is None:
        aforces = np.zeros((nconf, natoms, 3))
    if bP and aposs is None:
        aposs = np.zeros((nconf, natoms, 3))
    lib.scan(nconf, _np_as(poss, c_double_p), _np_as(rots, c_double_p), _np_as(Es, c_double_p),
             _np_as(aforces, c_double_p), _np_as(aposs, c_double_p), omp, bRelax, niter_max, dt, Fconv, Flim)
    return Es, aforces, aposs
