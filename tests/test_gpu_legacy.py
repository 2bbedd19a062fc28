"""The pyBall.MMFF_multi-compatible interface (firecore_b200.MMFF_multi over the
legacy symbols of libMMFFmulti_lib.so): init from xyz files, the named host
buffers, run / eval / scan, on the GPU."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_legacy_init_run_eval_scan(tmp_path):
    from firecore_b200 import MMFF_multi as mmff
    mmff.init(nSys_=8, xyz_name=os.path.join(HERE, "mol24.xyz"), surf_name=os.path.join(HERE, "NaCl_2x2_L2.xyz"),
              gridStep=0.2, nPBC=(1, 1, 0))
    mmff.getBuffs()
    assert mmff.natoms == 24 and mmff.nnode == 14 and mmff.nvecs == 38
    assert mmff.gpu_atoms.shape == (8, 38, 4) and mmff.gpu_REQs.shape == (8, 24, 4)
    assert (mmff.gpu_bkNeighs[0, :24] >= -1).all()
    p0 = mmff.gpu_atoms[:, :24, :3].copy()
    # perturb replicas differently through the host mirrors, then upload
    rng = np.random.default_rng(0)
    mmff.gpu_atoms[:, :24, :3] += rng.normal(0, 0.05, (8, 24, 3)).astype(np.float32)
    mmff.upload(bParams=False, bForces=False, bVel=True)
    mmff.set_opt(dt_max=0.1, dt_min=0.01, damp_max=0.1, minLastNeg=3)
    nsteps = mmff.run(nstepMax=3000, Fconv=1e-3)
    assert 0 < nsteps <= 3000
    assert np.isfinite(mmff.gpu_atoms).all()
    assert np.abs(mmff.gpu_atoms[:, :24, :3] - p0).max() > 1e-3     # the mirrors were refreshed
    E = mmff.eval()
    assert np.isfinite(E)
    assert np.allclose(mmff.Es[0], E)
    # scan_relaxed (MolWorld_sp3_multi.h:1242-1296): 5 placements, atom 0 pinned
    # to each target by a unit spring, every configuration relaxed on the queue
    poss = np.array([[5.6, 5.6, z] for z in (6.0, 6.5, 7.0, 7.5, 8.0)])
    Es, aforces, aposs = mmff.scan(poss, bF=True, bP=True, bRelax=True, niter_max=4000, Fconv=1e-3)
    assert np.isfinite(Es).all() and np.isfinite(aforces).all()
    assert aposs.shape == (5, 24, 3)
    # the pinned atom stays near its target (spring force = the net other force)
    d = np.linalg.norm(aposs[:, 0, :] - poss, axis=1)
    assert d.max() < 1.0, d
    # the replicas of init() are back
    mmff.download()
    assert mmff.gpu_atoms.shape == (8, 38, 4) and np.isfinite(mmff.gpu_atoms).all()
    mmff.saveXYZ(str(tmp_path / "out.xyz"), "#test", 1)
    assert (tmp_path / "out.xyz").read_text().startswith("24\n")
    assert mmff.getTypeName(0) in ("C", "N", "O")


def test_legacy_init_types_with_firecore_tables(tmp_path, monkeypatch):
    """init reads FireCore-format tables from common_resources/ under the working
    directory (as MolWorld_sp3::init does), types the molecule with
    mmff_build_xyz, and the device world evaluates that force field: forces and
    energy against the FP64 oracle on the same arrays."""
    from builder_tables import write_tables
    from firecore_b200 import MMFF_multi as mmff
    from firecore_b200 import topology as T
    from oracle import oracle as O
    O.build_oracle()
    tables = write_tables(str(tmp_path / "common_resources"))
    monkeypatch.chdir(tmp_path)
    xyz = os.path.join(HERE, "mol24.xyz")
    mmff.init(nSys_=4, xyz_name=xyz, nPBC=(1, 1, 0))
    mmff.getBuffs()
    d = T.build_xyz(xyz, tables)
    na, nn = d["natoms"], d["nnode"]
    assert mmff.natoms == na and mmff.nnode == nn
    assert [mmff.getTypeName(i) for i in range(na)] == d["type_names"]
    for buf, key in ((mmff.gpu_REQs, "REQs"), (mmff.gpu_MMpars, "apars"), (mmff.gpu_BLs, "bLs"), (mmff.gpu_BKs, "bKs"),
                     (mmff.gpu_Ksp, "Ksp"), (mmff.gpu_Kpp, "Kpp")):
        np.testing.assert_array_equal(buf[3], d[key].astype(np.float32), err_msg=key)
    np.testing.assert_array_equal(mmff.gpu_atoms[0, :, :3], d["apos"].astype(np.float32))
    np.testing.assert_array_equal(mmff.gpu_neighs[0, :na], d["neighs"])
    E = mmff.eval()
    b = T.to_batch(d)
    b.pos = mmff.gpu_atoms[0, :, :3].astype(np.float64)          # the float32 positions the device holds
    Fo, Eo = O.eval_forces(b, O.make_params(flags=O.DEFAULT_FLAGS, npbc=(1, 1, 0)))
    assert abs(E - Eo[0, 3]) <= 2e-6 * max(1.0, abs(Eo[0, 3])), (E, Eo[0])
    F = mmff.gpu_aforces[0, :, :3]
    scale = np.abs(Fo).max()
    assert np.abs(F - Fo).max() <= 2e-5 * scale, (np.abs(F - Fo).max(), scale)
    # and it relaxes
    mmff.set_opt(dt_max=0.05, dt_min=0.005, damp_max=0.1, minLastNeg=3)
    n = mmff.run(nstepMax=2000, Fconv=1e-3)
    assert 0 < n <= 2000 and np.isfinite(mmff.gpu_atoms).all()
    assert mmff.eval() < E


def test_legacy_distance_and_angle_constraints(tmp_path, monkeypatch):
    """addDistConstrain / addAngConstrain (libMMFF.h:41-47) act on every
    replica in the next run, as FireCore's default run path applies its
    Constrains to all replicas."""
    from firecore_b200 import MMFF_multi as mmff
    monkeypatch.chdir(tmp_path)                       # no FireCore tables here: the library's own table
    mmff.init(nSys_=4, xyz_name=os.path.join(HERE, "mol24.xyz"), nPBC=(1, 1, 0))
    mmff.getBuffs()
    p0 = mmff.gpu_atoms[:, :24, :3].copy()
    d0 = np.linalg.norm(p0[:, 0] - p0[:, 9], axis=1)
    mmff.set_opt(dt_max=0.05, dt_min=0.005, damp_max=0.1, minLastNeg=3)
    # relaxed without constraints
    mmff.run(nstepMax=3000, Fconv=1e-3)
    free = np.linalg.norm(mmff.gpu_atoms[:, 0, :3] - mmff.gpu_atoms[:, 9, :3], axis=1)
    # again from the start, atoms 0 and 9 held 1 A further apart
    mmff.gpu_atoms[:, :24, :3] = p0
    mmff.gpu_avel[:] = 0
    mmff.upload(bParams=False, bForces=False, bVel=True)
    mmff.addDistConstrain(0, 9, l=float(d0[0]) + 1.0, k=5.0, flim=20.0)
    mmff.addAngConstrain(1, 0, 2, ang0=2.0, k=0.5)
    mmff.run(nstepMax=3000, Fconv=1e-3)
    held = np.linalg.norm(mmff.gpu_atoms[:, 0, :3] - mmff.gpu_atoms[:, 9, :3], axis=1)
    assert np.isfinite(mmff.gpu_atoms).all()
    assert (held > free + 0.3).all(), (held, free)
    assert np.abs(held - held[0]).max() < 1e-3        # the same on every replica


def test_legacy_run_explores_with_gopt(tmp_path, monkeypatch):
    """init(T, gamma, nExplore, nRelax) + run(iParalel=2): the exploring cycle of
    run_ocl_opt with GOpt; every replica starts exploring, the cycle's state
    continues across calls and the replicas draw different noise."""
    import ctypes
    from firecore_b200 import MMFF_multi as mmff, _lib
    monkeypatch.chdir(tmp_path)
    mmff.init(nSys_=4, xyz_name=os.path.join(HERE, "mol24.xyz"), nPBC=(1, 1, 0), T=300.0, gamma=0.5, nExplore=20,
              nRelax=150)
    mmff.getBuffs()
    p0 = mmff.gpu_atoms[:, :24, :3].copy()
    assert mmff.run(nstepMax=300, Fconv=1e-3, iParalel=2) == 300
    gopt = np.zeros((4, 4), np.int32)
    lib = _lib.load()
    assert lib.mmff_get_explore(ctypes.c_void_p(gopt.ctypes.data), None) == 0
    assert (gopt[:, 2] + gopt[:, 3] >= 1).all(), gopt      # a phase ended on every replica
    assert mmff.run(nstepMax=200, Fconv=1e-3, iParalel=2) == 200
    g2 = np.zeros((4, 4), np.int32)
    assert lib.mmff_get_explore(ctypes.c_void_p(g2.ctypes.data), None) == 0
    assert (g2[:, 2] + g2[:, 3] >= gopt[:, 2] + gopt[:, 3]).all()
    mmff.MDloop(perframe=100, iParalel=3)                  # MDloop's run_ocl_opt: the same cycle goes on
    g3 = np.zeros((4, 4), np.int32)
    assert lib.mmff_get_explore(ctypes.c_void_p(g3.ctypes.data), None) == 0
    assert (g3[:, 2] + g3[:, 3] >= g2[:, 2] + g2[:, 3]).all()
    assert np.isfinite(mmff.gpu_atoms).all()
    p = mmff.gpu_atoms[:, :24, :3]
    assert np.abs(p - p0).max() > 1e-2
    assert np.abs(p[1] - p[0]).max() > 1e-3                 # different noise per replica
