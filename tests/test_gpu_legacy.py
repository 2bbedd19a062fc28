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
