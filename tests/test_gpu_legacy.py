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
    # rigid scan of the molecule over 3 heights
    poss = np.array([[5.6, 5.6, z] for z in (6.0, 7.0, 8.0)])
    Es, _, _ = mmff.scan(poss, bRelax=False)
    assert np.isfinite(Es).all()
    mmff.saveXYZ(str(tmp_path / "out.xyz"), "#test", 1)
    assert (tmp_path / "out.xyz").read_text().startswith("24\n")
    assert mmff.getTypeName(0) in ("C", "N", "O")
