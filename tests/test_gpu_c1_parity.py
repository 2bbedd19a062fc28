"""Parity at the scale of the GPU workload: 64 systems shaped like the 4096-replica
benchmark batch (60-atom molecules, random rigid rotation, 0.15 A noise, 3 A
above the NaCl slab, full 226 x 226 x 200 GridFF, 10 A cutoff, x,y images),
CUDA path through the C-ABI against the FP64 oracle on the same inputs.

Bars (FP32 force arithmetic, FP64 reductions):
  forces   : per atom (and pi vector) |F_gpu - F_ref| / |F_ref| <= 1e-5 for
             >= 99.9 % of them, and <= 3e-5 for every one (starting geometries,
             |F| ~ 0.01-50 eV/A)
  energies : |E_gpu - E_ref| / |E_ref| <= 1e-6 for every system
  relaxed  : both relax to max|F| < 1e-4 eV/A (<= 4000 FIRE steps, 10 eV/A
             clamp): the same systems converge (at most 2 differ at the step
             limit), final energies agree to
             1e-5 eV/atom, end points within 1e-3 A RMSD for >= 80 % of the
             systems, and for every system the same minimum (both end points
             re-relaxed by the FP64 oracle to Fmax < 1e-6 agree to 1e-3 A).
The relaxed-geometry fraction is the measured one (87 % on this batch): along
soft modes (k ~ 0.01 eV/A^2) an end point at Fmax < 1e-4 can sit ~0.01 A from
another, and the FP32 rounding of the bond and pair forces (~1e-6 eV/A per term
near a minimum) changes a few FIRE decisions on the way there.
"""
import numpy as np
import pytest

from firecore_b200 import systems as S
from firecore_b200.world import DEFAULT_FLAGS, FireParams, World
from oracle import oracle as O

pytestmark = pytest.mark.gpu

NSYS = 64
RCUT = 10.0


@pytest.fixture(scope="module")
def c1():
    sub = S.make_slab()
    w = World(0)
    C = w.grid_build(sub, return_coefs=True)
    b = S.config_replicas(seed=1, nrep=NSYS)
    w.set_params(flags=DEFAULT_FLAGS, npbc=(1, 1, 0), Rcut=RCUT)
    w.set_fire(FireParams(Flim=10.0))
    w.upload(b)
    yield w, b, sub, C
    w.set_params(flags=DEFAULT_FLAGS)
    w.set_fire(FireParams())


def test_c1_forces_and_energies_per_atom(c1):
    w, b, sub, C = c1
    w.restore()
    F, E = w.eval(True)
    pos = w.state()["pos"]
    Fo, Eo = O.eval_forces(b, O.make_params(sub.grid, npbc=(1, 1, 0), Rcut=RCUT), C, pos=pos)
    rel = np.linalg.norm(F - Fo, axis=1) / np.maximum(np.linalg.norm(Fo, axis=1), 1e-30)
    assert (rel <= 1e-5).mean() >= 0.999, np.quantile(rel, [0.5, 0.99, 0.999, 1.0])
    assert rel.max() <= 3e-5, rel.max()
    erel = np.abs(E[:, 3] - Eo[:, 3]) / np.abs(Eo[:, 3])
    assert erel.max() <= 1e-6, erel.max()
    # the reference's split into bonded / non-bonded / grid parts is kept (the
    # parts carry the 1-3 pair energies the total leaves out, ~1e2 eV)
    assert np.abs(E[:, :3] - Eo[:, :3]).max() <= 1e-5 * np.abs(Eo[:, :3]).sum(1).max()


def test_c1_relaxed_geometries(c1):
    w, b, sub, C = c1
    w.restore()
    pos0 = w.state()["pos"]
    w.relax(4000, 1e-4, conv_mode=1)
    st = w.state()
    P = O.make_params(sub.grid, npbc=(1, 1, 0), Rcut=RCUT)
    F = O.make_fire(Flim=10.0)
    r = O.relax(b, P, F, C, niter=4000, Fconv=1e-4, conv_mode=1, pos=pos0)
    assert ((st["status"] == 1) != (r["converged"] == 1)).sum() <= 2
    both = [s for s in range(b.nsys) if st["status"][s] == 1 and r["converged"][s] == 1]
    assert len(both) >= 16
    _, _, v = b.offsets()
    _, Eg = O.eval_forces(b, P, C, pos=st["pos"])
    _, Ec = O.eval_forces(b, P, C, pos=r["pos"])

    def rmsd(pa, pb, s):
        na = b.natoms[s]
        d = pa[v[s]:v[s] + na] - pb[v[s]:v[s] + na]
        return float(np.sqrt((d ** 2).sum(1).mean()))

    dE = np.array([abs(Eg[s, 3] - Ec[s, 3]) / b.natoms[s] for s in both])
    assert dE.max() <= 1e-5, dE.max()
    rm = np.array([rmsd(st["pos"], r["pos"], s) for s in both])
    assert (rm <= 1e-3).mean() >= 0.8, np.sort(rm)
    sb = b.subset(both)
    rows = np.concatenate([np.arange(v[s], v[s + 1]) for s in both])
    Ft = O.make_fire(Flim=10.0)
    td = O.relax(sb, P, Ft, C, niter=30000, Fconv=1e-6, conv_mode=1, pos=st["pos"][rows])
    to = O.relax(sb, P, Ft, C, niter=30000, Fconv=1e-6, conv_mode=1, pos=r["pos"][rows])
    assert (td["converged"] == 1).all() and (to["converged"] == 1).all()
    _, _, vb = sb.offsets()
    tight = [float(np.sqrt(((td["pos"][vb[k]:vb[k] + sb.natoms[k]] - to["pos"][vb[k]:vb[k] + sb.natoms[k]]) ** 2)
                           .sum(1).mean())) for k in range(sb.nsys)]
    assert max(tight) <= 1e-3, tight
