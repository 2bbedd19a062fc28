"""CUDA path (through the C-ABI) against the FP64 oracle and the reference's
golden outputs.  Tolerances (FP32 forces, FP64 reductions):
  forces   : max_i |F_gpu - F_ref| <= FTOL * max_i |F_ref|   per system
  energies : |E_gpu - E_ref| <= ETOL * (|E_bonded| + |E_nb| + |E_grid|)
  relaxed  : final energy within 1e-5 eV/atom, RMSD <= 1e-3 A
"""
import os

import numpy as np
import pytest

from conftest import batch_from_golden, grid_from_golden
from firecore_b200 import systems as S
from firecore_b200.world import DEFAULT_FLAGS, GRID, NONBONDED, PBC, FireParams, World
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FTOL = 1e-5
ETOL = 1e-5
FLAGSETS = {"full": DEFAULT_FLAGS, "nogrid": DEFAULT_FLAGS & ~GRID, "nopbc": DEFAULT_FLAGS & ~PBC & ~GRID}


@pytest.fixture(scope="module")
def world(golden):
    w = World(0)
    w.grid_upload(golden["C"], grid_from_golden(golden))
    return w


def per_system_force_err(b, F, Fr):
    a, n, v = b.offsets()
    errs = []
    for s in range(b.nsys):
        d = np.abs(F[v[s]:v[s + 1]] - Fr[v[s]:v[s + 1]]).max()
        errs.append(d / max(np.abs(Fr[v[s]:v[s + 1]]).max(), 1e-12))
    return np.array(errs)


def check_eval(world, b, grid, C, flags, npbc=(1, 1, 0), Rcut=-1.0):
    world.set_params(flags=flags, npbc=npbc, Rcut=Rcut)
    world.upload(b)
    F, E = world.eval(True)
    pos = world.state()["pos"]             # the positions the GPU holds (FP32 local frame)
    P = O.make_params(grid, flags=flags, npbc=npbc, Rcut=Rcut)
    Fo, Eo = O.eval_forces(b, P, C, pos=pos)
    ferr = per_system_force_err(b, F, Fo)
    scale = np.abs(Eo[:, :3]).sum(1)
    eerr = np.abs(E - Eo).max(1) / np.maximum(scale, 1e-9)
    return ferr, eerr


@pytest.mark.parametrize("tag", ["A", "B"])
@pytest.mark.parametrize("fset", list(FLAGSETS))
def test_eval_vs_oracle(world, golden, tag, fset):
    b = batch_from_golden(golden, tag)
    ferr, eerr = check_eval(world, b, grid_from_golden(golden), golden["C"], FLAGSETS[fset])
    assert ferr.max() < FTOL, ferr
    assert eerr.max() < ETOL, eerr


@pytest.mark.parametrize("tag", ["A", "B"])
def test_eval_vs_reference_golden(world, golden, tag):
    """Direct comparison with FireCore's own forces at the golden positions
    (includes the FP32 rounding of the inputs)."""
    b = batch_from_golden(golden, tag)
    world.set_params(flags=DEFAULT_FLAGS)
    world.upload(b)
    F, E = world.eval(True)
    ferr = per_system_force_err(b, F, golden[f"{tag}_full_F"])
    assert ferr.max() < 2e-4, ferr     # input rounding (p ~ 10 A in FP32) x bond stiffness dominates
    Er = golden[f"{tag}_full_E"]
    assert np.abs(E[:, 3] - Er[:, 3]).max() / np.abs(Er[:, :3]).sum(1).max() < 1e-5


def test_eval_cutoff_vs_oracle(world, golden):
    b = batch_from_golden(golden, "B")
    ferr, eerr = check_eval(world, b, grid_from_golden(golden), golden["C"], DEFAULT_FLAGS, Rcut=6.0)
    assert ferr.max() < FTOL and eerr.max() < ETOL


def test_grid_sample_vs_reference(world, golden):
    fe = world.grid_sample(golden["samp_pos"], golden["samp_PLQ"])
    ref = golden["samp_fe"]
    assert np.abs(fe - ref).max() <= 2e-5 * np.abs(ref).max()


def test_grid_build_vs_oracle(world, golden):
    from firecore_b200.systems import Substrate
    sub = Substrate(golden["spos"], golden["sREQ"], golden["slvec"], grid_from_golden(golden), 1.5, (1, 1, 0), (4, 4, 0))
    w2 = World(0)
    C = w2.grid_build(sub, return_coefs=True)
    ref = golden["C"]
    assert np.abs(C - ref).max() <= 1e-9 * np.abs(ref).max()
    # restore the module grid for later tests
    world.grid_upload(golden["C"], grid_from_golden(golden))


def check_eval_components(world, b, grid, C, npbc, Rcut):
    """Per-system FP32 force error against the summed magnitude of the force
    components (bonded incl. 1-3 subtraction, pairs, grid) and energy error
    against the summed component energies.  The generated molecules have close
    non-bonded contacts whose pair forces (hundreds of eV/A) cancel against the
    1-3 subtraction of the angle terms; FP32 rounding scales with those terms,
    not with the small net force."""
    world.set_params(flags=DEFAULT_FLAGS, npbc=npbc, Rcut=Rcut)
    world.upload(b)
    F, E = world.eval(True)
    pos = world.state()["pos"]
    mk = lambda fl: O.make_params(grid, flags=fl, npbc=npbc, Rcut=Rcut)
    Fo, Eo = O.eval_forces(b, mk(DEFAULT_FLAGS), C, pos=pos)
    comp = np.zeros_like(Fo)
    for fl in (DEFAULT_FLAGS & ~(GRID | NONBONDED), NONBONDED | (DEFAULT_FLAGS & PBC), GRID | (DEFAULT_FLAGS & PBC)):
        Fc, _ = O.eval_forces(b, mk(fl), C, pos=pos)
        comp += np.abs(Fc)
    a, n, v = b.offsets()
    ferr = np.array([np.abs(F[v[s]:v[s + 1]] - Fo[v[s]:v[s + 1]]).max() / comp[v[s]:v[s + 1]].max()
                     for s in range(b.nsys)])
    eerr = np.abs(E - Eo).max(1) / np.maximum(np.abs(Eo[:, :3]).sum(1), 1e-9)
    return ferr, eerr


@pytest.mark.parametrize("hbond", [False, True])
def test_uneven_pbc_cutoff_vs_oracle(world, golden, hbond):
    """Molecules of 20..400 atoms in a 22.56 A cell with x,y images and a 10 A
    cutoff: every size class, the CTA kernels' per-image candidate lists
    (large molecules reach their own images) and both pair-loop variants
    (with / without H-bond pseudo-charges).  The generated molecules have
    close non-bonded contacts whose pair forces (up to ~600 eV/A) cancel
    against the 1-3 subtraction of the angle terms, so the FP32 force error
    is measured against the summed magnitude of the force components."""
    sizes = [20, 33, 57, 64, 65, 120, 128, 129, 200, 256, 257, 330, 400]
    b = S.make_systems(sizes, seed=11, topo_mode=1, sigma=0.1, cell=(22.56, 22.56, 40.0), hbond=hbond)
    ferr, eerr = check_eval_components(world, b, grid_from_golden(golden), golden["C"], (1, 1, 0), 10.0)
    assert ferr.max() < FTOL, ferr
    assert eerr.max() < ETOL, eerr


def test_uneven_batch_vs_oracle(world, golden):
    sizes = [20, 33, 57, 64, 65, 120, 128, 129, 200, 256, 257, 400]
    b = S.make_systems(sizes, seed=3, topo_mode=1, sigma=0.1, cell=(11.28, 11.28, 40.0), npbc=(0, 0, 0))
    ferr, eerr = check_eval_components(world, b, grid_from_golden(golden), golden["C"], (0, 0, 0), 8.0)
    assert ferr.max() < FTOL, ferr
    assert eerr.max() < ETOL, eerr


FIRE_CASES = {"run_no_omp": dict(Flim=10.0),
              "bitzek": dict(Flim=10.0, variant=1, falpha=0.99, minLastNeg=5)}


@pytest.mark.parametrize("fire", list(FIRE_CASES))
def test_relax_vs_oracle(world, golden, fire):
    """Full relaxation (max |f| < 1e-4, Flim = 10): final energy and geometry.
    Both sides stop anywhere inside the Fmax < 1e-4 basin, so along soft modes
    (curvature ~0.1 eV/A^2) the end points may differ by a few 1e-3 A:
    energies must agree to 1e-5 eV/atom for every system, geometries to 1e-3 A
    RMSD for most (median) and 1e-2 A for all.  Same minimum: both end points,
    re-relaxed by the FP64 oracle to Fmax < 1e-6, agree to 1e-3 A for every
    system."""
    grid = grid_from_golden(golden)
    b = S.make_systems([24] * 16, seed=7, topo_mode=0, sigma=0.1, rotate=False, hbond=True,
                       cell=(11.28, 11.28, 40.0))
    world.set_params(flags=DEFAULT_FLAGS)
    fp = FireParams(**FIRE_CASES[fire])
    world.set_fire(fp)
    world.upload(b)
    pos0 = world.state()["pos"]
    world.relax(6000, 1e-4, conv_mode=1)
    st = world.state()
    P = O.make_params(grid)
    Fo = O.make_fire(**FIRE_CASES[fire])
    r = O.relax(b, P, Fo, golden["C"], niter=6000, Fconv=1e-4, conv_mode=1, pos=pos0)
    assert (st["status"] == 1).all(), st["status"]
    assert (r["converged"] == 1).all()
    a, n, v = b.offsets()
    _, Eg = O.eval_forces(b, P, golden["C"], pos=st["pos"])
    _, Ec = O.eval_forces(b, P, golden["C"], pos=r["pos"])
    rmsds = []
    for s in range(b.nsys):
        na = b.natoms[s]
        dE = abs(Eg[s, 3] - Ec[s, 3]) / na
        d = st["pos"][v[s]:v[s] + na] - r["pos"][v[s]:v[s] + na]
        rmsds.append(np.sqrt((d ** 2).sum(1).mean()))
        assert dE <= 1e-5, (s, dE)
    rmsds = np.array(rmsds)
    assert np.median(rmsds) <= 1e-3 and rmsds.max() <= 1e-2, rmsds
    Ft = O.make_fire(Flim=10.0)
    td = O.relax(b, P, Ft, golden["C"], niter=30000, Fconv=1e-6, conv_mode=1, pos=st["pos"])
    to = O.relax(b, P, Ft, golden["C"], niter=30000, Fconv=1e-6, conv_mode=1, pos=r["pos"])
    assert (td["converged"] == 1).all() and (to["converged"] == 1).all()
    tight = [np.sqrt(((td["pos"][v[s]:v[s] + b.natoms[s]] - to["pos"][v[s]:v[s] + b.natoms[s]]) ** 2).sum(1).mean())
             for s in range(b.nsys)]
    assert max(tight) <= 1e-3, tight
    world.set_fire(FireParams())


def test_relax_steps_match_reference_semantics(world, golden):
    """nsteps / status bookkeeping of run_no_omp: converged systems report the
    index of the converging step; unconverged ones the step limit."""
    b = batch_from_golden(golden, "A")
    world.set_params(flags=DEFAULT_FLAGS)
    world.set_fire(FireParams(Flim=10.0))
    world.upload(b)
    world.relax(50, 1e-4, conv_mode=0)
    st = world.state()
    assert (st["status"] == 2).all() and (st["nsteps"] == 50).all()
    assert np.allclose(st["fire"][:, 3], 50)
    world.relax(50, 1e-4, conv_mode=0)          # continues from the saved state
    assert np.allclose(world.state()["fire"][:, 3], 100)
    world.set_fire(FireParams())


def test_nan_system_is_retired_not_fatal(world, golden):
    """Failure detection: a system with two atoms on the same spot produces
    non-finite forces; it is flagged (status -1) and the others relax."""
    b = S.make_systems([24, 24, 24], seed=5, topo_mode=0, sigma=0.05, cell=(11.28, 11.28, 40.0))
    a, n, v = b.offsets()
    b.pos[v[1] + 20] = b.pos[v[1] + 21]          # two caps of system 1 coincide
    world.set_params(flags=DEFAULT_FLAGS)
    world.set_fire(FireParams(Flim=10.0))
    world.upload(b)
    world.relax(300, 1e-4, conv_mode=1)
    st = world.state()
    assert st["status"][1] == -1
    assert st["status"][0] in (1, 2) and st["status"][2] in (1, 2)
    world.set_fire(FireParams())


def test_queue_claims_every_system_once(world, golden):
    """More systems than resident CTAs: the persistent queue processes each once."""
    b = S.make_systems([24] * 3000, seed=9, topo_mode=0, sigma=0.05, cell=(11.28, 11.28, 40.0))
    world.set_params(flags=DEFAULT_FLAGS)
    world.upload(b)
    world.relax(7, 1e-12, conv_mode=1)
    st = world.state()
    assert (st["status"] == 2).all() and (st["nsteps"] == 7).all()
    assert np.allclose(st["fire"][:, 3], 7)


def test_bad_topology_rejected(world):
    b = S.make_systems([24], seed=1, cell=(11.28, 11.28, 40.0))
    b.neighs[3, 0] = 99                             # out of range
    with pytest.raises(RuntimeError, match="out of range"):
        world.upload(b)


@pytest.mark.parametrize("sizes", [[24] * 8, [20, 57, 64, 65, 120, 200, 300]])
def test_langevin_drive_vs_oracle(world, golden, sizes):
    """Langevin drive (MMFFsp3_loc::move_atom_Langevin): 20 steps on the device
    (warp- and CTA-per-system kernels) against the FP64 oracle fed the same
    counter-based noise stream; the stream is reproducible and continues
    across calls."""
    grid = grid_from_golden(golden)
    b = S.make_systems(sizes, seed=17, topo_mode=1, sigma=0.05, cell=(22.56, 22.56, 40.0))
    world.set_params(flags=DEFAULT_FLAGS, npbc=(1, 1, 0), Rcut=10.0)
    world.set_fire(FireParams(Flim=10.0))
    world.upload(b)
    pos0 = world.state()["pos"]
    world.set_md(dt=0.05, gamma=0.5, T=300.0, seed=99)
    world.md(10)
    world.md(10)                          # continues the random stream at step 10
    st = world.state()
    r = O.md(b, O.make_params(grid, npbc=(1, 1, 0), Rcut=10.0), golden["C"], nsteps=20, dt=0.05, gamma=0.5,
             T=300.0, seed=99, step0=0, pos=pos0, Flim=10.0)
    assert np.abs(st["pos"] - pos0).max() > 1e-3
    assert np.abs(st["pos"] - r["pos"]).max() < 1e-3, np.abs(st["pos"] - r["pos"]).max()
    world.restore()
    world.set_md(dt=0.05, gamma=0.5, T=300.0, seed=99)
    world.md(20)
    assert np.array_equal(world.state()["pos"], st["pos"])
    world.set_fire(FireParams())


def test_surface_direct_term_vs_oracle(world, golden):
    """Direct substrate term (getSurfMorse / getMorseQH): Morse + damped
    Coulomb of every atom against the substrate atoms and their images, warp-
    and CTA-per-system kernels, against the FP64 oracle."""
    from firecore_b200.world import SURF
    sub = S.make_slab(ncell=2, layers=2)
    b = S.make_systems([24] * 4 + [80, 150], seed=5, topo_mode=1, sigma=0.05, cell=(11.28, 11.28, 40.0))
    world.surf_upload(sub, Rdamp=1.0)
    world.set_params(flags=SURF, npbc=(0, 0, 0))
    world.upload(b)
    F, E = world.eval(True)
    pos = world.state()["pos"]
    a, n, v = b.offsets()
    rows = np.concatenate([np.arange(v[s], v[s] + b.natoms[s]) for s in range(b.nsys)])
    fe = O.surf(pos[rows], b.REQs, sub, 1.0)
    err = np.abs(F[rows] - fe[:, :3]).max() / np.abs(fe[:, :3]).max()
    assert err < 1e-5, err
    Es = np.array([fe[a[s]:a[s + 1], 3].sum() for s in range(b.nsys)])
    assert np.allclose(E[:, 2], Es, rtol=1e-5, atol=1e-5), (E[:, 2], Es)
    world.lib.mmff_surf_upload(0, None, None, None, None, 1.0)
    world.set_params(flags=DEFAULT_FLAGS)


def test_position_springs_vs_oracle(world, golden):
    """Per-atom position springs (relax_multi.cl:995-1010): anchors 0.3 A away
    from three atoms of every system, anisotropic constants; the relaxed
    geometries and energies match the FP64 oracle with the same springs, and
    eval reports the forces without them."""
    grid = grid_from_golden(golden)
    b = S.make_systems([24] * 8, seed=5, topo_mode=0, sigma=0.05, rotate=False, cell=(11.28, 11.28, 40.0))
    world.set_params(flags=DEFAULT_FLAGS)
    world.set_fire(FireParams(Flim=10.0))
    world.upload(b)
    pos0 = world.state()["pos"]
    a, n, v = b.offsets()
    anchor = np.zeros((int(b.natoms.sum()), 4)); anchor[:, 3] = -1.0
    K = np.zeros((int(b.natoms.sum()), 3))
    for s in range(b.nsys):
        for k, ia in enumerate((0, 5, 17)):
            anchor[a[s] + ia, :3] = pos0[v[s] + ia] + np.array([0.3, -0.2, 0.1]) * (1 + 0.1 * k)
            anchor[a[s] + ia, 3] = 1.0
            K[a[s] + ia] = (1.0, 2.0, 0.5)
    world.set_constraints(anchor, K)
    F0, _ = world.eval(False)
    Fo0, _ = O.eval_forces(b, O.make_params(grid), golden["C"], pos=pos0)
    assert np.abs(F0 - Fo0).max() <= 1e-5 * np.abs(Fo0).max()         # eval: no springs
    world.relax(6000, 1e-4, conv_mode=1)
    st = world.state()
    Kc = np.zeros((K.shape[0], 4)); Kc[:, :3] = K
    r = O.relax(b, O.make_params(grid), O.make_fire(Flim=10.0), golden["C"], niter=6000, Fconv=1e-4, conv_mode=1,
                pos=pos0, constr=anchor, constrK=Kc)
    world.set_constraints(None)
    world.set_fire(FireParams())
    assert (st["status"] == 1).all() and (r["converged"] == 1).all()
    for s in range(b.nsys):
        na = b.natoms[s]
        d = st["pos"][v[s]:v[s] + na] - r["pos"][v[s]:v[s] + na]
        assert np.sqrt((d ** 2).sum(1).mean()) <= 1e-2, s
        # the springs hold: anchored atoms moved toward their anchors
        for ia in (0, 5, 17):
            assert np.linalg.norm(st["pos"][v[s] + ia] - anchor[a[s] + ia, :3]) < np.linalg.norm(
                pos0[v[s] + ia] - anchor[a[s] + ia, :3]), (s, ia)
    _, Eg = O.eval_forces(b, O.make_params(grid), golden["C"], pos=st["pos"])
    _, Ec = O.eval_forces(b, O.make_params(grid), golden["C"], pos=r["pos"])
    assert (np.abs(Eg[:, 3] - Ec[:, 3]) / b.natoms).max() <= 1e-5


@pytest.mark.parametrize("threads", [0, 64])
def test_bond_constraints_vs_oracle(world, golden, threads):
    """Distance / angle constraints (FireCore's Constrains, constrains.h) in both
    relax engines (threads 0: the warp-per-system kernel for these 24-atom
    systems; 64: the CTA kernel), with three atoms per system held by position
    springs so that every system converges: relaxed geometries match the FP64
    oracle with the same constraints (the oracle's are pinned to FireCore's
    run_no_omp in test_oracle_golden.py), and eval reports forces without them."""
    grid = grid_from_golden(golden)
    b = S.make_systems([24] * 8, seed=5, topo_mode=0, sigma=0.05, rotate=False, cell=(11.28, 11.28, 40.0))
    dist = [(-1, 3, 12, 5.0, 5.2, 2.0, 2.0, 3.0), (3, 2, 17, 2.6, 2.8, 1.0, 1.0, 10.0, 0.0, 0.0, 0.0)]
    ang = [(-1, 1, 0, 2, 2.4, 1.5)]
    world.set_params(flags=DEFAULT_FLAGS)
    world.set_fire(FireParams(Flim=10.0))
    world.set_launch(threads=threads)
    a, n, v = b.offsets()
    try:
        world.upload(b)
        pos0 = world.state()["pos"]
        anchor = np.zeros((int(b.natoms.sum()), 4)); anchor[:, 3] = -1.0
        K = np.zeros((int(b.natoms.sum()), 4))
        for s in range(b.nsys):
            for ia in (0, 7, 17):
                anchor[a[s] + ia, :3] = pos0[v[s] + ia]; anchor[a[s] + ia, 3] = 1.0; K[a[s] + ia, :3] = 1.0
        world.set_constraints(anchor, K)
        world.set_bond_constraints(dist, ang)
        F0, _ = world.eval(False)
        Fo0, _ = O.eval_forces(b, O.make_params(grid), golden["C"], pos=pos0)
        assert np.abs(F0 - Fo0).max() <= 1e-5 * np.abs(Fo0).max()         # eval: no constraints
        world.relax(6000, 1e-4, conv_mode=1)
        st = world.state()
        world.set_bond_constraints()
        world.set_constraints(None)
    finally:
        world.set_fire(FireParams())
        world.set_launch(0)
    P, F = O.make_params(grid), O.make_fire(Flim=10.0)
    r = O.relax(b, P, F, golden["C"], niter=6000, Fconv=1e-4, conv_mode=1, pos=pos0, constr=anchor, constrK=K,
                dist=dist, angles=ang)
    r0 = O.relax(b, P, F, golden["C"], niter=6000, Fconv=1e-4, conv_mode=1, pos=pos0, constr=anchor, constrK=K)
    assert (st["status"] == 1).all() and (r["converged"] == 1).all()
    for s in range(b.nsys):
        na = b.natoms[s]
        d = st["pos"][v[s]:v[s] + na] - r["pos"][v[s]:v[s] + na]
        assert np.sqrt((d ** 2).sum(1).mean()) <= 1e-2, s
        # the constraints change the result (the unconstrained minimum is elsewhere)
        d0 = r0["pos"][v[s]:v[s] + na] - r["pos"][v[s]:v[s] + na]
        assert np.sqrt((d0 ** 2).sum(1).mean()) > 0.1, s
    # system 3 alone carries the second distance constraint
    l_gpu = np.linalg.norm(st["pos"][v[3] + 2] - st["pos"][v[3] + 17])
    l_orc = np.linalg.norm(r["pos"][v[3] + 2] - r["pos"][v[3] + 17])
    assert abs(l_gpu - l_orc) < 1e-2


def test_periodic_chain_vs_oracle(world, golden):
    """Bonds across the cell wall on the GPU: an infinite CH2 chain typed by the
    FireCore-format builder (this project's own small tables), 8 noisy copies:
    forces and energies of one evaluation, then relaxed geometries, against
    the FP64 oracle (itself pinned to FireCore on FireCore's periodic polymers,
    test_builder.py)."""
    from builder_tables import polyethylene, write_tables
    from firecore_b200 import topology as T
    import tempfile
    tmp = tempfile.mkdtemp()
    tables = write_tables(os.path.join(tmp, "t"))
    parts = []
    for k in range(8):
        path = os.path.join(tmp, f"pe{k}.xyz")
        with open(path, "w") as f:
            f.write(polyethylene(noise=0.05, seed=k))
        parts.append(T.to_batch(T.build_xyz(path, tables)))
    b = S.SystemBatch(*[np.concatenate([getattr(p, f) for p in parts]) for f in S.SystemBatch.__dataclass_fields__])
    assert (b.neighCell[b.neighs >= 0] != 4).any()
    flags = DEFAULT_FLAGS & ~O.GRID
    ferr, eerr = check_eval(world, b, None, None, flags, npbc=(1, 1, 0))
    assert ferr.max() < FTOL, ferr
    assert eerr.max() < ETOL, eerr
    world.set_params(flags=flags, npbc=(1, 1, 0))
    world.set_fire(FireParams(Flim=10.0))
    world.upload(b)
    pos0 = world.state()["pos"]
    world.relax(4000, 1e-4, conv_mode=1)
    st = world.state()
    world.set_fire(FireParams())
    P = O.make_params(None, flags=flags, npbc=(1, 1, 0))
    r = O.relax(b, P, O.make_fire(Flim=10.0), None, niter=4000, Fconv=1e-4, conv_mode=1, pos=pos0)
    assert (st["status"] == 1).all() and (r["converged"] == 1).all()
    _, Eg = O.eval_forces(b, P, None, pos=st["pos"])
    _, Ec = O.eval_forces(b, P, None, pos=r["pos"])
    assert (np.abs(Eg[:, 3] - Ec[:, 3]) / b.natoms).max() <= 1e-5
