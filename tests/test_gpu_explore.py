"""Exploring cycle of the global optimiser (GOpt as MolWorld_sp3_multi drives
it): the CUDA relax kernels (warp- and CTA-per-system) through the C-ABI
against the FP64 oracle's restatement, which is pinned to FireCore's
run_no_omp with bGopt (tests/test_oracle_golden.py).  Both sides draw the
Langevin noise from the same counter-based stream.  Positions are compared to
1e-3 A after tens of FIRE and Langevin steps (FP32 forces against FP64), the
cycle's counters exactly."""
import numpy as np
import pytest

from conftest import grid_from_golden
from firecore_b200 import systems as S
from firecore_b200.world import DEFAULT_FLAGS, FireParams, World
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SIZES = [[24] * 8, [20, 57, 64, 65, 120, 200, 300]]


@pytest.fixture(scope="module")
def world(golden):
    w = World(0)
    w.grid_upload(golden["C"], grid_from_golden(golden))
    return w


def _setup(world, sizes, seed):
    b = S.make_systems(sizes, seed=seed, topo_mode=1, sigma=0.05, cell=(22.56, 22.56, 40.0))
    world.set_params(flags=DEFAULT_FLAGS, npbc=(1, 1, 0), Rcut=10.0)
    world.set_fire(FireParams(Flim=10.0))
    world.upload(b)
    return b


def _oracle_params(golden):
    return O.make_params(grid_from_golden(golden), npbc=(1, 1, 0), Rcut=10.0), O.make_fire(Flim=10.0)


@pytest.mark.parametrize("sizes", SIZES)
def test_explore_give_up_cycle_vs_oracle(world, golden, sizes):
    """No system reaches Fconv: every 21 FIRE steps a relax phase is given up
    and 7 Langevin steps (nExplore 8) follow.  70 steps in two calls (the
    random stream and the cycle's state continue across calls)."""
    b = _setup(world, sizes, 23)
    st0 = world.state()
    world.set_md(dt=0.05, gamma=0.5, T=300.0, seed=7)
    world.set_explore(8, 20)
    world.explore(40, Fconv=1e-9, conv_mode=1)
    world.explore(30, Fconv=1e-9, conv_mode=1)
    st = world.state()
    gopt, minpos = world.explore_state()
    P, F = _oracle_params(golden)
    r = O.explore(b, P, F, golden["C"], nsteps=70, Fconv=1e-9, conv_mode=1, n_explore=8, n_relax=20, dt=0.05,
                  gamma=0.5, T=300.0, seed=7, step0=0, pos=st0["pos"], vel=st0["vel"], fire_state=st0["fire"])
    assert np.array_equal(gopt, r["gopt"]), (gopt, r["gopt"])
    assert (gopt[:, 3] == 2).all() and (gopt[:, 2] == 0).all()
    assert np.array_equal(minpos, st0["pos"])        # no minimum found: the positions of set_explore
    assert np.abs(st["pos"] - st0["pos"]).max() > 1e-2
    err = np.abs(st["pos"] - r["pos"]).max()
    assert err < 1e-3, err
    assert np.allclose(st["fire"][:, :3], r["fire_state"][:, :3], rtol=1e-6, atol=1e-9)
    assert (st["nsteps"] == 30).all() and (st["status"] == 2).all()     # steps of the last call


@pytest.mark.parametrize("sizes", SIZES)
def test_explore_minimum_then_explore_vs_oracle(world, golden, sizes):
    """Systems relaxed below Fconv find a minimum at the first step of the
    cycle: that geometry is kept, 9 Langevin steps at 300 K follow (nExplore 10)
    and FIRE resumes for the last 20 steps (the first of them ends the exploring
    phase and counts as step 0 of the relax phase)."""
    b = _setup(world, sizes, 31)
    world.relax(8000, 5e-5, conv_mode=1)
    st0 = world.state()
    ok = st0["status"] == 1
    assert ok.sum() >= len(sizes) // 2
    world.set_md(dt=0.05, gamma=0.5, T=300.0, seed=11)
    world.set_explore(10, 0)
    world.explore(30, Fconv=5e-4, conv_mode=1)
    st = world.state()
    gopt, minpos = world.explore_state()
    P, F = _oracle_params(golden)
    r = O.explore(b, P, F, golden["C"], nsteps=30, Fconv=5e-4, conv_mode=1, n_explore=10, n_relax=0, dt=0.05,
                  gamma=0.5, T=300.0, seed=11, step0=0, pos=st0["pos"], vel=st0["vel"], fire_state=st0["fire"])
    a, n, v = b.offsets()
    for s in np.flatnonzero(ok):
        assert tuple(gopt[s]) == (0, 19, 1, 0) == tuple(r["gopt"][s]), (s, gopt[s], r["gopt"][s])
        rows = slice(v[s], v[s + 1])
        assert np.abs(minpos[rows] - st0["pos"][rows]).max() < 1e-3      # the minimum: one FIRE step away
        assert np.abs(minpos[rows] - r["minpos"][rows]).max() < 1e-4
        assert np.abs(st["pos"][rows] - st0["pos"][rows]).max() > 1e-3  # the drive moved it
        err = np.abs(st["pos"][rows] - r["pos"][rows]).max()
        assert err < 1e-3, (s, err)


def test_explore_needs_setup(world):
    b = S.make_systems([24] * 2, seed=3, topo_mode=1, sigma=0.05, cell=(22.56, 22.56, 40.0))
    world.set_params(flags=DEFAULT_FLAGS, npbc=(1, 1, 0), Rcut=10.0)
    world.upload(b)
    with pytest.raises(RuntimeError, match="mmff_set_explore"):
        world.explore(5)
    with pytest.raises(RuntimeError, match="no exploring cycle"):
        world.explore_state()
    with pytest.raises(RuntimeError, match="n_explore must be >= 0"):
        world.set_explore(-1, 0)
    world.set_explore(4, 0)
    world.explore(5)
    gopt, _ = world.explore_state()
    assert (gopt[:, 1] >= 0).all() and gopt.shape == (2, 4)
    world.upload(b)                       # new systems: the cycle is set up again
    with pytest.raises(RuntimeError, match="mmff_set_explore"):
        world.explore(5)
