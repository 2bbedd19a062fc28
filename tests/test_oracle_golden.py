"""The FP64 oracle against FireCore's own C++ physics (golden fixtures made by
tests/golden/make_golden.py from oracle/_ref, the reference compiled from its
sources).  CPU only."""
import numpy as np
import pytest

from conftest import batch_from_golden, grid_from_golden
from oracle import oracle as O

FLAGSETS = {"full": O.DEFAULT_FLAGS, "nogrid": O.DEFAULT_FLAGS & ~O.GRID, "nopbc": O.DEFAULT_FLAGS & ~O.PBC & ~O.GRID}


@pytest.mark.parametrize("tag", ["A", "B"])
@pytest.mark.parametrize("fset", list(FLAGSETS))
def test_eval_matches_reference(golden, tag, fset):
    b = batch_from_golden(golden, tag)
    P = O.make_params(grid_from_golden(golden), flags=FLAGSETS[fset])
    F, E = O.eval_forces(b, P, golden["C"])
    Fr, Er = golden[f"{tag}_{fset}_F"], golden[f"{tag}_{fset}_E"]
    # same FP64 operation order as the reference: agreement to rounding
    assert np.abs(F - Fr).max() <= 1e-12 * max(1.0, np.abs(Fr).max())
    assert np.abs(E - Er).max() <= 1e-12 * max(1.0, np.abs(Er).max())


@pytest.mark.parametrize("tag", ["A", "B"])
@pytest.mark.parametrize("run", [("r200", 200), ("rfull", 3000)])
def test_fire_trajectory_matches_reference(golden, tag, run):
    name, nit = run
    b = batch_from_golden(golden, tag)
    P = O.make_params(grid_from_golden(golden))
    r = O.relax(b, P, O.make_fire(), golden["C"], niter=nit, Fconv=1e-4, conv_mode=0)
    assert np.array_equal(r["nsteps"], golden[f"{tag}_{name}_nsteps"])
    assert np.abs(r["pos"] - golden[f"{tag}_{name}_pos"]).max() < 1e-9
    assert np.abs(r["vel"] - golden[f"{tag}_{name}_vel"]).max() < 1e-9
    assert np.abs(r["fire_state"][:, :3] - golden[f"{tag}_{name}_fire"]).max() < 1e-12


def test_grid_sample_matches_reference(golden):
    P = O.make_params(grid_from_golden(golden))
    fe = O.grid_sample(golden["samp_pos"], golden["samp_PLQ"], golden["C"], P)
    assert np.abs(fe - golden["samp_fe"]).max() <= 1e-12 * np.abs(golden["samp_fe"]).max()


def test_req2plq_matches_reference(golden):
    assert np.array_equal(O.req2plq(golden["samp_REQ"]), golden["samp_PLQ"])


def test_grid_node_potentials_match_reference(golden):
    V = golden["V"]; idx = golden["node_idx"]
    mine = V[idx[:, 0], idx[:, 1], idx[:, 2]]
    ref = golden["node_V"]
    assert np.abs(mine - ref).max() <= 1e-7 * np.abs(ref).max()


def test_bspline_fit_is_limit_of_reference_fit(golden):
    # reference fit3D_omp (x-fastest [nz][ny][nx]) converged to Ftol=1e-13
    E = golden["fit_E"].transpose(2, 1, 0)
    C = O.bspline_fit(np.repeat(E[..., None], 3, axis=3))[..., 0]
    G = golden["fit_G"].transpose(2, 1, 0)
    assert np.abs(C - G).max() <= 1e-10 * np.abs(G).max()


def test_oracle_grid_potentials_reproduce_golden(golden):
    from firecore_b200.systems import Substrate
    sub = Substrate(golden["spos"], golden["sREQ"], golden["slvec"], grid_from_golden(golden), 1.5, (1, 1, 0), (4, 4, 0))
    V = O.grid_potentials(sub)
    assert np.abs(V - golden["V"]).max() <= 1e-12 * np.abs(golden["V"]).max()
    assert np.abs(O.bspline_fit(V) - golden["C"]).max() <= 1e-10 * np.abs(golden["C"]).max()
