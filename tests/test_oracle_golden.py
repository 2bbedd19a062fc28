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


# distance / angle constraints of the test below: (i0, i1, lmin, lmax, kmin, kmax, flim, shift a, b, c)
# and (centre, end 1, end 2, ang0, k); the second distance spring reaches into the next cell
DIST = [(0, 5, 2.0, 2.2, 1.5, 0.8, 3.0, 0.0, 0.0, 0.0), (2, 9, 12.0, 12.5, 0.6, 0.6, 0.5, 1.0, 0.0, 0.0)]
ANG = [(1, 0, 2, 2.0, 0.7)]


@pytest.mark.skipif(not O.ref_available(), reason="reference harness not built (FireCore tree absent)")
def test_constraints_match_reference_run_no_omp(golden):
    """The oracle's distance / angle constraints against FireCore's own
    Constrains::apply inside MolWorld_sp3::run_no_omp, run live through the
    reference harness: 300 FIRE steps of one golden molecule."""
    import ctypes
    b = batch_from_golden(golden, "A").subset([0])
    g = grid_from_golden(golden)
    flags = FLAGSETS["nogrid"]
    na, nn = int(b.natoms[0]), int(b.nnode[0])
    ref = O.ref()
    ref.ref_set_constraints.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                        ctypes.c_void_p]
    p = lambda a: ctypes.c_void_p(a.ctypes.data)  # noqa: E731
    pos = np.ascontiguousarray(b.pos)
    arr = [np.ascontiguousarray(x) for x in (b.neighs, b.neighCell, b.REQs)]
    nar = [np.ascontiguousarray(x) for x in (b.apars, b.bLs, b.bKs, b.Ksp, b.Kpp)]
    lv = np.ascontiguousarray(b.lvec[0].reshape(9))
    npbc = np.array([1, 1, 0], np.int32)
    gn = np.array(g.n, np.int32); gp0 = np.array(g.pos0); gst = np.array(g.step)
    bk = np.zeros((na, 4), np.int32); ng = np.zeros((na, 4), np.int32)
    C = np.ascontiguousarray(golden["C"])           # held: the harness reads it during the call
    ref.ref_setup(na, nn, p(pos), p(arr[0]), p(arr[1]), p(arr[2]), *[p(x) for x in nar], p(lv), p(npbc), flags, 1.5,
                  p(gn), p(gp0), p(gst), p(C), p(bk), p(ng))
    di = np.array([d[:2] for d in DIST], np.int32); dp = np.array([d[2:] for d in DIST], np.float64)
    ai = np.array([a[:3] for a in ANG], np.int32); ap = np.array([a[3:] for a in ANG], np.float64)
    ref.ref_set_constraints(len(DIST), p(di), p(dp), len(ANG), p(ai), p(ap))
    nit = 300
    pr = pos.copy(); vr = np.zeros_like(pr)
    fr = np.array([0.1, 0.1, 0.0, 0.1, 0.01, 0.1, 1.1, 0.5, 0.8, 3, 0.0])
    oE = np.zeros(nit); oF = np.zeros(nit)
    it = ref.ref_relax(nit, 1e-9, p(pr), p(vr), p(fr), p(oE), p(oF))
    r = O.relax(b, O.make_params(g, flags=flags), O.make_fire(), golden["C"], niter=nit, Fconv=1e-9, conv_mode=0,
                dist=[(-1,) + d for d in DIST], angles=[(-1,) + a for a in ANG])
    assert int(r["nsteps"][0]) == it
    assert np.abs(r["pos"] - pr).max() < 1e-9
    # and the constraints act: without them the trajectory differs
    r0 = O.relax(b, O.make_params(g, flags=flags), O.make_fire(), golden["C"], niter=nit, Fconv=1e-9, conv_mode=0)
    assert np.abs(r0["pos"] - pr).max() > 1e-3


@pytest.mark.skipif(not O.ref_available(), reason="reference harness not built (FireCore tree absent)")
@pytest.mark.parametrize("fset", ["nogrid", "full"])
def test_explore_cycle_matches_reference_run_no_omp(golden, fset, tmp_path, monkeypatch):
    """The oracle's exploring cycle against FireCore's MolWorld_sp3::run_no_omp
    with bGopt (GOpt update at the top of every step, FIRE scalars evolving while
    exploring, a minimum starting an exploring phase), run live through the
    reference harness: 1500 steps of one golden molecule that starts exploring,
    with nExplore 15 and a noise-free drive (T = 0, friction 0.1).  run_no_omp
    returns at every step where the system sits below Fconv, and its Langevin
    step takes the FIRE dt of the call's start, so the oracle runs the same
    pieces with that dt."""
    import ctypes
    # a minimum found makes run_no_omp append to ./gopt.xyz; a directory of
    # that name makes the open fail before the write
    monkeypatch.chdir(tmp_path)
    (tmp_path / "gopt.xyz").mkdir()
    b = batch_from_golden(golden, "A").subset([0])
    g = grid_from_golden(golden)
    flags = FLAGSETS[fset]
    na, nn = int(b.natoms[0]), int(b.nnode[0])
    ref = O.ref()
    ref.ref_set_gopt.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int]
    ref.ref_get_gopt.argtypes = [ctypes.c_void_p]
    p = lambda a: ctypes.c_void_p(a.ctypes.data)  # noqa: E731
    pos = np.ascontiguousarray(b.pos)
    arr = [np.ascontiguousarray(x) for x in (b.neighs, b.neighCell, b.REQs)]
    nar = [np.ascontiguousarray(x) for x in (b.apars, b.bLs, b.bKs, b.Ksp, b.Kpp)]
    lv = np.ascontiguousarray(b.lvec[0].reshape(9))
    npbc = np.array([1, 1, 0], np.int32)
    gn = np.array(g.n, np.int32); gp0 = np.array(g.pos0); gst = np.array(g.step)
    bk = np.zeros((na, 4), np.int32); ng = np.zeros((na, 4), np.int32)
    C = np.ascontiguousarray(golden["C"])           # held: the harness reads it during the calls
    ref.ref_setup(na, nn, p(pos), p(arr[0]), p(arr[1]), p(arr[2]), *[p(x) for x in nar], p(lv), p(npbc), flags, 1.5,
                  p(gn), p(gp0), p(gst), p(C), p(bk), p(ng))
    ref.ref_set_gopt(1, 15, 0.0, 0.1, 1, 0)
    try:
        pr = pos.copy(); vr = np.zeros_like(pr)
        fr = np.array([0.1, 0.1, 0.0, 0.1, 0.01, 0.1, 1.1, 0.5, 0.8, 3, 0.0])
        P = O.make_params(g, flags=flags); F = O.make_fire()
        st = dict(pos=None, vel=None, fire_state=None, gopt=np.array([[1, 0, 0, 0]], np.int32), minpos=None)
        total, found, N = 0, 0, 1500
        gs = np.zeros(2, np.int32)
        while total < N:
            nit = N - total
            oE = np.zeros(nit); oF = np.zeros(nit)
            dt0 = fr[0]
            it = ref.ref_relax(nit, 0.05, p(pr), p(vr), p(fr), p(oE), p(oF))
            ref.ref_get_gopt(p(gs))
            n = it + 1 if it < nit else nit          # run_no_omp breaks after step it
            st = O.explore(b, P, F, golden["C"], nsteps=n, Fconv=0.05, conv_mode=0, n_explore=15,
                           dt=float(np.float32(dt0)), gamma=0.1, T=0.0, pos=st["pos"], vel=st["vel"],
                           fire_state=st["fire_state"], gopt=st["gopt"], minpos=st["minpos"])
            assert tuple(st["gopt"][0][:2]) == tuple(gs)
            assert np.abs(st["pos"] - pr).max() < 1e-9
            assert np.abs(st["vel"] - vr).max() < 1e-9
            assert np.abs(st["fire_state"][0, :3] - fr[:3]).max() < 1e-9
            if gs[0] == 1 and gs[1] == 0:            # a minimum ended this call
                found += 1
                assert np.abs(st["minpos"] - pr).max() < 1e-9
            total += n
        assert found >= 3 and int(st["gopt"][0][2]) == found
    finally:
        ref.ref_set_gopt(0, 0, 0.0, 0.0, 0, 0)
