"""Uneven batching on the GPU: the captured relax graph, the launch-
configuration autotuner and its JSON persistence, and retire/refill of the
per-bucket work queues over mixed system sizes."""
import numpy as np
import pytest

from conftest import grid_from_golden
from firecore_b200 import systems as S
from firecore_b200.world import DEFAULT_FLAGS, FireParams, World

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def world():
    return World(0)


@pytest.fixture(autouse=True)
def _restore_launch_state(world):
    """Graph mode and tuned launch shapes are library-wide: put them back."""
    yield
    world.set_graph(False)
    for c in range(6):
        world.lib.mmff_set_tuning(c, -1, 1, 0, 0)


def uneven(world, golden, n=96, seed=5, lo=20, hi=300):
    grid = grid_from_golden(golden)
    sizes = S.loguniform_sizes(n, seed, lo, hi)
    b = S.make_systems(sizes, seed, topo_mode=1, sigma=0.1, rotate=True, cell=(22.56, 22.56, 40.0))
    world.set_params(flags=DEFAULT_FLAGS, Rcut=10.0)
    world.set_fire(FireParams(Flim=10.0))
    world.grid_upload(golden["C"], grid)
    world.upload(b)
    return b


def test_graph_relax_is_identical_to_direct_launches(world, golden):
    b = uneven(world, golden)
    world.set_graph(False)
    world.restore(); world.relax(300, 1e-4, conv_mode=1)
    d = world.state()
    world.set_graph(True)
    for _ in range(2):                       # capture, then replay of the cached graph
        world.restore(); world.relax(300, 1e-4, conv_mode=1)
        g = world.state()
        assert np.array_equal(d["pos"], g["pos"]) and np.array_equal(d["status"], g["status"])
        assert np.array_equal(d["nsteps"], g["nsteps"])
    world.restore(); world.relax(100, 1e-4, conv_mode=1)         # new key: recaptured
    assert (world.state()["nsteps"] <= 100).all()
    world.set_graph(False)


def test_grid_cache_is_bit_identical(world, golden):
    """The per-atom GridFF stencil cache of the CTA kernels changes no bit:
    a relaxation (cells change every few steps early on, rarely later) and an
    evaluation with the cache on and off; also after a restore, where every
    cached cell is stale."""
    b = uneven(world, golden, n=64, seed=9, lo=40, hi=300)
    world.set_launch(128, 0)                 # CTA engine for every size
    out = {}
    for on in (False, True, True):
        world.set_grid_cache(on)
        world.restore(); world.relax(400, 1e-4, conv_mode=1)
        st = world.state()
        F, E = world.eval(True)
        out.setdefault(on, []).append((st, F, E))
    world.set_grid_cache(True)
    world.set_launch(0, 0)
    (d, Fd, Ed), = out[False]
    for g, Fg, Eg in out[True]:
        assert np.array_equal(d["pos"], g["pos"]) and np.array_equal(d["nsteps"], g["nsteps"])
        assert np.array_equal(Fd, Fg) and np.array_equal(Ed, Eg)


def test_autotune_picks_a_launchable_config_and_keeps_physics(world, golden, tmp_path):
    b = uneven(world, golden)
    for c in range(6):
        world.lib.mmff_set_tuning(c, -1, 1, 0, 0)
    world.restore(); world.relax(200, 1e-4, conv_mode=1)
    _, E_def = world.eval()
    rows = world.autotune(nstep_probe=20, max_sample=32, path=str(tmp_path / "tune.json"))
    assert rows and all(r["us_per_system_step"] > 0 or r["us_per_system_step"] < 0 for r in rows)
    tuned = world.tuning()
    classes = {r["size_class"] for r in rows}
    assert set(tuned) == classes
    for c, t in tuned.items():
        ok = [r for r in rows if r["size_class"] == c and r["us_per_system_step"] > 0]
        best = min(ok, key=lambda r: r["us_per_system_step"])
        assert (t["threads"], t["pair_lanes"]) == (best["threads"], best["pair_lanes"])
    world.restore(); world.relax(200, 1e-4, conv_mode=1)
    _, E_tun = world.eval()
    # launch shape changes only the summation order of the pair sums
    assert np.allclose(E_tun[:, 3], E_def[:, 3], rtol=1e-4, atol=1e-4)
    # persistence round trip
    for c in range(6):
        world.lib.mmff_set_tuning(c, -1, 1, 0, 0)
    assert world.tuning() == {}
    assert world.load_tuning(str(tmp_path / "tune.json"))
    assert world.tuning() == tuned


def test_queue_retires_and_refills_mixed_sizes(world, golden):
    """Many more systems than resident slots, sizes 20..400: every system is
    claimed exactly once per call (nsteps set for all) and converged systems
    carry their converging step."""
    b = uneven(world, golden, n=3000, seed=9, lo=20, hi=400)
    world.set_graph(True)
    world.restore(); world.relax(400, 1e-4, conv_mode=1)
    st = world.state()
    assert ((st["status"] == 1) | (st["status"] == 2) | (st["status"] == -1)).all()
    assert (st["nsteps"] > 0).all() and (st["nsteps"] <= 400).all()
    assert (st["nsteps"][st["status"] == 2] == 400).all()
    world.set_graph(False)


def test_pair_lists_match_candidate_tiles(world, golden):
    """Shifted-image pair lists (Verlet lists with a 1 A skin, CTA kernels)
    against the per-step candidate tiles, on molecules of 150-400 atoms in a
    22.56 A cell with a 10 A cutoff (images of every large molecule within
    reach): the same pair-images inside the cutoff in a step (the counting
    kernels count each within-cutoff pair-image); 60 steps of damped dynamics
    without noise (no discrete decisions, atoms moving several A, so the lists
    are rebuilt) that agree to rounding; deterministic FIRE relaxations.  (FIRE
    trajectories of tiles and lists are not compared step for step: its
    velocity reset on cos(v, f) < 0 turns rounding differences into
    different paths.)"""
    import ctypes
    b = uneven(world, golden, n=48, seed=11, lo=150, hi=400)
    a, n, v = b.offsets()

    def run(on, nsteps, count):
        world.set_pair_lists(on)
        world.lib.mmff_set_counting(1 if count else 0)
        world.restore(); world.relax(nsteps, 1e-4, conv_mode=1)
        st = world.state()
        c = np.zeros(5, np.uint64)
        world.lib.mmff_get_counters(c.ctypes.data_as(ctypes.c_void_p))
        return st, c

    def dyn(on):
        world.set_pair_lists(on)
        world.restore()
        world.set_md(dt=0.05, gamma=0.5, T=0.0, seed=1)
        world.md(60)
        return world.state()

    try:
        _, c_tiles = run(False, 1, True)
        _, c_lists = run(True, 1, True)
        p0 = world.state()["pos"]
        m_tiles, m_lists = dyn(False), dyn(True)
        t_lists, _ = run(True, 400, False)
        t_again, _ = run(True, 400, False)
    finally:
        world.set_pair_lists(True)
        world.lib.mmff_set_counting(0)
    assert c_tiles[0] > 0 and c_tiles[0] == c_lists[0], (c_tiles, c_lists)
    # the workload reaches into the images: within-cutoff pair-images of the
    # shifted images at the start, a sizeable share of the count
    nimg = 0
    for s in range(b.nsys):
        p = b.pos[v[s]:v[s] + b.natoms[s]]
        for ix, iy in ((1, 0), (0, 1), (1, 1), (1, -1)):
            q = p + ix * b.lvec[s][0] + iy * b.lvec[s][1]
            nimg += 2 * int((((p[:, None] - q[None]) ** 2).sum(-1) < 100.0).sum())
    assert nimg > 0.01 * float(c_tiles[0]), (nimg, c_tiles)
    moved = np.abs(m_lists["pos"] - p0).max()
    assert moved > 1.0, moved                                          # rebuilds happened
    # systems larger than the cell start with atoms on top of their own images
    # (forces of 1e6 eV/A and more, which the fixed-point pair sums clamp per
    # contribution, so tiles and lists differ there by construction): compared
    # are the others
    fair = []
    for s in range(b.nsys):
        p = b.pos[v[s]:v[s] + b.natoms[s]]
        dmin = min(np.sqrt((((p[:, None] - (p[None] + ix * b.lvec[s][0] + iy * b.lvec[s][1])) ** 2).sum(-1)).min())
                   for ix, iy in ((1, 0), (0, 1), (1, 1), (1, -1)))
        fair.append(dmin > 1.5)
    assert sum(fair) >= 40, sum(fair)
    d = max(np.abs(m_tiles["pos"][v[s]:v[s + 1]] - m_lists["pos"][v[s]:v[s + 1]]).max()
            for s in range(b.nsys) if fair[s])
    assert d < 1e-3, d
    assert np.array_equal(t_lists["pos"], t_again["pos"])          # deterministic
