"""Learned warm-start proposal on the GPU against the FP64 oracle
(oracle/mlp_oracle.py): tensor-core forward and backward, AdamW, descriptors,
training, and the energy gate of the warm start."""
import numpy as np
import pytest

from conftest import batch_from_golden, grid_from_golden
from firecore_b200 import learned as L
from firecore_b200 import systems as S
from firecore_b200.world import DEFAULT_FLAGS, FireParams, World
from oracle import mlp_oracle as M
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def world():
    return World(0)


def setup_net(seed, n):
    """float32-exact parameters, raw features and targets; the oracle's
    standardised bf16 input computed in float32 exactly as the device does."""
    rng = np.random.default_rng(seed)
    p = L.init_params(seed)
    p["W3"][:3] *= 20.0
    p["b1"] = rng.normal(0, 0.2, 128); p["b2"] = rng.normal(0, 0.2, 128); p["b3"][:3] = rng.normal(0, 0.1, 3)
    p = {k: v.astype(np.float32).astype(np.float64) for k, v in p.items()}
    F = (rng.normal(size=(n, M.NFEAT)) * rng.uniform(0.1, 3.0, M.NFEAT) + rng.normal(size=M.NFEAT)).astype(np.float32)
    mean = F.mean(0).astype(np.float32); std = F.std(0).astype(np.float32)
    T = rng.normal(0, 0.3, (n, 3)).astype(np.float32)
    istd = (np.float32(1.0) / std).astype(np.float32)
    Xo = np.zeros((n, M.K0)); Xo[:, :M.NFEAT] = ((F - mean) * istd).astype(np.float32)
    return p, F, mean, std, T, M.bf16(Xo)


def relerr(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)


@pytest.mark.parametrize("n", [128, 1000, 20000])
def test_gradients_vs_oracle(world, n):
    """Gradient sums of every parameter tensor from the tcgen05 backward pass
    match the oracle (bf16 rounding at the same places) to 1e-2 relative norm;
    the loss to 1e-3.  n = 1000 leaves a ragged last tile."""
    p, F, mean, std, T, Xo = setup_net(n, n)
    s = 0.5
    prop = L.Proposal()
    prop.set_params(p, mean, std, s)
    loss, g = prop.grad(F, T)
    Tn = (T / np.float32(s)).astype(np.float32).astype(np.float64)
    lo, go = M.loss_and_grads(Xo, Tn, p, bf=True)
    assert abs(loss - lo) <= 1e-3 * lo, (loss, lo)
    for k in ("W1", "b1", "W2", "b2", "W3", "b3"):
        assert relerr(g[k], go[k]) < 1e-2, (k, relerr(g[k], go[k]))
    assert (g["W1"][:, M.NFEAT:] == 0).all() and (g["W3"][3:] == 0).all()


def test_forward_vs_oracle(world):
    p, F, mean, std, T, Xo = setup_net(5, 777)
    s = 0.25
    prop = L.Proposal()
    prop.set_params(p, mean, std, s)
    y = prop.infer(F)
    yo = M.forward(Xo, p, bf=True)[0][:, :3] * s
    # FP32 vs FP64 pre-activations can round a hidden activation to the
    # neighbouring bf16 value (2^-8 relative): rare outliers, bounded
    err = np.abs(y - yo) / np.abs(yo).max()
    assert np.quantile(err, 0.99) <= 1e-5 and err.max() <= 5e-3, (np.quantile(err, 0.99), err.max())


def test_adamw_vs_oracle(world):
    p, F, mean, std, T, Xo = setup_net(7, 256)
    prop = L.Proposal()
    prop.set_params(p, mean, std, 1.0)
    rng = np.random.default_rng(1)
    m = {k: np.zeros_like(v) for k, v in p.items()}
    v = {k: np.zeros_like(x) for k, x in p.items()}
    q = {k: x.copy() for k, x in p.items()}
    for t in (1, 2, 3):
        g = {k: rng.normal(0, 1e-2, x.shape).astype(np.float32).astype(np.float64) for k, x in p.items()}
        g["W1"][:, M.NFEAT:] = 0; g["W3"][3:] = 0; g["b3"][3:] = 0
        prop.adamw(g, lr=1e-3, wd=0.01)
        q = M.adamw(q, g, m, v, t, lr=1e-3, wd=0.01)
    got = prop.params()
    for k in q:
        assert np.abs(got[k] - q[k]).max() <= 2e-6, (k, np.abs(got[k] - q[k]).max())


def test_training_reduces_loss(world):
    """Device training (tcgen05 forward/backward + AdamW) fits a smooth target
    of the inputs: loss falls at least 10x in 400 steps."""
    rng = np.random.default_rng(11)
    n = 8192
    F = rng.normal(size=(n, M.NFEAT)).astype(np.float32)
    T = (0.3 * np.tanh(F[:, 65:68]) + 0.1 * F[:, 0:3] * F[:, 3:6]).astype(np.float32)
    prop = L.Proposal()
    prop.set_params(L.init_params(3), F.mean(0), F.std(0), float(T.std()))
    prop.set_data(F, T)
    losses = prop.train(400, batch_tiles=16, lr=3e-3, wd=0.0)
    assert np.isfinite(losses).all()
    assert losses[-20:].mean() < 0.1 * losses[:5].mean(), (losses[:5], losses[-20:])


def test_descriptors_vs_oracle(world, golden):
    """Descriptors of the device world against the oracle's FP64 restatement
    (radial bins and height to 1e-4; the FP32 GridFF force to 1e-3 relative)."""
    grid = grid_from_golden(golden)
    b = batch_from_golden(golden, "A")
    world.set_params(flags=DEFAULT_FLAGS)
    world.grid_upload(golden["C"], grid)
    world.upload(b)
    prop = L.Proposal()
    prop.set_elements(b.elements)
    NA = int(b.natoms.sum())
    f = prop.features(NA, z_top=0.0)
    pos = L.atom_rows(b, world.state()["pos"])
    P = O.make_params(grid)
    PLQ = O.req2plq(b.REQs)
    fg = O.grid_sample(pos, PLQ, golden["C"], P)[:, :3]
    fo = M.descriptors(pos, b.elements, b.natoms, b.lvec, (1, 1, 0), 0.0, fg)
    assert np.abs(f[:, :65] - fo[:, :65]).max() < 1e-4, np.abs(f[:, :65] - fo[:, :65]).max()
    assert np.abs(f[:, 65:] - fo[:, 65:]).max() <= 1e-3 * np.abs(fo[:, 65:]).max() + 1e-5
    assert (f[:, :64].sum(1) > 0).all()        # every atom has neighbours within 5 A


def test_warmstart_never_raises_energy(world, golden):
    """Energy gate: after learned moves (untrained network, large outputs)
    no system's total energy is above its starting energy, and every
    rejected move left the system where it was."""
    grid = grid_from_golden(golden)
    b = S.make_systems([24] * 8 + [40] * 8, seed=3, topo_mode=1, sigma=0.1, cell=(11.28, 11.28, 40.0))
    world.set_params(flags=DEFAULT_FLAGS)
    world.grid_upload(golden["C"], grid)
    world.upload(b)
    _, E0 = world.eval()
    pos0 = world.state()["pos"]
    prop = L.Proposal()
    p = L.init_params(4)
    p["W3"][:3] *= 5.0
    prop.set_params(p, np.zeros(M.NFEAT), np.ones(M.NFEAT), 0.05)
    prop.set_elements(b.elements)
    acc = prop.warmstart(b.nsys, nsteps=2)
    _, E1 = world.eval()
    pos1 = world.state()["pos"]
    assert ((acc >= 0) & (acc <= 2)).all()
    assert (E1[:, 3] <= E0[:, 3] + 1e-9 * np.abs(E0[:, 3])).all()
    a, _, v = b.offsets()
    for s in np.where(acc == 0)[0]:
        assert np.abs(pos1[v[s]:v[s + 1]] - pos0[v[s]:v[s + 1]]).max() < 1e-5


def test_trained_proposal_gain_over_plain_fire(world, golden):
    """What the learned part adds, measured on held-out molecules: a network
    trained on the plain relaxer's trajectories (descriptors at FIRE steps 0,
    10, 50 -> displacement to the relaxed geometry) makes energy-gated moves
    that lower the energy, never raise it, and the relaxation that follows
    reaches the same minima as plain FIRE.  The step counts with and without
    the warm start are printed (the gain is small: see the learned bench)."""
    import math
    grid = grid_from_golden(golden)
    world.set_params(flags=DEFAULT_FLAGS)
    world.set_fire(FireParams(Flim=10.0))
    world.grid_upload(golden["C"], grid)
    train = S.make_systems([24] * 256, seed=21, topo_mode=1, sigma=0.15, cell=(11.28, 11.28, 40.0))
    world.upload(train)
    prop = L.Proposal()
    F, T = L.trajectory_dataset(world, prop, train, snapshots=(0, 10, 50), nstep_max=1500)
    assert len(F) > 500
    prop.set_params(L.init_params(0), F.mean(0), F.std(0) + 1e-6, float(math.sqrt((T ** 2).mean())))
    prop.set_data(F, T)
    losses = prop.train(300, batch_tiles=16, lr=1e-3, wd=0.0)
    assert losses[-10:].mean() < losses[:3].mean()
    test = S.make_systems([24] * 128, seed=22, topo_mode=1, sigma=0.15, cell=(11.28, 11.28, 40.0))
    world.upload(test)
    prop.set_elements(test.elements)
    # plain FIRE
    world.restore(); world.relax(3000, 1e-4, conv_mode=1)
    sp = world.state(); _, Ep = world.eval()
    # learned warm start, then the same FIRE
    world.restore()
    _, E0 = world.eval()
    acc = prop.warmstart(test.nsys, nsteps=2)
    _, E1 = world.eval()
    assert (E1[:, 3] <= E0[:, 3] + 1e-9 * np.abs(E0[:, 3])).all()
    assert acc.sum() > 0 and (E0[:, 3] - E1[:, 3]).sum() > 0
    world.relax(3000, 1e-4, conv_mode=1)
    sl = world.state(); _, El = world.eval()
    both = (sp["status"] == 1) & (sl["status"] == 1)
    dE = np.abs(El[both, 3] - Ep[both, 3]) / test.natoms[both]
    print(f"held-out: {int(acc.sum())} learned moves kept; converged plain {int((sp['status'] == 1).sum())}, "
          f"learned {int((sl['status'] == 1).sum())}; median steps plain {np.median(sp['nsteps'][sp['status'] == 1])}, "
          f"learned {np.median(sl['nsteps'][sl['status'] == 1])}; same minimum for "
          f"{int((dE <= 1e-5).sum())} of {int(both.sum())}")
    assert np.median(dE) <= 1e-5


def test_rigid_projection_vs_oracle(world, golden):
    """The rigid-body projection of warm-start moves (rigid_kernel) against its
    FP64 restatement, and the move it makes keeps every bond length."""
    grid = grid_from_golden(golden)
    b = S.make_systems([24, 57, 130, 260], seed=8, topo_mode=1, sigma=0.1, cell=(22.56, 22.56, 40.0))
    world.set_params(flags=DEFAULT_FLAGS)
    world.grid_upload(golden["C"], grid)
    world.upload(b)
    prop = L.Proposal()
    pos = L.atom_rows(b, world.state()["pos"])
    rng = np.random.default_rng(1)
    disp = rng.normal(0, 0.2, pos.shape) + np.array([0.3, -0.1, -0.5])
    out = prop.project(disp)
    ref = M.rigid_projection(pos, disp, b.natoms)
    assert np.abs(out - ref).max() <= 2e-5 * np.abs(ref).max(), np.abs(out - ref).max()
    # a rigid move: distances inside each molecule unchanged
    moved = pos + ref
    o = 0
    for n in b.natoms:
        d0 = np.linalg.norm(pos[o:o + n, None] - pos[None, o:o + n], axis=2)
        d1 = np.linalg.norm(moved[o:o + n, None] - moved[None, o:o + n], axis=2)
        assert np.abs(d1 - d0).max() < 1e-9
        o += n


def test_tensor_core_wait_timeout_reports_and_recovers(world):
    """A completion wait of the tcgen05 kernel that nothing completes (a
    launch that issues no product and no commit) runs out after its short
    limit: the kernel returns the error status, frees its TMEM, and the next
    inference on the same context gives the same outputs as before."""
    p, F, mean, std, T, X = setup_net(5, 300)
    prop = L.Proposal()
    prop.set_params(p, mean, std, 1.0)
    before = prop.infer(F)
    assert prop.lib.mmff_kernel_launches() >= 0
    assert prop.lib.mmff_mlp_wait_test() == 1
    after = prop.infer(F)
    assert np.array_equal(before, after)
