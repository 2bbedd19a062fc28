"""Learned warm-start proposal over the device world (host side of the
``mmff_mlp_*`` entry points of libMMFFmulti_lib.so).

FireCore relaxes with plain FIRE only; this module adds a small MLP that
predicts, per atom, a displacement toward the relaxed geometry from local
descriptors, trained on trajectories of the plain batched relaxer.  A learned
move is kept for a system only when it lowers that system's total energy, and
plain FIRE always finishes every system under the same convergence test.

Descriptors, network, loss and optimiser are restated in FP64 in
``oracle/mlp_oracle.py`` (the test-side checker).  Everything here runs on the
GPU through the library; there is no CPU path.
"""
from __future__ import annotations

import numpy as np

from . import _lib

NFEAT, K0, HID, NOP = 68, 80, 128, 16
_SHAPES = (("W1", (HID, K0)), ("b1", (HID,)), ("W2", (HID, HID)), ("b2", (HID,)), ("W3", (NOP, HID)), ("b3", (NOP,)))


def _check(rc, what):
    if rc < 0:
        raise RuntimeError(f"{what} failed: {_lib.load().mmff_last_error().decode()}")
    return rc


def flatten(p: dict) -> np.ndarray:
    return np.concatenate([np.asarray(p[k], np.float32).reshape(-1) for k, _ in _SHAPES]).astype(np.float32)


def unflatten(v: np.ndarray) -> dict:
    out, o = {}, 0
    for k, s in _SHAPES:
        n = int(np.prod(s))
        out[k] = np.asarray(v[o:o + n], np.float64).reshape(s)
        o += n
    return out


def init_params(seed: int = 0) -> dict:
    """He-style initial weights; padding rows/columns zero; small last layer."""
    rng = np.random.default_rng(seed)
    W1 = np.zeros((HID, K0)); W1[:, :NFEAT] = rng.normal(0, 1 / np.sqrt(NFEAT), (HID, NFEAT))
    W2 = rng.normal(0, 1 / np.sqrt(HID), (HID, HID))
    W3 = np.zeros((NOP, HID)); W3[:3] = rng.normal(0, 0.1 / np.sqrt(HID), (3, HID))
    return dict(W1=W1, b1=np.zeros(HID), W2=W2, b2=np.zeros(HID), W3=W3, b3=np.zeros(NOP))


class Proposal:
    """The network and its training set, resident on the world's GPU."""

    def __init__(self):
        self.lib = _lib.load()
        self.mean = self.std = None
        self.out_scale = 1.0

    # ------------------------------------------------------------ parameters
    def set_params(self, p: dict, mean, std, out_scale: float):
        self.mean = np.ascontiguousarray(mean, np.float32)
        self.std = np.ascontiguousarray(np.maximum(std, 1e-6), np.float32)
        self.out_scale = float(out_scale)
        flat = flatten(p)
        _check(self.lib.mmff_mlp_set_params(_lib.ptr(flat), _lib.ptr(self.mean), _lib.ptr(self.std), self.out_scale),
               "mmff_mlp_set_params")

    def params(self) -> dict:
        flat = np.zeros(sum(int(np.prod(s)) for _, s in _SHAPES), np.float32)
        _check(self.lib.mmff_mlp_get_params(_lib.ptr(flat)), "mmff_mlp_get_params")
        return unflatten(flat)

    # ------------------------------------------------------------ network
    def grad(self, feat, target):
        """(loss, gradient dict) of one batch, in network units."""
        F = np.ascontiguousarray(feat, np.float32); T = np.ascontiguousarray(target, np.float32)
        g = np.zeros(flatten(init_params()).shape, np.float32)
        loss = np.zeros(1)
        _check(self.lib.mmff_mlp_grad(F.shape[0], _lib.ptr(F), _lib.ptr(T), _lib.ptr(g), _lib.ptr(loss)), "mmff_mlp_grad")
        return float(loss[0]), unflatten(g)

    def adamw(self, g: dict | None, lr=1e-3, wd=0.01):
        flat = None if g is None else flatten(g)
        _check(self.lib.mmff_mlp_adamw(_lib.ptr(flat), lr, wd), "mmff_mlp_adamw")

    def infer(self, feat) -> np.ndarray:
        F = np.ascontiguousarray(feat, np.float32)
        out = np.zeros((F.shape[0], 3), np.float32)
        _check(self.lib.mmff_mlp_infer(F.shape[0], _lib.ptr(F), _lib.ptr(out)), "mmff_mlp_infer")
        return out

    def set_data(self, feat, target):
        F = np.ascontiguousarray(feat, np.float32); T = np.ascontiguousarray(target, np.float32)
        _check(self.lib.mmff_mlp_set_data(F.shape[0], _lib.ptr(F), _lib.ptr(T)), "mmff_mlp_set_data")

    def train(self, nsteps: int, batch_tiles: int = 512, lr=1e-3, wd=0.01) -> np.ndarray:
        """AdamW steps over the training set (batch_tiles x 128 atoms per step)."""
        losses = np.zeros(nsteps)
        _check(self.lib.mmff_mlp_train(nsteps, batch_tiles, lr, wd, _lib.ptr(losses)), "mmff_mlp_train")
        return losses

    # ------------------------------------------------------------ world
    def set_elements(self, elements):
        e = np.ascontiguousarray(elements, np.int32)
        _check(self.lib.mmff_mlp_set_elements(_lib.ptr(e)), "mmff_mlp_set_elements")

    def features(self, natoms_total: int, z_top: float = 0.0) -> np.ndarray:
        out = np.zeros((natoms_total, NFEAT), np.float32)
        _check(self.lib.mmff_mlp_features(z_top, _lib.ptr(out)), "mmff_mlp_features")
        return out

    def set_projection(self, mode: int):
        """0: warm-start moves are the per-atom displacements; 1: their rigid-body
        projection per system (one translation + rotation per molecule)."""
        _check(self.lib.mmff_mlp_set_projection(int(mode)), "mmff_mlp_set_projection")

    def project(self, disp) -> np.ndarray:
        """Rigid-body projection [sum natoms, 3] of displacements at the current positions."""
        d = np.ascontiguousarray(disp, np.float64)
        out = np.zeros_like(d)
        _check(self.lib.mmff_mlp_project(_lib.ptr(d), _lib.ptr(out)), "mmff_mlp_project")
        return out

    def warmstart(self, nsys: int, nsteps: int = 2, z_top: float = 0.0) -> np.ndarray:
        acc = np.zeros(nsys, np.int32)
        _check(self.lib.mmff_mlp_warmstart(nsteps, z_top, _lib.ptr(acc)), "mmff_mlp_warmstart")
        return acc


def atom_rows(batch, pos_vecs):
    """Atom rows [sum natoms, 3] of a per-vector array [sum nvecs, 3]."""
    a, _, v = batch.offsets()
    return np.concatenate([pos_vecs[v[s]:v[s] + batch.natoms[s]] for s in range(batch.nsys)])


def rigid_part(p0, p1, natoms):
    """Per system, the rigid-body move (Kabsch: rotation about the centroid and
    translation) that best maps positions p0 onto p1, as per-atom
    displacements [sum natoms, 3]: the part of a relaxation a rigid
    warm-start move can make."""
    out = np.zeros_like(p0, dtype=np.float64)
    o = 0
    for n in natoms:
        a = np.asarray(p0[o:o + n], np.float64); b = np.asarray(p1[o:o + n], np.float64)
        ca, cb = a.mean(0), b.mean(0)
        U, _, Vt = np.linalg.svd((a - ca).T @ (b - cb))
        d = np.sign(np.linalg.det(Vt.T @ U.T))
        R = Vt.T @ np.diag([1.0, 1.0, d]) @ U.T
        out[o:o + n] = (a - ca) @ R.T + cb - a
        o += n
    return out


def trajectory_dataset(world, prop: Proposal, batch, snapshots=(0, 25, 100), nstep_max=4000, Fconv=1e-4,
                       z_top: float = 0.0, target: str = "full"):
    """(features, targets) pairs from the plain batched relaxer: descriptors at
    the given FIRE step counts and, as targets, the displacement from there to
    the relaxed geometry (target="full"), or only its rigid-body part per
    molecule (target="rigid": what a rigid warm-start move can use, without
    the conformational changes no local descriptor predicts); only systems
    that converge contribute.  ``world`` holds ``batch`` (uploaded, FIRE
    parameters set)."""
    prop.set_elements(batch.elements)
    NA = int(batch.natoms.sum())
    feats, poss = [], []
    done = 0
    for s in sorted(snapshots):
        if s > done:
            world.relax(s - done, Fconv, conv_mode=1)
            done = s
        feats.append(prop.features(NA, z_top))
        poss.append(atom_rows(batch, world.state()["pos"]))
    world.relax(nstep_max - done, Fconv, conv_mode=1)
    st = world.state()
    final = atom_rows(batch, st["pos"])
    conv_atom = np.repeat(st["status"] == 1, batch.natoms)
    F = np.concatenate([f[conv_atom] for f in feats])
    if target == "rigid":
        T = np.concatenate([rigid_part(p, final, batch.natoms)[conv_atom] for p in poss])
    else:
        T = np.concatenate([(final - p)[conv_atom] for p in poss])
    return F, T
