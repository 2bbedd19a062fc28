"""CPU oracle (test infrastructure only) for the learned warm-start proposal.

The learned proposal has no counterpart in FireCore: the reference relaxes
with plain FIRE only (MolWorld_sp3::run_no_omp, cpp/common/molecular/
MolWorld_sp3.h:2261-2490).  The network and its inputs are this project's
specification, restated here in FP64 numpy so that the CUDA descriptor,
forward, backward and AdamW kernels can be checked number by number:

* per-atom descriptor (68 features): for the 32 nearest neighbours within
  5 A (all periodic images of the pair-term image set, the atom itself only
  in shifted images), 16 Gaussian radial bins (centres k/3 A, k = 0..15,
  sigma 0.3 A) per element channel (H, C, N, O); the height above the slab
  top; the GridFF force on the atom (B-spline sample with the atom's PLQ);
* network 68 -> 128 -> 128 -> 3 with SiLU, inputs standardised by stored
  mean/std and zero-padded to 80 columns, outputs padded to 16 rows (rows
  3..15 of W3 and b3 stay zero); loss = sum over atoms and the 3 components
  of (y - t)^2 / B for a batch of B atoms;
* AdamW (decoupled weight decay on the weight matrices, not the biases).

``bf16=True`` rounds to bfloat16 exactly where the GPU kernels store bf16
(inputs, weights, the hidden activations, SiLU derivatives, output and
hidden gradients) so that the comparison isolates accumulation order.
"""
from __future__ import annotations

import numpy as np

NBIN, NCH, NNB = 16, 4, 32
RCUT_D, SIGMA_D = 5.0, 0.3
MU = np.arange(NBIN) * (RCUT_D / (NBIN - 1))
NFEAT, K0, HID, NOUT, NOUT_PAD = 68, 80, 128, 3, 16


def bf16(x):
    """Round-to-nearest-even to bfloat16, returned as float64."""
    a = np.ascontiguousarray(x, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    out = r.view(np.float32).astype(np.float64)
    return np.where(np.isfinite(a), out, a.astype(np.float64))


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


# ------------------------------------------------------------------ descriptors

def image_shifts(lvec, npbc):
    """Shift vectors in the pair-term order (x fastest, then y, then z)."""
    out = []
    for iz in range(-npbc[2], npbc[2] + 1):
        for iy in range(-npbc[1], npbc[1] + 1):
            for ix in range(-npbc[0], npbc[0] + 1):
                out.append(lvec[0] * ix + lvec[1] * iy + lvec[2] * iz)
    return np.array(out)


def descriptors(pos, elem, natoms, lvecs, npbc, z_top, fgrid):
    """Raw (unstandardised) features [sum natoms, 68].

    pos: [sum natoms, 3] world positions; elem: channel 0..3 per atom;
    lvecs: [nsys, 3, 3]; fgrid: [sum natoms, 3] GridFF forces."""
    nsys = len(natoms)
    out = np.zeros((int(np.sum(natoms)), NFEAT))
    off = 0
    for s in range(nsys):
        n = int(natoms[s])
        P = pos[off:off + n]
        E = elem[off:off + n]
        sh = image_shifts(lvecs[s], npbc)
        for i in range(n):
            cand = []
            for k, d in enumerate(sh):
                v = P + d - P[i]
                r = np.sqrt((v * v).sum(1))
                for j in range(n):
                    if j == i and not d.any():
                        continue
                    if r[j] < RCUT_D:
                        cand.append((r[j], k, j))
            cand.sort()
            for r, _, j in cand[:NNB]:
                c = min(int(E[j]), NCH - 1)
                out[off + i, c * NBIN:(c + 1) * NBIN] += np.exp(-(r - MU) ** 2 / (2 * SIGMA_D ** 2))
            out[off + i, 64] = P[i, 2] - z_top
            out[off + i, 65:68] = fgrid[off + i]
        off += n
    return out


def standardise(F, mean, std, bf=False):
    """Standardised, zero-padded network input [B, 80]."""
    X = np.zeros((F.shape[0], K0))
    X[:, :NFEAT] = (F - mean) / std
    return bf16(X) if bf else X


# ------------------------------------------------------------------ network

def init_params(seed=0):
    rng = np.random.default_rng(seed)
    W1 = np.zeros((HID, K0)); W1[:, :NFEAT] = rng.normal(0, 1 / np.sqrt(NFEAT), (HID, NFEAT))
    W2 = rng.normal(0, 1 / np.sqrt(HID), (HID, HID))
    W3 = np.zeros((NOUT_PAD, HID)); W3[:NOUT] = rng.normal(0, 0.1 / np.sqrt(HID), (NOUT, HID))
    return dict(W1=W1, b1=np.zeros(HID), W2=W2, b2=np.zeros(HID), W3=W3, b3=np.zeros(NOUT_PAD))


def forward(X, p, bf=False):
    r = bf16 if bf else (lambda a: a)
    z1 = r(X) @ r(p["W1"]).T + p["b1"]
    h1 = r(silu(z1))
    z2 = h1 @ r(p["W2"]).T + p["b2"]
    h2 = r(silu(z2))
    y = h2 @ r(p["W3"]).T + p["b3"]
    return y, (z1, h1, z2, h2)


def loss_and_grads(X, T, p, bf=False):
    """Loss and gradients for targets T [B, 3] (normalised displacements)."""
    r = bf16 if bf else (lambda a: a)
    B = X.shape[0]
    y, (z1, h1, z2, h2) = forward(X, p, bf)
    d = y[:, :NOUT] - T
    loss = (d * d).sum() / B
    dy = np.zeros((B, NOUT_PAD)); dy[:, :NOUT] = 2.0 * d / B
    dy = r(dy)
    g = {}
    g["W3"] = dy.T @ h2
    g["b3"] = dy.sum(0)
    dz2 = r((dy @ r(p["W3"])) * r(dsilu(z2)))
    g["W2"] = dz2.T @ h1
    g["b2"] = dz2.sum(0)
    dz1 = r((dz2 @ r(p["W2"])) * r(dsilu(z1)))
    g["W1"] = dz1.T @ r(X)
    g["b1"] = dz1.sum(0)
    return loss, g


def adamw(p, g, m, v, t, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8, wd=0.01):
    """One AdamW step (t counts from 1); weight decay on W1, W2, W3 only."""
    out = {}
    for k in p:
        m[k] = b1 * m[k] + (1 - b1) * g[k]
        v[k] = b2 * v[k] + (1 - b2) * g[k] * g[k]
        mh = m[k] / (1 - b1 ** t)
        vh = v[k] / (1 - b2 ** t)
        upd = mh / (np.sqrt(vh) + eps)
        if k.startswith("W"):
            upd = upd + wd * p[k]
        out[k] = p[k] - lr * upd
    # padding rows/columns stay zero
    out["W1"][:, NFEAT:] = 0.0
    out["W3"][NOUT:] = 0.0
    out["b3"][NOUT:] = 0.0
    return out


def rigid_projection(pos, disp, natoms):
    """Rigid-body projection of per-atom displacements, per system (the warm
    start's projection, restated in FP64): t = mean d; w solves
    (sum |u|^2 1 - u u^T) w = sum u x (d - t) with u = p - centroid; the
    projected displacement is t + (R(w) - 1) u, R the rotation by |w| about w.
    pos, disp [sum natoms, 3]; natoms [nsys]."""
    out = np.zeros_like(disp, dtype=np.float64)
    o = 0
    for n in natoms:
        p = np.asarray(pos[o:o + n], np.float64)
        d = np.asarray(disp[o:o + n], np.float64)
        u = p - p.mean(0)
        t = d.mean(0)
        e = d - t
        A = np.eye(3) * (u * u).sum() - u.T @ u
        A += np.eye(3) * (1e-9 * np.trace(A) + 1e-12)
        b = np.cross(u, e).sum(0)
        w = np.linalg.solve(A, b) if np.linalg.det(A) > 0 else np.zeros(3)
        th = np.linalg.norm(w)
        R = np.eye(3)
        if th > 1e-12:
            k = w / th
            K = np.array([[0, -k[2], k[1]], [k[2], 0, -k[0]], [-k[1], k[0], 0]])
            R = np.eye(3) + np.sin(th) * K + (1 - np.cos(th)) * K @ K
        out[o:o + n] = t + u @ R.T - u
        o += n
    return out
