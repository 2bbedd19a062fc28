"""Host-side checks of the learned-proposal network (no GPU):

* every tcgen05.mma of the network kernel, replayed on the CPU: the shared-
  memory and instruction descriptors the library encodes are decoded with the
  canonical SWIZZLE_NONE layouts (K-major: 8 rows x 16 B core matrices, rows
  at stride byte offset, k groups at leading byte offset; MN-major: the
  transpose), read from a packed image of known matrices, and must give the
  product the kernel relies on, with every byte inside its own buffer;
* the FP64 oracle's gradients against central finite differences;
* the oracle's AdamW and bf16 rounding."""
import ctypes

import numpy as np
import pytest

from firecore_b200 import _lib
from oracle import mlp_oracle as M

TILE, K0, HID, NOP = 128, 80, 128, 16


def cm_off(r, k, K):
    return (r // 8) * (K * 16) + (k // 8) * 128 + (r % 8) * 16 + (k % 8) * 2


def pack(mat, img, off):
    R, K = mat.shape
    for r in range(R):
        for k in range(K):
            img[(off + cm_off(r, k, K)) // 2] = mat[r, k]


def read_operand(img, desc, rows, mn_major, region):
    """rows x 16 operand of one MMA k-step, read through a matrix descriptor."""
    start = (desc & 0x3FFF) << 4
    lbo = ((desc >> 16) & 0x3FFF) << 4
    sbo = ((desc >> 32) & 0x3FFF) << 4
    assert (desc >> 46) & 3 == 1, "descriptor version must be 1"
    assert (desc >> 61) == 0 and ((desc >> 49) & 7) == 0, "SWIZZLE_NONE, base offset 0"
    out = np.zeros((rows, 16))
    for m in range(rows):
        for k in range(16):
            if mn_major:
                a = start + (m % 8) * 2 + (m // 8) * sbo + (k % 8) * 16 + (k // 8) * lbo
            else:
                a = start + (m % 8) * 16 + (m // 8) * sbo + (k % 8) * 2 + (k // 8) * lbo
            assert region[0] <= a < region[1], (hex(a), region)
            out[m, k] = img[a // 2]
    return out


def test_mma_plan_replay():
    lib = _lib.load()
    lay = np.zeros(16, np.int32)
    lib.mmff_mlp_layout(_lib.ptr(lay))
    sm_total = int(lay[7])
    assert sm_total + 1024 <= 232448, "fits the 227 KB opt-in shared memory of one CTA"
    rng = np.random.default_rng(3)
    ri = lambda *s: rng.integers(-3, 4, s).astype(np.float64)     # exact in bf16 and in the sums
    mats = dict(W1=ri(HID, K0), W2=ri(HID, HID), W3=ri(NOP, HID), ONE=np.ones((NOP, TILE)), X=ri(TILE, K0),
                H1=ri(TILE, HID), H2=ri(TILE, HID), S2=ri(TILE, HID), DY=ri(TILE, NOP))
    offs = dict(W1=0, W2=HID * K0 * 2, W3=HID * K0 * 2 + HID * HID * 2)
    offs["ONE"] = offs["W3"] + NOP * HID * 2
    offs["X"] = offs["ONE"] + NOP * TILE * 2
    offs["H1"] = offs["X"] + TILE * K0 * 2
    offs["H2"] = offs["H1"] + TILE * HID * 2
    offs["S2"] = offs["H2"] + TILE * HID * 2
    offs["DY"] = offs["S2"] + TILE * HID * 2
    assert offs["X"] == lay[13] and offs["DY"] == lay[14]
    img = np.zeros(sm_total // 2)
    regions = {}
    for k, m in mats.items():
        pack(m, img, offs[k])
        regions[offs[k]] = (offs[k], offs[k] + m.size * 2)
    ops = np.zeros(14 * 16, np.int32)
    nop = lib.mmff_mlp_plan(_lib.ptr(ops))
    assert nop == 10
    ops = ops[:14 * nop].reshape(nop, 14)
    X, W1, W2, W3, ONE = mats["X"], mats["W1"], mats["W2"], mats["W3"], mats["ONE"]
    H1, H2, S2, DY = mats["H1"], mats["H2"], mats["S2"], mats["DY"]
    expect = [X @ W1.T, H1 @ W2.T, H2 @ W3.T, H2.T @ DY, DY @ W3, S2.T @ H1, S2.T @ ONE.T, S2 @ W2, H2.T @ X,
              H2.T @ ONE.T]
    cols = []
    for i, o in enumerate(ops):
        dcol, N, nk, acc, a_off, a_lbo, a_sbo, a_step, a_mn, b_off, b_lbo, b_sbo, b_step, b_mn = (int(x) for x in o)
        idesc = lib.mmff_mlp_instr_desc(N, a_mn, b_mn)
        assert (idesc >> 4) & 3 == 1 and (idesc >> 7) & 7 == 1 and (idesc >> 10) & 7 == 1   # F32 <- BF16 x BF16
        assert ((idesc >> 17) & 0x3F) * 8 == N and ((idesc >> 24) & 0x1F) * 16 == 128
        assert ((idesc >> 15) & 1) == a_mn and ((idesc >> 16) & 1) == b_mn
        assert N % 16 == 0 and 16 <= N <= 256
        D = np.zeros((128, N))
        for k in range(nk):
            da = lib.mmff_mlp_smem_desc(a_off + k * a_step, a_lbo, a_sbo)
            db = lib.mmff_mlp_smem_desc(b_off + k * b_step, b_lbo, b_sbo)
            A = read_operand(img, da, 128, a_mn, regions[a_off])
            B = read_operand(img, db, N, b_mn, regions[b_off])
            D += A @ B.T
        assert np.array_equal(D, expect[i]), f"product {i}"
        cols.append((dcol, dcol + N, acc))
    # accumulators (acc) never share TMEM columns with anything else
    for i, (a0, a1, acc) in enumerate(cols):
        assert 0 <= a0 < a1 <= 512
        for j, (b0, b1, accj) in enumerate(cols):
            if i != j and (acc or accj):
                assert a1 <= b0 or b1 <= a0, (i, j)


def test_oracle_gradients_finite_difference():
    rng = np.random.default_rng(0)
    p = M.init_params(1)
    p["W3"][:3] *= 30.0
    X = np.zeros((40, M.K0)); X[:, :M.NFEAT] = rng.normal(size=(40, M.NFEAT))
    T = rng.normal(size=(40, 3))
    L, g = M.loss_and_grads(X, T, p)
    h = 1e-6
    for key, idx in [("W1", (5, 7)), ("b1", (3,)), ("W2", (10, 100)), ("b2", (77,)), ("W3", (1, 50)), ("b3", (2,))]:
        q = {k: v.copy() for k, v in p.items()}
        q[key][idx] += h
        Lp, _ = M.loss_and_grads(X, T, q)
        q[key][idx] -= 2 * h
        Lm, _ = M.loss_and_grads(X, T, q)
        fd = (Lp - Lm) / (2 * h)
        assert abs(fd - g[key][idx]) <= 1e-6 * max(1.0, abs(fd)), (key, fd, g[key][idx])


def test_oracle_adamw_and_bf16():
    assert M.bf16(np.array([1.0 + 2 ** -9]))[0] == 1.0            # ties to even
    assert M.bf16(np.array([1.0 + 3 * 2 ** -9]))[0] == 1.0 + 2 ** -7
    p = M.init_params(2)
    g = {k: np.ones_like(v) for k, v in p.items()}
    m = {k: np.zeros_like(v) for k, v in p.items()}
    v = {k: np.zeros_like(v) for k, v in p.items()}
    q = M.adamw(p, g, m, v, 1, lr=1e-3, wd=0.0)
    d = p["b1"] - q["b1"]
    assert np.allclose(d, 1e-3, rtol=1e-6)          # first step moves by lr
    assert (q["W1"][:, M.NFEAT:] == 0).all() and (q["W3"][3:] == 0).all()
