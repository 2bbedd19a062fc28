"""Generate the golden fixtures by running FireCore's own C++ physics.

Run in a container where the reference tree is present (it builds
oracle/_ref/libref_harness.so from the reference sources with oracle/Makefile):

    python tests/golden/make_golden.py

Writes tests/golden/mmff_small.npz: small seeded inputs (molecules, slab grid)
and the reference's outputs for them:
  * per system, one force evaluation (MMFFsp3_loc::eval_atom +
    NBFF::evalLJQs_ng4_PBC_atom_omp + GridFF::addAtom(BsplineDouble) +
    MMFFsp3_loc::assemble_atom), for three switch settings;
  * 200 FIRE steps and a full relaxation through MolWorld_sp3::run_no_omp;
  * B-spline samples (GridFF::getForce_Bspline), REQ->PLQ (REQ2PLQ_d),
    grid-node potentials (GridFF::evalGridFFPoint_Mors/_Coul) and a
    Bspline::fit3D_omp fit of a small grid;
  * the back-neighbour tables MMFFsp3_loc::makeBackNeighs builds.
The B-spline coefficients fed to the reference are the FP64 oracle's exact fit
of the oracle's node potentials; both are checked here too.
"""
import ctypes
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from firecore_b200 import systems as S  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "mmff_small.npz")


def p(a):
    return ctypes.c_void_p(a.ctypes.data)


def small_substrate():
    return S.make_slab(ncell=2, grid_step=0.4, nz=40, nPBC_coul=(4, 4, 0))


def main():
    O.build_oracle(with_ref=True)
    ref = O.ref()
    sub = small_substrate()
    V = O.grid_potentials(sub)
    C = O.bspline_fit(V)
    g = sub.grid
    b = S.make_systems([24] * 4, seed=7, topo_mode=0, sigma=0.1, rotate=False, hbond=True,
                       cell=(sub.lvec[0, 0], sub.lvec[1, 1], 40.0))
    b2 = S.make_systems([30, 41], seed=11, topo_mode=1, sigma=0.1, rotate=True, hbond=False,
                        cell=(sub.lvec[0, 0], sub.lvec[1, 1], 40.0))
    out = dict(grid_n=np.array(g.n), grid_pos0=np.array(g.pos0), grid_step=np.array(g.step), V=V, C=C,
               spos=sub.spos, sREQ=sub.sREQ, slvec=sub.lvec)
    npbc = np.array([1, 1, 0], np.int32)
    gn = np.array(g.n, np.int32); gp0 = np.array(g.pos0); gst = np.array(g.step)
    fire0 = [0.1, 0.1, 0.0, 0.1, 0.01, 0.1, 1.1, 0.5, 0.8, 3, 0.0]
    flag_sets = {"full": O.DEFAULT_FLAGS, "nogrid": O.DEFAULT_FLAGS & ~O.GRID,
                 "nopbc": O.DEFAULT_FLAGS & ~O.PBC & ~O.GRID}
    for tag, batch in (("A", b), ("B", b2)):
        a_off, n_off, v_off = batch.offsets()
        for k, v in batch.__dict__.items():
            out[f"{tag}_{k}"] = v
        for fname, flags in flag_sets.items():
            F = np.zeros_like(batch.pos); E = np.zeros((batch.nsys, 4))
            for s in range(batch.nsys):
                na, nn = int(batch.natoms[s]), int(batch.nnode[s])
                pos = np.ascontiguousarray(batch.pos[v_off[s]:v_off[s + 1]])
                arr = [np.ascontiguousarray(x[a_off[s]:a_off[s + 1]]) for x in (batch.neighs, batch.neighCell, batch.REQs)]
                nar = [np.ascontiguousarray(x[n_off[s]:n_off[s + 1]]) for x in (batch.apars, batch.bLs, batch.bKs, batch.Ksp, batch.Kpp)]
                lv = np.ascontiguousarray(batch.lvec[s].reshape(9))
                bk = np.zeros((na, 4), np.int32); ng = np.zeros((na, 4), np.int32)
                ref.ref_setup(na, nn, p(pos), p(arr[0]), p(arr[1]), p(arr[2]), *[p(x) for x in nar], p(lv), p(npbc),
                              flags, 1.5, p(gn), p(gp0), p(gst), p(C), p(bk), p(ng))
                if fname == "full":
                    assert np.array_equal(bk, batch.bkneighs[a_off[s]:a_off[s + 1]]), "bkneighs differ"
                    assert np.array_equal(ng, batch.neighs[a_off[s]:a_off[s + 1]]), "cap neighs differ"
                f = np.zeros((na + nn, 3)); e = np.zeros(4)
                ref.ref_eval(p(f), p(e))
                F[v_off[s]:v_off[s + 1]] = f; E[s] = e
                if fname == "full":
                    # 200 FIRE steps, then a full relaxation from the start
                    for tagr, nit in (("r200", 200), ("rfull", 3000)):
                        pr = pos.copy(); vr = np.zeros_like(pr); fr = np.array(fire0)
                        oE = np.zeros(nit); oF = np.zeros(nit)
                        ref.ref_setup(na, nn, p(pos), p(arr[0]), p(arr[1]), p(arr[2]), *[p(x) for x in nar], p(lv),
                                      p(npbc), flags, 1.5, p(gn), p(gp0), p(gst), p(C), p(bk), p(ng))
                        it = ref.ref_relax(nit, 1e-4, p(pr), p(vr), p(fr), p(oE), p(oF))
                        out.setdefault(f"{tag}_{tagr}_pos", np.zeros_like(batch.pos))[v_off[s]:v_off[s + 1]] = pr
                        out.setdefault(f"{tag}_{tagr}_vel", np.zeros_like(batch.pos))[v_off[s]:v_off[s + 1]] = vr
                        out.setdefault(f"{tag}_{tagr}_fire", np.zeros((batch.nsys, 3)))[s] = fr[:3]
                        out.setdefault(f"{tag}_{tagr}_nsteps", np.zeros(batch.nsys, np.int32))[s] = it
                        out.setdefault(f"{tag}_{tagr}_Fend", np.zeros(batch.nsys))[s] = oF[min(it, nit - 1)]
            out[f"{tag}_{fname}_F"] = F
            out[f"{tag}_{fname}_E"] = E
    # grid samples inside the band, with random PLQ
    rng = np.random.default_rng(5)
    L = sub.lvec[0, 0]
    pts = np.stack([rng.uniform(-0.3 * L, 1.3 * L, 64), rng.uniform(-0.3 * L, 1.3 * L, 64),
                    rng.uniform(g.pos0[2] + 1.5, g.pos0[2] + g.step[2] * (g.n[2] - 6), 64)], 1)
    REQ = np.stack([rng.uniform(1.5, 2.0, 64), np.sqrt(rng.uniform(0.002, 0.01, 64)), rng.normal(0, 0.3, 64),
                    np.zeros(64)], 1)
    PLQ = np.zeros_like(REQ)
    REQ = np.ascontiguousarray(REQ); pts = np.ascontiguousarray(pts)
    ref.ref_req2plq(64, p(REQ), ctypes.c_double(1.5), p(PLQ))
    fe = np.zeros((64, 4))
    ref.ref_grid_sample(64, p(pts), p(PLQ), p(fe))
    out.update(samp_pos=pts, samp_REQ=REQ, samp_PLQ=PLQ, samp_fe=fe)
    # grid-node potentials at a few nodes
    idx = rng.integers(0, [g.n[0], g.n[1], g.n[2]], size=(16, 3))
    pts2 = np.stack([g.pos0[k] + g.step[k] * idx[:, k] for k in range(3)], 1)
    Vp = np.zeros((16, 3))
    # arrays held in names for the duration of each native call
    pts2 = np.ascontiguousarray(pts2); sp = np.ascontiguousarray(sub.spos); sq = np.ascontiguousarray(sub.sREQ)
    lv = np.ascontiguousarray(sub.lvec.reshape(9))
    nm = np.array(sub.nPBC_mors, np.int32); nc = np.array(sub.nPBC_coul, np.int32)
    ref.ref_grid_points(16, p(pts2), sub.spos.shape[0], p(sp), p(sq), p(lv), p(nm), p(nc), ctypes.c_double(1.5), p(Vp))
    out.update(node_idx=idx, node_V=Vp)
    # Bspline::fit3D_omp on a small smooth periodic-in-xy grid (x-fastest order)
    nsx, nsy, nsz = 8, 10, 12
    xs = np.arange(nsx)[None, None, :] / nsx; ys = np.arange(nsy)[None, :, None] / nsy
    zs = np.arange(nsz)[:, None, None] / nsz
    Ef = np.cos(2 * np.pi * xs) * np.sin(2 * np.pi * ys) * np.exp(-2 * zs) + 0.3 * np.cos(4 * np.pi * (xs + ys)) * zs
    Ef = np.ascontiguousarray(Ef + 0 * zs)
    Gf = np.zeros_like(Ef)
    ns = np.array([nsx, nsy, nsz], np.int32)
    nit = ref.ref_fit3d(p(ns), p(Ef), p(Gf), ctypes.c_double(1e-13), 200000,
                        ctypes.c_double(0.3))
    out.update(fit_E=Ef, fit_G=Gf, fit_niter=np.array(nit))
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
