"""Python host side of the B200 relaxer: a thin wrapper over the C-ABI of
``libMMFFmulti_lib.so`` (``include/MMFFmulti_lib.h``).

There is no CPU fallback: every compute call goes to the CUDA kernels and
raises ``RuntimeError`` if the library or a CUDA device is missing.
"""
from __future__ import annotations

import ctypes
import json
import os
from dataclasses import dataclass

import numpy as np

from . import _lib
from .systems import GridSpec, Substrate, SystemBatch

# flag bits (include/MMFFmulti_lib.h, mmff_set_params)
BONDS, PIPI, PISIGMA, ANGLES = 1, 2, 4, 8
SUB_ANGLE_NB, SUB_BOND_NB, CLAMP_NB = 16, 32, 64
NONBONDED, GRID, PBC, SURF = 128, 256, 512, 1024
# MolWorld_sp3::run_no_omp with bNonBondNeighs (ForceField.h:170-186)
DEFAULT_FLAGS = BONDS | PIPI | PISIGMA | ANGLES | SUB_ANGLE_NB | NONBONDED | GRID | PBC

STATUS_CONVERGED, STATUS_MAXSTEPS, STATUS_NAN = 1, 2, -1


@dataclass
class FireParams:
    """FIRE parameters; defaults = DynamicOpt after setTimeSteps(0.1)
    (cpp/common/math/DynamicOpt.h:73-95,199-205).  Flim > 0 clamps each
    assembled force vector as relax_multi.cl:980-983 does."""
    dt_max: float = 0.1
    dt_min: float = 0.01
    damp_max: float = 0.1
    finc: float = 1.1
    fdec: float = 0.5
    falpha: float = 0.8
    minLastNeg: int = 3
    cv_kill: float = 0.0
    Flim: float = -1.0
    variant: int = 0       # 0: run_no_omp velocity kick; 1: Bitzek et al. 2006 mixing


def _check(rc, what):
    if rc < 0:
        raise RuntimeError(f"{what} failed: {_lib.load().mmff_last_error().decode()}")
    return rc


class World:
    """Device-resident batch of MMFF systems on one GPU."""

    def __init__(self, device: int = 0):
        self.lib = _lib.load()
        _check(self.lib.mmff_init_device(device), "mmff_init_device")
        self.batch: SystemBatch | None = None
        self.grid: GridSpec | None = None

    # ---------------------------------------------------------------- setup
    def set_params(self, flags=DEFAULT_FLAGS, npbc=(1, 1, 0), Rcut=-1.0, alphaMorse=1.5, FmaxNonBonded=10.0):
        npbc = np.ascontiguousarray(npbc, np.int32)
        _check(self.lib.mmff_set_params(flags, _lib.ptr(npbc), Rcut, alphaMorse, FmaxNonBonded), "mmff_set_params")

    def set_fire(self, F: FireParams = FireParams()):
        _check(self.lib.mmff_set_fire(F.dt_max, F.dt_min, F.damp_max, F.finc, F.fdec, F.falpha, int(F.minLastNeg),
                                      F.cv_kill, F.Flim, int(F.variant)), "mmff_set_fire")

    def set_launch(self, threads=0, pair_split=0):
        _check(self.lib.mmff_set_launch(threads, pair_split), "mmff_set_launch")

    def set_grid_cache(self, on: bool = True):
        """Per-atom GridFF stencil cache of the CTA relax kernels (bit-identical results)."""
        _check(self.lib.mmff_set_grid_cache(int(on)), "mmff_set_grid_cache")

    def set_pair_lists(self, on: bool = True, skin: float = 0.0):
        """Shifted-image pair lists in the CTA relax kernels (cutoff, 2-D cell):
        on (default) or per-step candidate tiles; skin > 0 sets their skin [A]."""
        _check(self.lib.mmff_set_pair_lists(int(bool(on)), float(skin)), "mmff_set_pair_lists")

    def set_graph(self, on: bool = True):
        """Replay mmff_relax as one captured CUDA graph per parameter set."""
        _check(self.lib.mmff_set_graph(int(on)), "mmff_set_graph")

    # ---------------------------------------------------------------- autotuner
    SIZE_CLASSES = {0: "<=32 atoms", 1: "<=64 atoms", 2: "<=64 atoms (forced CTA)", 3: "<=128 atoms",
                    4: "<=256 atoms", 5: ">256 atoms"}

    def autotune(self, nstep_probe: int = 50, max_sample: int = 1 << 20, path: str | None = None):
        """Time the candidate launch configurations of every size class present
        and keep the fastest; with ``path``, the choice is saved as JSON.
        By default every system of a class is in the probe, so the timing is of
        the machine as full as production runs fill it (a small sample would
        time per-system latency instead of throughput)."""
        rep = np.zeros((64, 6), np.float32)
        n = _check(self.lib.mmff_autotune(int(nstep_probe), int(max_sample), _lib.ptr(rep), 64), "mmff_autotune")
        rows = [dict(size_class=int(r[0]), kind="warp" if r[1] == 1 else "cta", atoms_per_lane=int(r[2]),
                     threads=int(r[3]), pair_lanes=int(r[4]), us_per_system_step=float(r[5])) for r in rep[:min(n, 64)]]
        if path:
            self.save_tuning(path, rows)
        return rows

    def tuning(self):
        out = {}
        for c in range(6):
            t = np.zeros(4, np.int32)
            _check(self.lib.mmff_get_tuning(c, _lib.ptr(t)), "mmff_get_tuning")
            if t[0] >= 0:
                out[c] = dict(kind=int(t[0]), atoms_per_lane=int(t[1]), threads=int(t[2]), pair_lanes=int(t[3]))
        return out

    def save_tuning(self, path: str, report=None):
        doc = {"tuning": {str(c): v for c, v in self.tuning().items()}, "report": report or []}
        with open(path, "w") as f:
            json.dump(doc, f, indent=1)

    def load_tuning(self, path: str) -> bool:
        if not os.path.exists(path):
            return False
        doc = json.load(open(path))
        for c, v in doc.get("tuning", {}).items():
            _check(self.lib.mmff_set_tuning(int(c), v["kind"], v["atoms_per_lane"], v["threads"], v["pair_lanes"]),
                   "mmff_set_tuning")
        return True

    def grid_upload(self, coefs: np.ndarray, grid: GridSpec):
        c = np.ascontiguousarray(coefs, np.float64)
        assert c.shape == (grid.n[0], grid.n[1], grid.n[2], 3)
        p0 = np.array(grid.pos0, np.float64); st = np.array(grid.step, np.float64)
        _check(self.lib.mmff_grid_upload(int(grid.n[0]), int(grid.n[1]), int(grid.n[2]), _lib.ptr(p0), _lib.ptr(st),
                                         _lib.ptr(c)), "mmff_grid_upload")
        self.grid = grid

    def grid_build(self, sub: Substrate, return_coefs: bool = False):
        g = sub.grid
        spos = np.ascontiguousarray(sub.spos, np.float64); sREQ = np.ascontiguousarray(sub.sREQ, np.float64)
        lv = np.ascontiguousarray(sub.lvec.reshape(9), np.float64)
        nm = np.array(sub.nPBC_mors, np.int32); nc = np.array(sub.nPBC_coul, np.int32)
        p0 = np.array(g.pos0, np.float64); st = np.array(g.step, np.float64)
        out = np.zeros((g.n[0], g.n[1], g.n[2], 3)) if return_coefs else None
        _check(self.lib.mmff_grid_build(spos.shape[0], _lib.ptr(spos), _lib.ptr(sREQ), _lib.ptr(lv), _lib.ptr(nm),
                                        _lib.ptr(nc), sub.alphaMorse, int(g.n[0]), int(g.n[1]), int(g.n[2]),
                                        _lib.ptr(p0), _lib.ptr(st), _lib.ptr(out)), "mmff_grid_build")
        self.grid = g
        return out

    def upload(self, b: SystemBatch, vel=None):
        arrs = dict(natoms=np.ascontiguousarray(b.natoms, np.int32), nnode=np.ascontiguousarray(b.nnode, np.int32),
                    pos=np.ascontiguousarray(b.pos, np.float64),
                    vel=None if vel is None else np.ascontiguousarray(vel, np.float64),
                    neighs=np.ascontiguousarray(b.neighs, np.int32), neighCell=np.ascontiguousarray(b.neighCell, np.int32),
                    bkneighs=np.ascontiguousarray(b.bkneighs, np.int32), REQs=np.ascontiguousarray(b.REQs, np.float64),
                    apars=np.ascontiguousarray(b.apars, np.float64), bLs=np.ascontiguousarray(b.bLs, np.float64),
                    bKs=np.ascontiguousarray(b.bKs, np.float64), Ksp=np.ascontiguousarray(b.Ksp, np.float64),
                    Kpp=np.ascontiguousarray(b.Kpp, np.float64), lvec=np.ascontiguousarray(b.lvec.reshape(-1, 9), np.float64))
        a = arrs
        _check(self.lib.mmff_systems_upload(b.nsys, _lib.ptr(a["natoms"]), _lib.ptr(a["nnode"]), _lib.ptr(a["pos"]),
                                            _lib.ptr(a["vel"]), _lib.ptr(a["neighs"]), _lib.ptr(a["neighCell"]),
                                            _lib.ptr(a["bkneighs"]), _lib.ptr(a["REQs"]), _lib.ptr(a["apars"]),
                                            _lib.ptr(a["bLs"]), _lib.ptr(a["bKs"]), _lib.ptr(a["Ksp"]),
                                            _lib.ptr(a["Kpp"]), _lib.ptr(a["lvec"])), "mmff_systems_upload")
        self.batch = b

    def set_constraints(self, anchor=None, K=None):
        """Per-atom position springs for relaxations (relax_multi.cl:995-1010):
        anchor [sum natoms, 4] = (x, y, z, on if > 0) in world coordinates,
        K [sum natoms, 3 or 4] spring constants; None clears."""
        if anchor is None:
            _check(self.lib.mmff_set_constraints(None, None), "mmff_set_constraints")
            return
        a = np.ascontiguousarray(anchor, np.float64)
        k = np.zeros((a.shape[0], 4)); k[:, :np.asarray(K).shape[1]] = K
        _check(self.lib.mmff_set_constraints(_lib.ptr(a), _lib.ptr(k)), "mmff_set_constraints")

    def set_bond_constraints(self, dist=(), angles=()):
        """Distance / angle constraints between atoms for relaxations (FireCore's
        Constrains, constrains.h): dist = [(system or -1, i0, i1, lmin, lmax, kmin,
        kmax, flim[, sa, sb, sc])], angles = [(system or -1, centre, end1, end2,
        ang0_rad, k)]; local atom indices; empty clears."""
        di = np.array([[int(x) for x in d[:3]] for d in dist], np.int32).reshape(-1, 3)
        dp = np.zeros((len(dist), 8))
        for r, d in enumerate(dist):
            dp[r, :len(d) - 3] = d[3:]
        ai = np.array([[int(x) for x in a[:4]] for a in angles], np.int32).reshape(-1, 4)
        ap = np.array([a[4:6] for a in angles], np.float64).reshape(-1, 2)
        _check(self.lib.mmff_set_bond_constraints(len(dist), _lib.ptr(di), _lib.ptr(dp), len(angles), _lib.ptr(ai),
                                                  _lib.ptr(ap)), "mmff_set_bond_constraints")

    def restore(self):
        _check(self.lib.mmff_systems_restore(), "mmff_systems_restore")

    def set_state(self, pos, vel=None, reset_fire=True):
        pos = np.ascontiguousarray(pos, np.float64)
        vel = None if vel is None else np.ascontiguousarray(vel, np.float64)
        _check(self.lib.mmff_systems_set_state(_lib.ptr(pos), _lib.ptr(vel), int(reset_fire)), "mmff_systems_set_state")

    # ---------------------------------------------------------------- compute
    def eval(self, energy: bool = True):
        """Forces [sum nvecs, 3] (float64 copies of the FP32 results) and energies [nsys, 4]."""
        _check(self.lib.mmff_eval(int(energy)), "mmff_eval")
        b = self.batch
        F = np.zeros((int(b.nvecs.sum()), 3))
        _check(self.lib.mmff_get_forces(_lib.ptr(F)), "mmff_get_forces")
        E = None
        if energy:
            E = np.zeros((b.nsys, 4))
            _check(self.lib.mmff_get_energies(_lib.ptr(E)), "mmff_get_energies")
        return F, E

    def relax(self, nstep_max: int, Fconv: float = 1e-4, conv_mode: int = 1, sync: bool = True):
        _check(self.lib.mmff_relax(int(nstep_max), float(Fconv), int(conv_mode)), "mmff_relax")
        if sync:
            self.sync()

    def surf_upload(self, sub: Substrate, Rdamp: float = 1.0):
        """Substrate atoms for the direct term (flag SURF; no grid needed)."""
        spos = np.ascontiguousarray(sub.spos, np.float64); sREQ = np.ascontiguousarray(sub.sREQ, np.float64)
        lv = np.ascontiguousarray(sub.lvec.reshape(9), np.float64); nm = np.array(sub.nPBC_mors, np.int32)
        _check(self.lib.mmff_surf_upload(spos.shape[0], _lib.ptr(spos), _lib.ptr(sREQ), _lib.ptr(lv), _lib.ptr(nm),
                                         float(Rdamp)), "mmff_surf_upload")

    def set_md(self, dt=0.05, gamma=0.1, T=300.0, seed=12345):
        """Langevin drive parameters (resets the random stream's step count)."""
        _check(self.lib.mmff_set_md(float(dt), float(gamma), float(T), int(seed)), "mmff_set_md")

    def md(self, nsteps: int, sync: bool = True):
        """nsteps Langevin steps of every system."""
        _check(self.lib.mmff_md(int(nsteps)), "mmff_md")
        if sync:
            self.sync()

    def set_explore(self, n_explore: int, n_relax: int = 0, start_exploring: bool = False):
        """Set up (and reset) the exploring cycle of the global optimiser for the
        current systems: n_explore Langevin steps (``set_md``'s drive) after every
        minimum found or after n_relax FIRE steps without one (0: never)."""
        _check(self.lib.mmff_set_explore(int(n_explore), int(n_relax), int(bool(start_exploring))),
               "mmff_set_explore")

    def explore(self, nsteps: int, Fconv: float = 1e-4, conv_mode: int = 1, sync: bool = True):
        """nsteps steps of the exploring cycle for every system."""
        _check(self.lib.mmff_explore(int(nsteps), float(Fconv), int(conv_mode)), "mmff_explore")
        if sync:
            self.sync()

    def explore_state(self):
        """(gopt [nsys, 4] = (exploring, steps in phase, minima found, phases given
        up), the last minimum found [sum nvecs, 3] in world coordinates)."""
        b = self.batch
        gopt = np.zeros((b.nsys, 4), dtype=np.int32)
        minpos = np.zeros((int(b.nvecs.sum()), 3))
        _check(self.lib.mmff_get_explore(_lib.ptr(gopt), _lib.ptr(minpos)), "mmff_get_explore")
        return gopt, minpos

    def sync(self):
        _check(self.lib.mmff_sync(), "mmff_sync")

    def state(self):
        b = self.batch
        nv = int(b.nvecs.sum())
        pos = np.zeros((nv, 3)); vel = np.zeros((nv, 3)); fire = np.zeros((b.nsys, 4))
        st = np.zeros(b.nsys, np.int32); ns = np.zeros(b.nsys, np.int32); fc = np.zeros(b.nsys)
        _check(self.lib.mmff_get_state(_lib.ptr(pos), _lib.ptr(vel), _lib.ptr(fire), _lib.ptr(st), _lib.ptr(ns),
                                       _lib.ptr(fc)), "mmff_get_state")
        return dict(pos=pos, vel=vel, fire=fire, status=st, nsteps=ns, fconv=fc)

    def grid_sample(self, pos, PLQ):
        pos = np.ascontiguousarray(pos, np.float64); PLQ = np.ascontiguousarray(PLQ, np.float64)
        fe = np.zeros((pos.shape[0], 4))
        _check(self.lib.mmff_grid_sample(pos.shape[0], _lib.ptr(pos), _lib.ptr(PLQ), _lib.ptr(fe)), "mmff_grid_sample")
        return fe

    # ---------------------------------------------------------------- timing
    def timer_start(self):
        _check(self.lib.mmff_timer_start(), "mmff_timer_start")

    def timer_stop(self) -> float:
        ms = self.lib.mmff_timer_stop()
        if ms < 0:
            raise RuntimeError("mmff_timer_stop failed")
        return ms

    def buckets(self):
        out = []
        for b in range(max(0, self.lib.mmff_num_buckets())):
            info = np.zeros(7, np.int32)
            _check(self.lib.mmff_bucket_info(b, _lib.ptr(info)), "mmff_bucket_info")
            out.append(dict(zip(["threads", "pair_split", "nsys", "maxNA", "maxNN", "smem", "ctas"], info.tolist())))
        return out
