#!/usr/bin/env python
"""Relaxed systems/s to max|F| < 1e-4 eV/A on B200: learned + batched vs plain
batched FIRE (the default workload), or the plain path alone.

Default workload (--workload learned, N=1): 16384 fresh molecules of 20-400
atoms (log-uniform; C:N:O:H = 10:2:2:10 heavy-atom trees, random rigid
rotation + 0.15 A noise) 3 A above a rigid rock-salt slab (a = 5.64 A,
3 layers, 4x4 cells, +-0.9 e), B-spline GridFF 226x226x200 (0.1 A), LJ +
Coulomb pairs with a 10 A cutoff over x,y PBC images, FP32 forces / FP64 FIRE
reductions, FIRE dt 0.1 with the 10 eV/A force clamp, at most 4000 steps per
system.  The network (68 -> 128 -> 128 -> 3, SiLU, bf16 on tcgen05) is
first trained on the plain relaxer's trajectories of separately seeded
molecules; then both arms relax the same 16384 molecules: plain FIRE, and two
energy-gated learned moves per molecule followed by the same FIRE.  value =
the learned arm's converged systems / device time.

--workload replicas: 4096 rotated replicas of one 60-atom molecule, plain FIRE.
--workload uneven: a queue of 32768 molecules of 20-400 atoms, plain FIRE.

One bench step = one full relaxation of the batch from its initial state (the
persistent kernels retire converged systems and claim the next ones).  Values
are converged systems / device time of the timed steps, all ranks (one
process per GPU, independent systems per rank: weak scaling).

--impl reference times FireCore's own FP64 CPU relaxation (oracle/_ref, the
reference's MolWorld_sp3::run_no_omp compiled from its sources) on the box's
host cores, on a bounded sample of the same molecules.
"""
import argparse
import json
import math
import multiprocessing as mp
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "relaxed systems/s to Fmax<1e-4 eV/A on 1 B200 (plain batched FIRE)"
UNIT = "systems/s"
FCONV = 1e-4
MAXSTEPS = 4000
RCUT = 10.0
FLIM = 10.0
PAIR_FLOPS = 32          # algorithmic FP32 flops per pair-image (both directions counted)
GRID_BYTES = 1024        # 64 float4 gathers per atom B-spline sample
# DRAM bytes (read + write) per system-step of the relax kernel the autotuner
# picks for the 4096-replica workload, from an ncu capture of that kernel on
# 4096 systems x 200 steps (98.6 + 54.9 MB); scaled by the system-steps of a launch
DRAM_BYTES_PER_SYSTEM_STEP = 187.4


def env_rank():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def workload(rank, nsys, kind="replicas"):
    from firecore_b200 import systems as S
    sub = S.make_slab()                      # 226 x 226 x 200, nPBC_coul (25,25,0)
    if kind == "uneven":
        batch = S.config_uneven(seed=2 + 7919 * rank, nsys=nsys)
    else:
        batch = S.config_replicas(seed=1 + 7919 * rank, nrep=nsys)
    return sub, batch


def workload_name(args):
    if args.workload == "uneven":
        return (f"queue of {args.nsys} distinct molecules, 20-400 atoms log-uniform (CSR, size buckets, one "
                f"persistent kernel per bucket claiming systems from its work queue: converged systems retire and "
                f"their CTA slots refill) on NaCl slab, GridFF 226x226x200, Rcut {RCUT} A, Fmax<{FCONV}, "
                f"<= {MAXSTEPS} FIRE steps")
    return (f"{args.nsys} replicas x 60-atom molecule on NaCl slab, GridFF 226x226x200, "
            f"Rcut {RCUT} A, Fmax<{FCONV}, <= {MAXSTEPS} FIRE steps")


def cpu_info():
    model = "unknown"
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return model, os.cpu_count() or 1


class ClockSampler:
    """nvidia-smi clocks / throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        self.f.flush()
        rows = []
        try:
            for line in open(self.f.name):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        except OSError:
            pass
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


# --------------------------------------------------------------------------- our arm
def run_ours(args):
    import torch
    rank, wsize, lrank = env_rank()
    torch.cuda.set_device(lrank)
    dist = None
    if wsize > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    from firecore_b200 import _lib
    from firecore_b200.world import DEFAULT_FLAGS, NONBONDED, PBC, FireParams, World
    lib = _lib.load()
    sub, batch = workload(rank, args.nsys, args.workload)
    w = World(lrank)
    t0 = time.perf_counter()
    C = w.grid_build(sub, return_coefs=True)
    w.sync()
    grid_build_s = time.perf_counter() - t0
    # --terms pairs (profiling only): the relax kernels with the pair term alone
    pairs_only = args.terms == "pairs"
    w.set_params(flags=(NONBONDED | PBC) if pairs_only else DEFAULT_FLAGS, npbc=(1, 1, 0), Rcut=RCUT)
    w.set_fire(FireParams(Flim=FLIM))
    w.upload(batch)
    nsys = batch.nsys
    natoms = batch.natoms.astype(np.int64)
    # launch shapes from the autotuner (untimed; the choice is reported)
    t0 = time.perf_counter()
    tune_rows = []
    if args.tuning and w.load_tuning(args.tuning):
        pass                                    # saved launch shapes of an earlier run
    elif not args.no_tune:
        tune_rows = w.autotune(nstep_probe=50, path=args.tuning)
    tune_s = time.perf_counter() - t0
    w.set_graph(True)
    # counting pass (untimed): algorithmic work of one relaxation of this batch
    lib.mmff_set_counting(1)
    w.restore(); w.relax(MAXSTEPS, FCONV, 1)
    cnt = (np.ctypeslib.ctypes.c_ulonglong * 5)()
    lib.mmff_get_counters(np.ctypeslib.ctypes.cast(cnt, np.ctypeslib.ctypes.c_void_p))
    pair_images, grid_samples, force_evals = int(cnt[0]), int(cnt[1]), int(cnt[2])
    lib.mmff_set_counting(0)
    st0 = w.state()
    if pairs_only:
        args.no_cpu = args.no_e2e = True
        attr_t, attr_pairs, attr_grid = {"all": 1.0, "no_pairs": 1.0, "no_grid": 1.0}, 0, 0
    else:
        attr_t, attr_pairs, attr_grid = term_attribution(w, lib)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")   # > 126 MB L2

    def one_step():
        flush.zero_()
        torch.cuda.synchronize()
        w.timer_start()
        w.restore()
        w.relax(MAXSTEPS, FCONV, 1, sync=False)
        ms = w.timer_stop()
        status = np.zeros(nsys, np.int32)
        lib.mmff_get_state(None, None, None, _lib.ptr(status), None, None)
        return ms, int((status == 1).sum()), int((status == -1).sum())

    for _ in range(args.warmup):
        one_step()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    times, conv, nans = [], 0, 0
    with ClockSampler(lrank) as clk:
        t_wall = time.perf_counter()
        for _ in range(args.steps):
            ms, c, n = one_step()
            times.append(ms); conv += c; nans += n
        torch.cuda.synchronize()
        t_wall = time.perf_counter() - t_wall
    if dist:
        dist.barrier()
    clocks = clk.summary()
    t_dev = sum(times) / 1e3
    # e2e through the public API: host positions in, host state out, every step
    e2e = None
    if not args.no_e2e:
        pos_h = np.ascontiguousarray(batch.pos)
        nv = int(batch.nvecs.sum())
        t_e2e, conv_e2e = 0.0, 0
        for k in range(max(1, args.steps)):
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            w.set_state(pos_h, None, reset_fire=True)
            w.relax(MAXSTEPS, FCONV, 1, sync=True)
            st = w.state()
            t_e2e += time.perf_counter() - t1
            conv_e2e += int((st["status"] == 1).sum())
        h2d = nv * 16 * 2 + nsys * 32
        d2h = nv * 16 * 2 + nsys * (32 + 4 + 4 + 4)
        e2e = {"value": conv_e2e / t_e2e, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h}
    tot_conv, t_max, e2e_v = aggregate_ranks(conv, t_dev, e2e["value"] if e2e else None, dist, "cuda")
    if e2e:
        e2e["value"] = e2e_v
    value = tot_conv / t_max
    ms_step = 1e3 * t_max / args.steps
    # roofline of the relax kernel: pair term on FP32 CUDA cores
    fp32_peak = lib.mmff_peak_fp32()
    l2_peak = lib.mmff_peak_l2(64)
    t_launch = t_dev / args.steps
    achieved_tf = PAIR_FLOPS * pair_images / t_launch / 1e12
    grid_gbs = GRID_BYTES * grid_samples / t_launch / 1e9
    t_pair = (attr_t["all"] - attr_t["no_pairs"]) / 1e3
    t_grid = (attr_t["all"] - attr_t["no_grid"]) / 1e3
    pair_tf = PAIR_FLOPS * attr_pairs / t_pair / 1e12 if t_pair > 0 else None
    grid_term_gbs = GRID_BYTES * attr_grid / t_grid / 1e9 if t_grid > 0 else None
    out = None
    parity = parity_subset(w, batch, sub, C) if (rank == 0 and not pairs_only) else None
    if rank == 0:
        cpu = cpu_baseline(batch, sub, C, args, st0) if not args.no_cpu else None
        if cpu:
            parity["relaxed_geometry"] = cpu.pop("geometry")
        nconv0 = int((st0["status"] == 1).sum())
        steps_conv = st0["nsteps"][st0["status"] == 1]
        out = {
            "metric": METRIC if not pairs_only else "profiling: relax kernels with the pair term only (not the metric)",
            "value": value, "unit": UNIT, "n_gpus": wsize, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 forces / f64 FIRE reductions", "data": "synthetic (seeded generator)",
            "config": {"workload": workload_name(args),
                       "systems_per_gpu": args.nsys, "l2": "flushed (256 MB write) before every step",
                       "parallelism": f"replicas x{wsize}"},
            "converged_per_step": conv / args.steps, "nan_per_step": nans / args.steps,
            "median_steps_to_converge": float(np.median(steps_conv)) if len(steps_conv) else None,
            "converged_fraction": nconv0 / nsys,
            "grid_build_s": grid_build_s, "wall_s_timed": t_wall,
            "gpu_launches": args.steps * len(w.buckets()),
            "roofline": {"bound": "fp32", "achieved": achieved_tf, "peak": fp32_peak, "unit": "TFLOP/s",
                         "frac": achieved_tf / fp32_peak if fp32_peak > 0 else None,
                         "traffic": DRAM_BYTES_PER_SYSTEM_STEP * force_evals,
                         "peak_source": "measured FFMA microbenchmark (mmff_peak_fp32) on this GPU",
                         "work": f"{PAIR_FLOPS} flop x {pair_images} pair-images per launch",
                         "grid_l2": {"achieved": grid_gbs, "peak": l2_peak, "unit": "GB/s",
                                     "frac": grid_gbs / l2_peak if l2_peak > 0 else None,
                                     "work": f"{GRID_BYTES} B x {grid_samples} atom samples per launch"},
                         "pair_term": {"achieved": pair_tf, "peak": fp32_peak, "unit": "TFLOP/s",
                                       "frac": pair_tf / fp32_peak if (pair_tf and fp32_peak > 0) else None,
                                       "time_ms": 1e3 * t_pair, "work": f"{PAIR_FLOPS} flop x {attr_pairs} pair-images",
                                       "method": "200-step relax of the batch with all terms minus without the pair term"},
                         "grid_term": {"achieved": grid_term_gbs, "peak": l2_peak, "unit": "GB/s",
                                       "frac": grid_term_gbs / l2_peak if (grid_term_gbs and l2_peak > 0) else None,
                                       "time_ms": 1e3 * t_grid,
                                       "method": "200-step relax with all terms minus without GridFF"},
                         "term_times_ms": attr_t},
            "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks, "parity_vs_oracle": parity,
            "buckets": w.buckets(), "relax_graph": True,
            "autotune": {"seconds": tune_s, "chosen": {str(k): v for k, v in w.tuning().items()},
                         "candidates": [[r["size_class"], r["kind"], r["threads"], r["pair_lanes"],
                                         round(r["us_per_system_step"], 4)] for r in tune_rows]},
        }
        print(json.dumps(out))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return out


def aggregate_ranks(conv, t_dev, e2e_value, dist, device):
    """Whole-job numbers of the replica ranks (disjoint systems, no exchange on
    the data path): converged systems and end-to-end rates summed, device time
    the maximum over ranks.  Every rank makes the same two collective calls."""
    if dist is None:
        return float(conv), float(t_dev), e2e_value
    import torch
    s = torch.tensor([float(conv), 0.0 if e2e_value is None else float(e2e_value)], device=device, dtype=torch.float64)
    dist.all_reduce(s)
    m = torch.tensor([float(t_dev)], device=device, dtype=torch.float64)
    dist.all_reduce(m, op=dist.ReduceOp.MAX)
    return float(s[0]), float(m[0]), (None if e2e_value is None else float(s[1]))


def term_attribution(w, lib, nsteps=200):
    """Device time of each force term inside the fused relax kernel: the same
    fixed-length relaxation (Fmax < 0 never converges, so every system runs
    nsteps steps) with all terms, and with one term switched off.  Returns
    times [ms] and the pair-images / grid samples of the full run."""
    from firecore_b200.world import ANGLES, BONDS, DEFAULT_FLAGS, GRID, NONBONDED, PIPI, PISIGMA, SUB_ANGLE_NB
    # without the pair term the 1-3 subtraction of the angle terms must go too,
    # or the molecules collapse and retire as non-finite
    variants = {"all": DEFAULT_FLAGS, "no_pairs": DEFAULT_FLAGS & ~(NONBONDED | SUB_ANGLE_NB),
                "no_grid": DEFAULT_FLAGS & ~GRID, "no_bonded": DEFAULT_FLAGS & ~(BONDS | ANGLES | PIPI | PISIGMA)}
    times, nan = {}, {}
    for name, fl in variants.items():
        w.set_params(flags=fl, npbc=(1, 1, 0), Rcut=RCUT)
        best = 1e30
        for _ in range(3):
            w.restore()
            w.sync()
            w.timer_start()
            w.relax(nsteps, 0.0, 1, sync=False)
            best = min(best, w.timer_stop())
        times[name] = best
        st = np.zeros(w.batch.nsys, np.int32)
        lib.mmff_get_state(None, None, None, _lib_ptr(st), None, None)
        nan[name] = int((st == -1).sum())
    w.set_params(flags=DEFAULT_FLAGS, npbc=(1, 1, 0), Rcut=RCUT)
    lib.mmff_set_counting(1)
    w.restore(); w.relax(nsteps, 0.0, 1)
    cnt = (np.ctypeslib.ctypes.c_ulonglong * 5)()
    lib.mmff_get_counters(np.ctypeslib.ctypes.cast(cnt, np.ctypeslib.ctypes.c_void_p))
    lib.mmff_set_counting(0)
    w.restore()
    times["retired_nonfinite"] = nan
    return times, int(cnt[0]), int(cnt[1])


def _lib_ptr(a):
    from firecore_b200 import _lib
    return _lib.ptr(a)


def parity_subset(w, batch, sub, C, nsub=64):
    """Device against the FP64 oracle on the first nsub systems (untimed).
    Forces at the starting geometries (|F| ~ 1-10 eV/A): per system the largest
    per-atom force error over the largest force.  At the final geometries the
    forces are ~Fconv, so their error is stated in eV/A, and the energies in
    eV/atom.  Leaves the device state at the starting geometries."""
    from oracle import oracle as O
    idx = list(range(min(nsub, batch.nsys)))
    a, n, v = batch.offsets()
    sb = batch.subset(idx)
    _, _, vs = sb.offsets()
    rows = np.concatenate([np.arange(v[s], v[s + 1]) for s in idx])
    P = O.make_params(sub.grid, npbc=(1, 1, 0), Rcut=RCUT)
    F, E = w.eval(True)
    pos = w.state()["pos"]
    Fo, Eo = O.eval_forces(sb, P, C, pos=pos[rows])
    Fd = F[rows]
    fabs = [float(np.abs(Fd[vs[k]:vs[k + 1]] - Fo[vs[k]:vs[k + 1]]).max()) for k in range(len(idx))]
    eerr = np.abs(E[idx, 3] - Eo[:, 3]) / sb.natoms
    w.restore()
    F0, _ = w.eval(True)
    Fo0, _ = O.eval_forces(sb, P, C, pos=batch.pos[rows])
    F0 = F0[rows]
    frel = [float(np.linalg.norm(F0[vs[k]:vs[k + 1]] - Fo0[vs[k]:vs[k + 1]], axis=1).max()
                  / max(np.linalg.norm(Fo0[vs[k]:vs[k + 1]], axis=1).max(), 1e-12)) for k in range(len(idx))]
    return {"systems": len(idx),
            "start_max_force_rel_err": max(frel), "start_median_force_rel_err": float(np.median(frel)),
            "final_max_force_abs_err_eV_per_A": max(fabs),
            "final_max_energy_err_eV_per_atom": float(eerr.max()),
            "final_median_energy_err_eV_per_atom": float(np.median(eerr)),
            "reference": "FP64 oracle (restatement pinned to FireCore's compiled run_no_omp physics)"}


def geometry_parity(batch, st0, r, nsample, P, F, C, ncores):
    """Relaxed geometries of the device (st0) against the oracle's FP64
    relaxation of the same first nsample systems (r): atom RMSD per system
    converged in both.  At Fmax < 1e-4 eV/A a soft mode (a molecule sliding on
    the slab, k ~ 0.01 eV/A^2) leaves ~0.01 A of slack, so FP32 and FP64
    trajectories stop at different points of the same basin; both end points
    are therefore also re-relaxed in FP64 to Fmax < 1e-6 eV/A (untimed) and
    compared again: agreement there means the same minimum."""
    from oracle import oracle as O
    _, _, v = batch.offsets()
    both = [s for s in range(nsample) if st0["status"][s] == 1 and r["converged"][s] == 1]
    if not both:
        return {"systems_converged_in_both": 0}
    sb = batch.subset(both)
    _, _, vb = sb.offsets()
    rows = np.concatenate([np.arange(v[s], v[s + 1]) for s in both])
    _, _, vs = batch.subset(range(nsample)).offsets()
    rows_r = np.concatenate([np.arange(vs[s], vs[s + 1]) for s in both])

    def rmsd(pa, pb):
        out = []
        for k in range(len(both)):
            na = int(sb.natoms[k])
            d = pa[vb[k]:vb[k] + na, :3] - pb[vb[k]:vb[k] + na, :3]
            out.append(float(np.sqrt((d ** 2).sum(1).mean())))
        return np.array(out)

    pd, po = st0["pos"][rows], r["pos"][rows_r]
    r0 = rmsd(pd, po)
    td = O.relax(sb, P, F, C, niter=30000, Fconv=1e-6, conv_mode=1, pos=pd, nthreads=ncores)
    to = O.relax(sb, P, F, C, niter=30000, Fconv=1e-6, conv_mode=1, pos=po, nthreads=ncores)
    ok = (td["converged"] == 1) & (to["converged"] == 1)
    r1 = rmsd(td["pos"], to["pos"])[ok]
    return {"systems_converged_in_both": len(both),
            "fraction_rmsd_le_1e-3_A": float((r0 <= 1e-3).mean()),
            "median_rmsd_A": float(np.median(r0)), "max_rmsd_A": float(r0.max()),
            "same_minimum": {"method": "both end points re-relaxed by the FP64 oracle to Fmax < 1e-6 eV/A",
                             "systems": int(ok.sum()),
                             "fraction_rmsd_le_1e-3_A": float((r1 <= 1e-3).mean()) if len(r1) else None,
                             "median_rmsd_A": float(np.median(r1)) if len(r1) else None,
                             "max_rmsd_A": float(r1.max()) if len(r1) else None}}


def cpu_baseline(batch, sub, C, args, st0):
    """The FP64 oracle (OpenMP over systems) on a bounded sample of the same
    workload, same parameters (10 A cutoff, force clamp, Fmax criterion).  Its
    relaxed geometries are compared with the device's (st0) as well."""
    from oracle import oracle as O
    model, ncores = cpu_info()
    nsample = int(min(batch.nsys, max(64, 32 * ncores), 1024))
    if args.workload == "uneven":             # up to 400 atoms: ~25x the pair work of a 60-atom system
        nsample = int(min(batch.nsys, max(16, 2 * ncores)))
    sb = batch.subset(range(nsample))
    P = O.make_params(sub.grid, npbc=(1, 1, 0), Rcut=RCUT)
    F = O.make_fire(Flim=FLIM)
    t0 = time.perf_counter()
    r = O.relax(sb, P, F, C, niter=MAXSTEPS, Fconv=FCONV, conv_mode=1, nthreads=ncores)
    dt = time.perf_counter() - t0
    conv = int((r["converged"] == 1).sum())
    return {"value": conv / dt, "unit": UNIT, "cores": ncores, "kind": "port",
            "sample": f"{nsample} of the systems, full relaxation each ({conv} converged, {dt:.1f} s), CPU: {model}",
            "geometry": geometry_parity(batch, st0, r, nsample, P, F, C, ncores)}


# --------------------------------------------------------------------------- learned vs plain
LEARNED_METRIC = "relaxed systems/s to Fmax<1e-4 eV/A on 1 B200: learned+batched vs plain FIRE"
SNAPSHOTS = (0, 25, 100, 400)       # FIRE steps at which training descriptors are taken
NWARM = 2                           # learned warm-start moves per system
PROJECTION = 1                      # warm-start moves: rigid-body projection of the network's displacements
TRAIN_TARGET = "rigid"              # training targets: the rigid-body part of the displacement to the minimum


def learned_name(args):
    return (f"{args.nsys} fresh molecules per GPU, 20-400 atoms log-uniform (CSR, size buckets, persistent kernels "
            f"with in-kernel retire/refill, one CUDA graph per relaxation) on NaCl slab, GridFF 226x226x200, Rcut "
            f"{RCUT} A; learned arm: {NWARM} energy-gated learned moves per system (rigid-body projection of the "
            f"network's per-atom displacements), then FIRE to Fmax<{FCONV} "
            f"(<= {MAXSTEPS} steps); plain arm: FIRE only on the same inputs; network trained on the plain "
            f"relaxer's trajectories of {args.train_sys} separately seeded molecules")


def count_work(w, lib, nstep_max):
    """Algorithmic work of one plain relaxation of the uploaded batch (counting
    build of the same kernels, untimed): pair-images inside the cutoff, atom
    GridFF samples, system force evaluations."""
    lib.mmff_set_counting(1)
    w.restore(); w.relax(nstep_max, FCONV, 1)
    cnt = (np.ctypeslib.ctypes.c_ulonglong * 5)()
    lib.mmff_get_counters(np.ctypeslib.ctypes.cast(cnt, np.ctypeslib.ctypes.c_void_p))
    lib.mmff_set_counting(0)
    return int(cnt[0]), int(cnt[1]), int(cnt[2])


def run_learned(args):
    """The metric's own configuration: learned warm start + batched FIRE
    against plain batched FIRE on the same fresh uneven systems.

    Training set (untimed): descriptors at FIRE steps SNAPSHOTS of the plain
    relaxer on separately seeded systems, targets = displacement to the
    relaxed geometry (converged systems only); the network is trained on the
    GPU (tcgen05 forward/backward + AdamW).  One bench step = one full
    relaxation of the production batch from its initial state: plain arm =
    one relax call (one graph launch); learned arm = NWARM energy-gated learned
    moves per system, then the same relax call.  value = the learned arm's
    converged systems / its device time (L2 flushed before every step)."""
    import torch
    from firecore_b200 import _lib
    from firecore_b200 import learned as L
    from firecore_b200 import systems as S
    from firecore_b200.world import DEFAULT_FLAGS, FireParams, World
    rank, wsize, lrank = env_rank()
    torch.cuda.set_device(lrank)
    dist = None
    if wsize > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    lib = _lib.load()
    sub = S.make_slab()
    w = World(lrank)
    t0 = time.perf_counter()
    C = w.grid_build(sub, return_coefs=True)
    w.sync()
    grid_build_s = time.perf_counter() - t0
    w.set_params(flags=DEFAULT_FLAGS, npbc=(1, 1, 0), Rcut=RCUT)
    w.set_fire(FireParams(Flim=FLIM))
    w.set_graph(True)
    prop = L.Proposal()
    # ---- training set from the plain relaxer (separately seeded systems)
    t0 = time.perf_counter()
    train = S.config_uneven(seed=1001 + 7919 * rank, nsys=args.train_sys)
    w.upload(train)
    F, T = L.trajectory_dataset(w, prop, train, snapshots=SNAPSHOTS, nstep_max=MAXSTEPS, Fconv=FCONV,
                                target=TRAIN_TARGET)
    data_s = time.perf_counter() - t0
    rng = np.random.default_rng(0)
    perm = rng.permutation(len(F))
    scale = float(np.sqrt((T ** 2).mean()))
    prop.set_params(L.init_params(0), F.mean(0), F.std(0) + 1e-6, scale)
    prop.set_data(F[perm], T[perm])
    w.sync(); w.timer_start()
    losses = prop.train(args.train_steps, batch_tiles=512, lr=1e-3, wd=0.01)
    train_ms = w.timer_stop()
    # ---- production systems, both arms on the same inputs
    prod = S.config_uneven(seed=2002 + 7919 * rank, nsys=args.nsys)
    w.upload(prod)
    nsys = prod.nsys
    t0 = time.perf_counter()
    tune_rows = []
    if args.tuning and w.load_tuning(args.tuning):
        pass
    elif not args.no_tune:
        tune_rows = w.autotune(nstep_probe=50, path=args.tuning)
    tune_s = time.perf_counter() - t0
    prop.set_elements(prod.elements)
    prop.set_projection(PROJECTION)
    pair_images, grid_samples, force_evals = count_work(w, lib, MAXSTEPS)
    attr_t, attr_pairs, attr_grid = term_attribution(w, lib)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")   # > 126 MB L2
    status = np.zeros(nsys, np.int32)

    def arm(learned):
        flush.zero_()
        torch.cuda.synchronize()
        l0 = lib.mmff_kernel_launches()
        w.timer_start()
        w.restore()
        acc = prop.warmstart(nsys, NWARM) if learned else None
        w.relax(MAXSTEPS, FCONV, 1, sync=False)
        ms = w.timer_stop()
        nl = lib.mmff_kernel_launches() - l0
        lib.mmff_get_state(None, None, None, _lib.ptr(status), None, None)
        return ms, int((status == 1).sum()), int((status == -1).sum()), acc, nl

    for _ in range(args.warmup):
        arm(False)
        arm(True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    res = {"plain": dict(ms=[], conv=0, nan=0, launches=0), "learned": dict(ms=[], conv=0, nan=0, launches=0, acc=[])}
    with ClockSampler(lrank) as clk:
        t_wall = time.perf_counter()
        for _ in range(args.steps):
            for name in ("plain", "learned"):
                ms, c, n, acc, nl = arm(name == "learned")
                r = res[name]
                r["ms"].append(ms); r["conv"] += c; r["nan"] += n; r["launches"] += nl
                if acc is not None:
                    r["acc"].append(float(np.mean(acc)))
        torch.cuda.synchronize()
        t_wall = time.perf_counter() - t_wall
    if dist:
        dist.barrier()
    clocks = clk.summary()
    st_l = w.state()            # final state of the learned arm (last timed step)
    # e2e through the public API with host buffers: positions in, learned
    # moves + relaxation, state out, every step
    e2e = None
    if not args.no_e2e:
        pos_h = np.ascontiguousarray(prod.pos)
        nv = int(prod.nvecs.sum())
        t_e2e, conv_e2e = 0.0, 0
        for _ in range(max(1, args.steps)):
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            w.set_state(pos_h, None, reset_fire=True)
            prop.warmstart(nsys, NWARM)
            w.relax(MAXSTEPS, FCONV, 1, sync=True)
            st = w.state()
            t_e2e += time.perf_counter() - t1
            conv_e2e += int((st["status"] == 1).sum())
        h2d = nv * 16 * 2 + nsys * 32
        d2h = nv * 16 * 2 + nsys * (32 + 4 + 4 + 4) + nsys * 4
        e2e = {"value": conv_e2e / t_e2e, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "path": "World.set_state -> Proposal.warmstart -> World.relax -> World.state (C-ABI, host arrays)"}
    parity = learned_parity(prod, sub, C, w) if rank == 0 else None      # device holds the learned arm's end state
    buckets = w.buckets()
    refsem = None if args.no_refsem else reference_semantics(w, prod, args)
    tl = sum(res["learned"]["ms"]) / 1e3
    tp = sum(res["plain"]["ms"]) / 1e3
    tot_l, tmax_l, e2e_v = aggregate_ranks(res["learned"]["conv"], tl, e2e["value"] if e2e else None, dist, "cuda")
    tot_p, tmax_p, _ = aggregate_ranks(res["plain"]["conv"], tp, None, dist, "cuda")
    if e2e:
        e2e["value"] = e2e_v
    value = tot_l / tmax_l
    plain_value = tot_p / tmax_p
    out = None
    if rank == 0:
        # roofline of the relax kernel, from the plain arm (its work is counted)
        fp32_peak = lib.mmff_peak_fp32()
        l2_peak = lib.mmff_peak_l2(64)
        t_launch = tp / args.steps
        achieved_tf = PAIR_FLOPS * pair_images / t_launch / 1e12
        grid_gbs = GRID_BYTES * grid_samples / t_launch / 1e9
        t_pair = (attr_t["all"] - attr_t["no_pairs"]) / 1e3
        t_grid = (attr_t["all"] - attr_t["no_grid"]) / 1e3
        pair_tf = PAIR_FLOPS * attr_pairs / t_pair / 1e12 if t_pair > 0 else None
        grid_term_gbs = GRID_BYTES * attr_grid / t_grid / 1e9 if t_grid > 0 else None
        cpu = None if args.no_cpu else cpu_baseline_uneven(prod, sub, C)
        med = lambda st: float(np.median(st["nsteps"][st["status"] == 1])) if (st["status"] == 1).any() else None
        out = {
            "metric": LEARNED_METRIC, "value": value, "unit": UNIT, "n_gpus": wsize, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * tmax_l / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 forces / f64 FIRE reductions; bf16 network, f32 accumulation",
            "data": "synthetic (seeded generator)",
            "config": {"workload": learned_name(args), "systems_per_gpu": args.nsys,
                       "l2": "flushed (256 MB write) before every step", "parallelism": f"replicas x{wsize}"},
            "plain": {"value": plain_value, "ms_per_step": 1e3 * tmax_p / args.steps,
                      "converged_per_step": res["plain"]["conv"] / args.steps},
            "learned": {"value": value, "converged_per_step": res["learned"]["conv"] / args.steps,
                        "moves_kept_per_system": float(np.mean(res["learned"]["acc"])) if res["learned"]["acc"] else None,
                        "median_steps": med(st_l)},
            "speedup_learned_over_plain": value / plain_value if plain_value > 0 else None,
            "converged_fraction": res["learned"]["conv"] / args.steps / nsys,
            "nan_per_step": res["learned"]["nan"] / args.steps,
            "grid_build_s": grid_build_s, "wall_s_timed": t_wall,
            "gpu_launches": res["learned"]["launches"] + res["plain"]["launches"],
            "gpu_launches_per_step": {"learned": res["learned"]["launches"] / args.steps,
                                      "plain": res["plain"]["launches"] / args.steps},
            "roofline": {"bound": "fp32", "achieved": achieved_tf, "peak": fp32_peak, "unit": "TFLOP/s",
                         "frac": achieved_tf / fp32_peak if fp32_peak > 0 else None,
                         "traffic": None,
                         "kernel": "relax_kernel / relax_warp_kernel (all size buckets), plain arm",
                         "peak_source": "measured FFMA microbenchmark (mmff_peak_fp32) on this GPU",
                         "work": f"{PAIR_FLOPS} flop x {pair_images} pair-images per launch",
                         "grid_l2": {"achieved": grid_gbs, "peak": l2_peak, "unit": "GB/s",
                                     "frac": grid_gbs / l2_peak if l2_peak > 0 else None,
                                     "work": f"{GRID_BYTES} B x {grid_samples} atom samples per launch"},
                         "pair_term": {"achieved": pair_tf, "peak": fp32_peak, "unit": "TFLOP/s",
                                       "frac": pair_tf / fp32_peak if (pair_tf and fp32_peak > 0) else None,
                                       "time_ms": 1e3 * t_pair, "work": f"{PAIR_FLOPS} flop x {attr_pairs} pair-images",
                                       "method": "200-step relax of the batch with all terms minus without the pair term"},
                         "grid_term": {"achieved": grid_term_gbs, "peak": l2_peak, "unit": "GB/s",
                                       "frac": grid_term_gbs / l2_peak if (grid_term_gbs and l2_peak > 0) else None,
                                       "time_ms": 1e3 * t_grid,
                                       "method": "200-step relax with all terms minus without GridFF"},
                         "term_times_ms": attr_t},
            "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks, "parity_vs_oracle": parity,
            "reference_semantics": refsem,
            "buckets": buckets, "relax_graph": True,
            "autotune": {"seconds": tune_s, "chosen": {str(k): v for k, v in w.tuning().items()},
                         "candidates": [[r["size_class"], r["kind"], r["threads"], r["pair_lanes"],
                                         round(r["us_per_system_step"], 4)] for r in tune_rows]},
            "training": {"rows": int(len(F)), "snapshots": list(SNAPSHOTS), "target": TRAIN_TARGET,
                         "steps": args.train_steps,
                         "batch_atoms": 512 * 128, "first_loss": float(losses[0]),
                         "last_loss": float(np.mean(losses[-20:])), "train_ms": train_ms, "data_generation_s": data_s},
        }
        print(json.dumps(out))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return out


def reference_semantics(w, prod, args, nsub=4096):
    """The plain GPU path on FireCore's own run_no_omp semantics -- all pairs x
    9 PBC images (no cutoff), no force clamp, sum f^2 < Fconv^2 -- on the first
    nsub production molecules: the like-for-like counterpart of the reference
    arm (which times exactly that on the host cores).  One untimed run, then
    one timed run; the world is left on the benchmark's parameters with the
    full batch uploaded again."""
    from firecore_b200.world import DEFAULT_FLAGS, FireParams
    n = min(nsub, prod.nsys)
    sb = prod.subset(range(n))
    w.set_params(flags=DEFAULT_FLAGS, npbc=(1, 1, 0), Rcut=-1.0)
    w.set_fire(FireParams())
    w.upload(sb)
    w.relax(MAXSTEPS, FCONV, 0)
    w.restore()
    w.sync()
    w.timer_start()
    w.relax(MAXSTEPS, FCONV, 0, sync=False)
    ms = w.timer_stop()
    st = w.state()
    conv = int((st["status"] == 1).sum())
    w.set_params(flags=DEFAULT_FLAGS, npbc=(1, 1, 0), Rcut=RCUT)
    w.set_fire(FireParams(Flim=FLIM))
    w.upload(prod)
    return {"value": conv / (ms / 1e3), "unit": UNIT, "systems": n, "converged": conv, "ms": ms,
            "semantics": "plain batched FIRE on the GPU with FireCore's run_no_omp semantics: all pairs x 9 PBC "
                         "images, no force clamp, sum f^2 < Fconv^2 (the reference arm's semantics)"}


def learned_parity(prod, sub, C, w, nsub=32):
    """Final energies and forces of the learned arm (the device's current
    state) against the FP64 oracle at the same final geometries (first nsub
    converged systems): eV/atom and the largest per-atom force error in eV/A
    (the forces there are ~Fconv)."""
    from oracle import oracle as O
    st = w.state()
    Fd, E = w.eval(True)
    idx = [int(i) for i in np.where(st["status"] == 1)[0][:nsub]]
    if not idx:
        return None
    sb = prod.subset(idx)
    _, _, v = prod.offsets()
    rows = np.concatenate([np.arange(v[s], v[s + 1]) for s in idx])
    P = O.make_params(sub.grid, npbc=(1, 1, 0), Rcut=RCUT)
    Fo, Eo = O.eval_forces(sb, P, C, pos=st["pos"][rows])
    na = prod.natoms[idx].astype(np.float64)
    dE = np.abs(E[idx, 3] - Eo[:, 3]) / na
    return {"systems": len(idx), "final_max_energy_err_eV_per_atom": float(dE.max()),
            "final_median_energy_err_eV_per_atom": float(np.median(dE)),
            "final_max_force_abs_err_eV_per_A": float(np.abs(Fd[rows] - Fo).max()),
            "reference": "FP64 oracle (restatement pinned to FireCore's compiled run_no_omp physics)"}


def cpu_baseline_uneven(prod, sub, C):
    """FP64 oracle port (OpenMP over systems, all host cores), plain FIRE with
    the same parameters, on a bounded sample of the production molecules
    (2 per core: ~10-30 s of CPU work)."""
    from oracle import oracle as O
    model, ncores = cpu_info()
    nsample = int(min(prod.nsys, max(16, 2 * ncores)))
    sb = prod.subset(range(nsample))
    P = O.make_params(sub.grid, npbc=(1, 1, 0), Rcut=RCUT)
    F = O.make_fire(Flim=FLIM)
    t0 = time.perf_counter()
    r = O.relax(sb, P, F, C, niter=MAXSTEPS, Fconv=FCONV, conv_mode=1, nthreads=ncores)
    dt = time.perf_counter() - t0
    conv = int((r["converged"] == 1).sum())
    return {"value": conv / dt, "unit": UNIT, "cores": ncores, "kind": "port",
            "sample": f"first {nsample} production molecules, plain FIRE to Fmax<{FCONV}, full relaxation each "
                      f"({conv} converged, {dt:.1f} s), CPU: {model}"}


# --------------------------------------------------------------------------- reference arm
_REF = {}


def _ref_worker(args):
    """Relax systems through FireCore's own MolWorld_sp3::run_no_omp."""
    idx = args
    from oracle import oracle as O
    ref = O.ref()
    import ctypes
    b, C, g = _REF["batch"], _REF["C"], _REF["grid"]
    p = lambda a: ctypes.c_void_p(a.ctypes.data)
    a_off, n_off, v_off = b.offsets()
    npbc = np.array([1, 1, 0], np.int32)
    gn = np.array(g.n, np.int32); gp0 = np.array(g.pos0); gst = np.array(g.step)
    out = []
    for s in idx:
        na, nn = int(b.natoms[s]), int(b.nnode[s])
        pos = np.ascontiguousarray(b.pos[v_off[s]:v_off[s + 1]])
        arr = [np.ascontiguousarray(x[a_off[s]:a_off[s + 1]]) for x in (b.neighs, b.neighCell, b.REQs)]
        nar = [np.ascontiguousarray(x[n_off[s]:n_off[s + 1]]) for x in (b.apars, b.bLs, b.bKs, b.Ksp, b.Kpp)]
        lv = np.ascontiguousarray(b.lvec[s].reshape(9))
        bk = np.zeros((na, 4), np.int32); ng = np.zeros((na, 4), np.int32)
        ref.ref_setup(na, nn, p(pos), p(arr[0]), p(arr[1]), p(arr[2]), *[p(x) for x in nar], p(lv), p(npbc),
                      O.DEFAULT_FLAGS, 1.5, p(gn), p(gp0), p(gst), p(C), p(bk), p(ng))
        vel = np.zeros_like(pos)
        fire = np.array([0.1, 0.1, 0.0, 0.1, 0.01, 0.1, 1.1, 0.5, 0.8, 3, 0.0])
        oE = np.zeros(MAXSTEPS); oF = np.zeros(MAXSTEPS)
        it = ref.ref_relax(MAXSTEPS, FCONV, p(pos), p(vel), p(fire), p(oE), p(oF))
        out.append(1 if it < MAXSTEPS else 0)
    return out


def run_reference(args):
    """FireCore's own FP64 CPU relaxation (MolWorld_sp3::run_no_omp, compiled
    from the reference sources into oracle/_ref/libref_harness.so) on a
    bounded sample of the same molecules, one process per host core.

    Inputs: the molecules come from the host-only generator library
    (libmmff_gen.so, no CUDA); the 226x226x200 FP64 B-spline grid is an input
    of both arms that a CPU direct sum would take ~5 core-hours to build, so a
    one-time child process builds it with this repository's GPU grid builder
    and caches it on the box (untimed).  This process maps only the reference
    harness and the generator."""
    rank, wsize, _ = env_rank()
    if rank != 0:
        return
    from oracle import oracle as O
    model, ncores = cpu_info()
    if args.workload == "learned":
        from firecore_b200 import systems as S
        sub, batch = S.make_slab(), S.config_uneven(seed=2002, nsys=args.nsys)
    else:
        sub, batch = workload(0, args.nsys, args.workload)
    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libref_harness.so was not built (no reference tree)"}))
        return
    O.ref()                    # the timed library, mapped here before the workers fork
    cache = os.path.join(tempfile.gettempdir(), "mmff_grid_226x226x200.npy")
    if not os.path.exists(cache):
        code = ("import sys,numpy as np; sys.path.insert(0,%r); from firecore_b200 import systems as S; "
                "from firecore_b200.world import World; w=World(0); C=w.grid_build(S.make_slab(), return_coefs=True); "
                "np.save(%r, C)") % (ROOT, cache)
        subprocess.check_call([sys.executable, "-c", code])
    C = np.load(cache)
    _REF.update(batch=batch, C=C, grid=sub.grid)
    nsample = int(min(batch.nsys, max(8, 2 * ncores)))
    if args.workload != "replicas":
        nsample = int(min(batch.nsys, max(8, ncores)))      # up to 400 atoms each: ~25x a 60-atom molecule
    chunks = [list(range(k, nsample, ncores)) for k in range(min(ncores, nsample))]
    ctx = mp.get_context("fork")
    times, conv = [], 0
    with ctx.Pool(len(chunks)) as pool:
        for step in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            res = pool.map(_ref_worker, chunks)
            dt = time.perf_counter() - t0
            if step >= args.warmup:
                times.append(dt)
                conv += sum(sum(r) for r in res)
    value = conv / sum(times)
    desc = learned_name(args) if args.workload == "learned" else workload_name(args)
    print(json.dumps({
        "impl": "reference", "metric": LEARNED_METRIC if args.workload == "learned" else METRIC, "value": value,
        "unit": UNIT, "n_gpus": wsize, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
        "config": {"workload": desc, "reference_path": "FireCore has no learned warm start: its plain FIRE relaxation "
                                                       "(run_no_omp semantics: all pairs x 9 PBC images, no force clamp, "
                                                       "sum f^2 < Fconv^2) on the same molecules"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": len(chunks), "kind": "reference",
                         "sample": f"first {nsample} of the molecules per step, MolWorld_sp3::run_no_omp (FP64, "
                                   f"compiled from the reference sources), {len(chunks)} processes, CPU: {model}"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def main():
    global MAXSTEPS
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None, help="timed steps (default 3 learned, 5 otherwise)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nsys", type=int, default=None, help="systems per GPU (default 4096 replicas; a 32768-system queue uneven; 16384 learned)")
    ap.add_argument("--workload", default="learned", choices=["learned", "replicas", "uneven"])
    ap.add_argument("--train-sys", type=int, default=2048,
                    help="--workload learned: systems whose trajectories train the network")
    ap.add_argument("--train-steps", type=int, default=2000)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--terms", default="all", choices=["all", "pairs"],
                    help="replicas / uneven: 'pairs' runs the relax kernels with the pair term alone (profiling only)")
    ap.add_argument("--no-refsem", action="store_true",
                    help="--workload learned: skip the GPU run on the reference's semantics")
    ap.add_argument("--no-tune", action="store_true", help="skip the launch-shape autotuner (heuristic shapes)")
    ap.add_argument("--tuning", default=None,
                    help="JSON file of launch shapes: loaded if it exists, else written by the autotuner")
    ap.add_argument("--maxsteps", type=int, default=MAXSTEPS, help="FIRE step limit per system (profiling runs use fewer)")
    args = ap.parse_args()
    MAXSTEPS = args.maxsteps
    if args.nsys is None:
        args.nsys = {"learned": 16384, "uneven": 32768}.get(args.workload, 4096)
    if args.steps is None:
        args.steps = 3 if args.workload == "learned" else 5
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "learned":
        run_learned(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
