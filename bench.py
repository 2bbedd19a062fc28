#!/usr/bin/env python
"""Relaxed systems/s to max|F| < 1e-4 eV/A on B200 (plain batched FIRE path).

Workload (N=1): 4096 replicas of one seeded 60-atom molecule (C:N:O:H =
10:2:2:10), random rigid rotation + 0.15 A noise, 3 A above a rigid rock-salt
slab (a = 5.64 A, 3 layers, 4x4 cells, +-0.9 e), B-spline GridFF 226x226x200
(0.1 A), LJ + Coulomb pairs with a 10 A cutoff over x,y PBC images, FP32
forces / FP64 FIRE reductions, FIRE dt 0.1 with the 10 eV/A force clamp, at
most 4000 steps per system.

One bench step = one full relaxation of the batch from its initial state (the
persistent kernel retires converged systems and claims the next ones).
value = converged systems / device time of the timed steps, all ranks
(one process per GPU, independent systems per rank: weak scaling).

--impl reference times FireCore's own FP64 CPU relaxation (oracle/_ref, the
reference's MolWorld_sp3::run_no_omp compiled from its sources) on the box's
host cores, on a bounded sample of the same systems.
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


def env_rank():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def workload(rank, nsys):
    from firecore_b200 import systems as S
    sub = S.make_slab()                      # 226 x 226 x 200, nPBC_coul (25,25,0)
    batch = S.config_replicas(seed=1 + 7919 * rank, nrep=nsys)
    return sub, batch


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
    from firecore_b200.world import DEFAULT_FLAGS, FireParams, World
    lib = _lib.load()
    sub, batch = workload(rank, args.nsys)
    w = World(lrank)
    t0 = time.perf_counter()
    C = w.grid_build(sub, return_coefs=True)
    w.sync()
    grid_build_s = time.perf_counter() - t0
    w.set_params(flags=DEFAULT_FLAGS, npbc=(1, 1, 0), Rcut=RCUT)
    w.set_fire(FireParams(Flim=FLIM))
    w.upload(batch)
    nsys = batch.nsys
    natoms = batch.natoms.astype(np.int64)
    # counting pass (untimed): algorithmic work of one relaxation of this batch
    lib.mmff_set_counting(1)
    w.restore(); w.relax(MAXSTEPS, FCONV, 1)
    cnt = (np.ctypeslib.ctypes.c_ulonglong * 3)()
    lib.mmff_get_counters(np.ctypeslib.ctypes.cast(cnt, np.ctypeslib.ctypes.c_void_p))
    pair_images, grid_samples, force_evals = int(cnt[0]), int(cnt[1]), int(cnt[2])
    lib.mmff_set_counting(0)
    st0 = w.state()
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
    # aggregate over ranks: converged systems summed, time = max over ranks
    tot_conv, t_max = conv, t_dev
    if dist:
        tt = torch.tensor([float(conv), t_dev], device="cuda", dtype=torch.float64)
        c_t = tt[0:1].clone(); dist.all_reduce(c_t)
        m_t = tt[1:2].clone(); dist.all_reduce(m_t, op=dist.ReduceOp.MAX)
        tot_conv, t_max = float(c_t.item()), float(m_t.item())
        if e2e:
            ee = torch.tensor([e2e["value"]], device="cuda", dtype=torch.float64)
            dist.all_reduce(ee)
            e2e["value"] = float(ee.item())
    value = tot_conv / t_max
    ms_step = 1e3 * t_max / args.steps
    # roofline of the relax kernel: pair term on FP32 CUDA cores
    fp32_peak = lib.mmff_peak_fp32()
    l2_peak = lib.mmff_peak_l2(64)
    t_launch = t_dev / args.steps
    achieved_tf = PAIR_FLOPS * pair_images / t_launch / 1e12
    grid_gbs = GRID_BYTES * grid_samples / t_launch / 1e9
    out = None
    if rank == 0:
        cpu = cpu_baseline(batch, sub, C, args) if not args.no_cpu else None
        nconv0 = int((st0["status"] == 1).sum())
        steps_conv = st0["nsteps"][st0["status"] == 1]
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": wsize, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 forces / f64 FIRE reductions", "data": "synthetic (seeded generator)",
            "config": {"workload": f"{args.nsys} replicas x 60-atom molecule on NaCl slab, GridFF 226x226x200, "
                                   f"Rcut {RCUT} A, Fmax<{FCONV}, <= {MAXSTEPS} FIRE steps",
                       "systems_per_gpu": args.nsys, "l2": "flushed (256 MB write) before every step",
                       "parallelism": f"replicas x{wsize}"},
            "converged_per_step": conv / args.steps, "nan_per_step": nans / args.steps,
            "median_steps_to_converge": float(np.median(steps_conv)) if len(steps_conv) else None,
            "converged_fraction": nconv0 / nsys,
            "grid_build_s": grid_build_s, "wall_s_timed": t_wall,
            "gpu_launches": args.steps * len(w.buckets()),
            "roofline": {"bound": "fp32", "achieved": achieved_tf, "peak": fp32_peak, "unit": "TFLOP/s",
                         "frac": achieved_tf / fp32_peak if fp32_peak > 0 else None, "traffic": None,
                         "peak_source": "measured FFMA microbenchmark (mmff_peak_fp32) on this GPU",
                         "work": f"{PAIR_FLOPS} flop x {pair_images} pair-images per launch",
                         "grid_l2": {"achieved": grid_gbs, "peak": l2_peak, "unit": "GB/s",
                                     "frac": grid_gbs / l2_peak if l2_peak > 0 else None,
                                     "work": f"{GRID_BYTES} B x {grid_samples} atom samples per launch"}},
            "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks,
            "buckets": w.buckets(),
        }
        print(json.dumps(out))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return out


def cpu_baseline(batch, sub, C, args):
    """The FP64 oracle (OpenMP over systems) on a bounded sample of the same
    workload, same parameters (10 A cutoff, force clamp, Fmax criterion)."""
    from oracle import oracle as O
    model, ncores = cpu_info()
    nsample = int(min(batch.nsys, max(16, 4 * ncores), 256))
    sb = batch.subset(range(nsample))
    P = O.make_params(sub.grid, npbc=(1, 1, 0), Rcut=RCUT)
    F = O.make_fire(Flim=FLIM)
    t0 = time.perf_counter()
    r = O.relax(sb, P, F, C, niter=MAXSTEPS, Fconv=FCONV, conv_mode=1, nthreads=ncores)
    dt = time.perf_counter() - t0
    conv = int((r["converged"] == 1).sum())
    return {"value": conv / dt, "unit": UNIT, "cores": ncores, "kind": "port",
            "sample": f"{nsample} of the systems, full relaxation each ({conv} converged, {dt:.1f} s), CPU: {model}"}


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
    rank, wsize, _ = env_rank()
    if rank != 0:
        return
    from oracle import oracle as O
    model, ncores = cpu_info()
    sub, batch = workload(0, args.nsys)
    # substrate grid (an input of both arms): built once on the GPU in a child
    # process and cached; this process itself never initialises CUDA, so the
    # worker pool below can fork.
    cache = os.path.join(tempfile.gettempdir(), "mmff_grid_226x226x200.npy")
    if not os.path.exists(cache):
        code = ("import sys,numpy as np; sys.path.insert(0,%r); from firecore_b200 import systems as S; "
                "from firecore_b200.world import World; w=World(0); C=w.grid_build(S.make_slab(), return_coefs=True); "
                "np.save(%r, C)") % (ROOT, cache)
        subprocess.check_call([sys.executable, "-c", code])
    C = np.load(cache)
    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libref_harness.so was not built (no reference tree)"}))
        return
    _REF.update(batch=batch, C=C, grid=sub.grid)
    nsample = int(min(batch.nsys, max(8, 2 * ncores)))
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
            if step == 0 and args.warmup > 0:
                pass
    value = conv / sum(times)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": wsize, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
        "config": {"workload": f"{args.nsys} replicas x 60-atom molecule on NaCl slab, GridFF 226x226x200; reference "
                               f"semantics: all pairs x 9 PBC images, no force clamp, sum f^2 < Fconv^2"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": len(chunks), "kind": "reference",
                         "sample": f"{nsample} systems per step, MolWorld_sp3::run_no_omp (FP64, compiled from "
                                   f"the reference sources), {len(chunks)} processes, CPU: {model}"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def main():
    global MAXSTEPS
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nsys", type=int, default=4096)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--maxsteps", type=int, default=MAXSTEPS, help="FIRE step limit per system (profiling runs use fewer)")
    args = ap.parse_args()
    MAXSTEPS = args.maxsteps
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
